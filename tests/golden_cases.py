"""Circuits whose outputs are pinned by fixtures from the reference build.

Each case is a dict: name, n, num_clbits, seed (measurement engine seed),
mapping (or None), prep (state preparation before the circuit), circuit,
samples (number of bin/qcs-style repetitions; 1 = run once). The reference
run (tests/golden/make_golden.py) and the tests both build the cases from
this module, so they see identical doubles.
"""

import sys
from pathlib import Path

sys.path.insert(0, str(Path(__file__).resolve().parent.parent / "rqs-svg_b200"))

from qcs_b200 import GATES  # noqa: E402
from qcs_b200 import circuits as C  # noqa: E402

SEED = 12345   # value the seed shim hands to std::random_device


def _h_all(n):
    return [("h", (), (q,), (), ()) for q in range(n)]


def cases():
    out = []
    # every gate kind, several placements, with positive and negative controls
    for i, name in enumerate(sorted(GATES)):
        n = 7
        circ = _h_all(n) + C.random_circuit(n, 3, seed=100 + i, max_controls=0, gates=["u3"])
        circ += C.random_circuit(n, 12, seed=200 + i, max_controls=3, gates=[name])
        out.append(dict(name=f"gate_{name}", n=n, num_clbits=0, mapping=None, prep="zero", circuit=circ, samples=1))
    # mixed random circuits
    for n, g, s in [(5, 80, 1), (8, 150, 2), (10, 200, 3)]:
        out.append(dict(name=f"random_n{n}", n=n, num_clbits=0, mapping=None, prep="zero",
                        circuit=C.random_circuit(n, g, seed=s, max_controls=3), samples=1))
    # measurement semantics: interleaved measurements, measured qubits as
    # implicit controls, contradicting controls, re-measurement
    for n, s in [(6, 11), (8, 12)]:
        circ = _h_all(n) + C.random_circuit(n, 60, seed=s, max_controls=2, measure_prob=0.15,
                                            gates=["h", "u3", "x", "rx", "rz", "p", "sx", "ry"])
        circ += [("measure", (q,), (q,), (), ()) for q in range(n)]
        out.append(dict(name=f"measure_n{n}", n=n, num_clbits=n, mapping=None, prep="zero", circuit=circ, samples=4))
    # GHZ and bin/qcs-style repeated shots of a layered circuit
    n = 6
    ghz = [("h", (), (0,), (), ())] + [("x", (), (q,), (), (0,)) for q in range(1, n)]
    ghz += [("measure", (q,), (q,), (), ()) for q in range(n)]
    out.append(dict(name="ghz_shots", n=n, num_clbits=n, mapping=None, prep="zero", circuit=ghz, samples=16))
    out.append(dict(name="layered_shots", n=10, num_clbits=10, mapping=None, prep="zero",
                    circuit=C.layered_u3_cz(10, 6, seed=5, measure=True), samples=64))
    out.append(dict(name="layered_state", n=12, num_clbits=0, mapping=None, prep="zero",
                    circuit=C.layered_u3_cz(12, 8, seed=6), samples=1))
    out.append(dict(name="plain_at_scale_small", n=11, num_clbits=0, mapping=None, prep="zero",
                    circuit=C.layered_u3_cz_cx_toffoli(11, 6, seed=7), samples=1))
    qc, _ = C.qft(9, seed=8)
    out.append(dict(name="qft9", n=9, num_clbits=0, mapping=None, prep="zero", circuit=qc, samples=1))
    # mappings: gates on logical qubits, file written in logical order
    out.append(dict(name="mapping_perm", n=7, num_clbits=0, mapping=[3, 0, 6, 1, 5, 2, 4], prep="zero",
                    circuit=C.random_circuit(7, 60, seed=21, max_controls=2), samples=1))
    out.append(dict(name="mapping_measure", n=6, num_clbits=6, mapping=[5, 4, 3, 2, 1, 0], prep="zero",
                    circuit=_h_all(6) + C.random_circuit(6, 30, seed=22, max_controls=1, measure_prob=0.2,
                                                         gates=["u3", "x", "rz"])
                    + [("measure", (q,), (q,), (), ()) for q in range(6)], samples=3))
    # state preparations
    for prep in ("sequential", "flat", "random"):
        out.append(dict(name=f"prep_{prep}", n=6, num_clbits=0, mapping=None, prep=prep,
                        circuit=C.random_circuit(6, 20, seed=31, max_controls=1), samples=1))
    out.append(dict(name="prep_entangled", n=5, num_clbits=0, mapping=None, prep="entangled_after_gates",
                    circuit=C.random_circuit(5, 20, seed=32, max_controls=1), samples=1))
    # reset
    circ = _h_all(5) + [("u3", (0.3, 0.2, 0.1), (1,), (), ())]
    out.append(dict(name="reset", n=5, num_clbits=0, mapping=None, prep="reset", circuit=circ, samples=1))
    return out


def run_case(sim, case):
    """Execute one case on an allocated Simulator the way bin/qcs would
    (src/qcs_main.cpp:153-193). Returns (clbit strings per sample, state)."""
    shots = []
    for k in range(case["samples"]):
        prep = case["prep"]
        if prep in ("sequential", "flat", "random"):
            sim.set_state(prep)
        if prep == "entangled_after_gates":
            sim.run(case["circuit"])
            sim.set_state("entangled")
        elif prep == "reset":
            sim.run(case["circuit"])
            sim.reset(1)
            sim.reset(3)
        else:
            sim.run(case["circuit"])
        if case["num_clbits"]:
            shots.append(sim.clbits_string())
        if k != case["samples"] - 1:
            sim.reinitialize_mapping()
            sim.set_state("zero")
            sim.reset_clbits()
            sim.reset_measurement_state()
    return shots, sim.statevector()
