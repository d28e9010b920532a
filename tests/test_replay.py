"""Kept flush plans and the collapse-only flush.

A flush whose queue was seen before (the same ops with the same matrices,
bit for bit: a circuit re-run for every sample, as `bin/qcs` does) launches
the kept plan without planning. The replayed run must equal the planned run
bit for bit and the oracle to 1e-12, across register passes, phase-run
tables (QFT), plain gate steps, 8 x 8 tensor passes on the FP64 tensor cores
and complex64 tcgen05 passes. A queue that differs in one parameter is
planned anew. A flush that holds only the collapses of measurements runs as
one masked write pass; its state and clbits equal the oracle's.
"""

import numpy as np
import pytest

import qcs_b200
from qcs_b200 import circuits as C

pytestmark = pytest.mark.gpu

CASES = {
    "layered": (16, lambda: C.layered_u3_cz(16, 8, seed=11), qcs_b200.TENSOR_NEVER, 128),
    "qft_tables": (16, lambda: C.qft(16, seed=3)[0], qcs_b200.TENSOR_NEVER, 128),
    "random_plain_steps": (14, lambda: C.random_circuit(14, 300, seed=9, max_controls=3), qcs_b200.TENSOR_AUTO, 128),
    "tensor8": (18, lambda: C.layered_u3_cz_cx_toffoli(18, 4, seed=5), qcs_b200.TENSOR_ALWAYS_8X8, 128),
    "tcgen05_c64": (18, lambda: C.layered_u3_cz_cx_toffoli(18, 4, seed=5), qcs_b200.TENSOR_ALWAYS, 64),
}


def _oracle_state(oracle_lib, n, circ):
    with qcs_b200.Simulator(oracle_lib, n) as sim:
        sim.run(circ)
        return sim.statevector()


@pytest.mark.parametrize("case", sorted(CASES))
def test_replayed_flush_equals_planned(gpu_lib, oracle_lib, case):
    n, make, mode, precision = CASES[case]
    circ = make()
    with qcs_b200.Simulator(gpu_lib, n, fusion=qcs_b200.FUSION_GREEDY, precision=precision) as sim:
        sim.set_tensor_passes(mode)
        sim.run(circ)
        first = sim.statevector()
        s1 = sim.stats()
        sim.set_state("zero")
        sim.run(circ)
        second = sim.statevector()
        s2 = sim.stats()
        # the plan's own stage matrices, built on its first replay, serve
        # the later ones: no matrix builds from the second replay on
        sim.set_state("zero")
        sim.run(circ)
        third = sim.statevector()
        s3 = sim.stats()
    assert s1["replayed_flushes"] == 0
    assert s2["replayed_flushes"] == 1 and s3["replayed_flushes"] == 2
    launches2 = s2["kernel_launches"] - s1["kernel_launches"]
    launches3 = s3["kernel_launches"] - s2["kernel_launches"]
    if s1["tensor_passes"] > 0:
        assert launches3 == launches2 - s1["tensor_passes"]
    else:
        assert launches3 == launches2
    assert third.tobytes() == first.tobytes()
    # the same launches: the same passes of each kind, bit-identical results
    for key in ("fused_passes", "tensor_passes", "tensor8_passes", "tcgen05_passes", "plain_gate_kernels"):
        assert s2[key] == 2 * s1[key], key
    assert first.tobytes() == second.tobytes()
    ref = _oracle_state(oracle_lib, n, circ)
    if precision == 128:
        assert float(np.max(np.abs(second - ref))) <= 1e-12
    else:
        assert qcs_b200.fidelity(second, ref) >= 1 - 1e-6
    if case == "tensor8":
        assert s1["tensor8_passes"] > 0
    if case == "tcgen05_c64":
        assert s1["tcgen05_passes"] > 0


def test_changed_parameter_is_planned_anew(gpu_lib, oracle_lib):
    n = 16
    circ = C.layered_u3_cz(n, 6, seed=2)
    # the same structure, one rotation angle changed (a change in the last
    # bit of an angle may leave the gate's matrix, and so the plan, as it is)
    changed = list(circ)
    for i, g in enumerate(changed):
        if g[0] == "u3":
            params = list(g[1])
            params[0] += 0.25
            changed[i] = (g[0], tuple(params)) + tuple(g[2:])
            break
    assert changed != circ
    with qcs_b200.Simulator(gpu_lib, n, fusion=qcs_b200.FUSION_GREEDY) as sim:
        sim.run(circ)
        sim.synchronize()
        sim.set_state("zero")
        sim.run(changed)
        got = sim.statevector()
        assert sim.stats()["replayed_flushes"] == 0
        sim.set_state("zero")
        sim.run(changed)
        again = sim.statevector()
        assert sim.stats()["replayed_flushes"] == 1
    ref = _oracle_state(oracle_lib, n, changed)
    assert float(np.max(np.abs(got - ref))) <= 1e-12
    assert got.tobytes() == again.tobytes()


@pytest.mark.parametrize("precision", [128, 64])
def test_collapse_only_flush(gpu_lib, oracle_lib, precision):
    """Samples of a measured circuit: gates, then every qubit measured, the
    state read (a flush of collapses only), reset; repeated so that later
    samples replay the kept plan. States and clbits against the oracle."""
    n = 14
    circ = C.layered_u3_cz(n, 6, seed=4)
    meas = [("measure", (q,), (q,), (), ()) for q in range(n)]
    seed = 77
    got_bits, got_states = [], []
    with qcs_b200.Simulator(gpu_lib, n, n, seed=seed, fusion=qcs_b200.FUSION_GREEDY, precision=precision) as sim:
        for _ in range(3):
            sim.run(circ + meas)
            got_bits.append(sim.clbits_string())
            got_states.append(sim.statevector())
            sim.set_state("zero")
            sim.reset_clbits()
            sim.reset_measurement_state()
        replayed = sim.stats()["replayed_flushes"]
    ref_bits, ref_states = [], []
    with qcs_b200.Simulator(oracle_lib, n, n, seed=seed) as sim:
        for _ in range(3):
            sim.run(circ + meas)
            ref_bits.append(sim.clbits_string())
            ref_states.append(sim.statevector())
            sim.set_state("zero")
            sim.reset_clbits()
            sim.reset_measurement_state()
    assert replayed == 2
    assert got_bits == ref_bits
    tol = 1e-12 if precision == 128 else 1e-6
    for got, ref in zip(got_states, ref_states):
        assert float(np.max(np.abs(got - ref))) <= tol
        # one amplitude is left: the measured basis state
        assert np.count_nonzero(got) == 1
