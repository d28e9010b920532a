"""complex64 registers (a B200 extension; the reference is complex128 only).

Gate arithmetic runs in FP32, so results are compared with the complex128
oracle by fidelity (>= 1 - 1e-6) and by a max amplitude error bound scaled
to the circuit length; reductions (norms, <Z>, probabilities) accumulate in
FP64. Both execution modes are covered.
"""

import os
import tempfile

import numpy as np
import pytest

import qcs_b200
from qcs_b200 import FUSION_GREEDY, FUSION_PLAIN, GATES
from qcs_b200 import circuits as C

pytestmark = pytest.mark.gpu

MODES = [FUSION_PLAIN, FUSION_GREEDY]
FID = 1e-6


def _run(lib, n, circ, precision=None, fusion=None, seed=1, mapping=None, start=None):
    with qcs_b200.Simulator(lib, n, n, seed=seed, mapping=mapping, fusion=fusion, precision=precision) as sim:
        if start is not None:
            sim.set_statevector(start)
        sim.run(circ)
        return sim.statevector(), sim.clbits_string()


def _random_state(n, seed):
    rng = np.random.default_rng(seed)
    v = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    return v / np.linalg.norm(v)


def test_precision_is_reported(gpu_lib):
    import ctypes

    with qcs_b200.Simulator(gpu_lib, 4, precision=64) as sim:
        bits = ctypes.c_int()
        gpu_lib.call("qcs_simulator_get_precision", sim.h, ctypes.byref(bits))
        assert bits.value == 64
    sim = qcs_b200.Simulator(gpu_lib, 4, allocate=False)
    with pytest.raises(qcs_b200.QCSError, match="precision"):
        gpu_lib.call("qcs_simulator_set_precision", sim.h, 32)
    sim.close()


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("name", sorted(GATES))
def test_every_gate_kind_c64(gpu_lib, oracle_lib, name, mode):
    for n in (3, 9, 13):
        circ = C.random_circuit(n, 30, seed=n * 7 + sum(map(ord, name)), max_controls=3, gates=[name])
        start = _random_state(n, n)
        got, _ = _run(gpu_lib, n, circ, precision=64, fusion=mode, start=start)
        ref, _ = _run(oracle_lib, n, circ, start=start)
        assert qcs_b200.fidelity(got, ref) >= 1 - FID
        assert np.max(np.abs(got - ref)) <= 1e-5


@pytest.mark.parametrize("mode", MODES)
def test_deep_circuits_c64(gpu_lib, oracle_lib, mode):
    n = 20
    for circ in (C.u3_random_matching(n, 12, seed=3), C.qft(n, seed=4)[0], C.layered_u3_cz_cx_toffoli(n, 8, seed=5)):
        got, _ = _run(gpu_lib, n, circ, precision=64, fusion=mode)
        ref, _ = _run(oracle_lib, n, circ)
        assert qcs_b200.fidelity(got, ref) >= 1 - FID
        assert abs(np.vdot(got, got).real - 1.0) <= 1e-5


@pytest.mark.parametrize("mode", MODES)
def test_mapping_file_and_expectation_c64(gpu_lib, oracle_lib, mode):
    n = 11
    mapping = [5, 2, 9, 0, 10, 1, 7, 3, 8, 4, 6]
    circ = C.layered_u3_cz(n, 4, seed=8)
    with tempfile.TemporaryDirectory() as d:
        out = []
        for lib, prec in ((gpu_lib, 64), (oracle_lib, None)):
            with qcs_b200.Simulator(lib, n, mapping=mapping, precision=prec, fusion=mode if prec else None) as sim:
                sim.run(circ)
                p = os.path.join(d, f"{len(out)}.bin")
                sim.save_statevector(p)
                z, norm = sim.expectation_z()
                out.append((np.fromfile(p, dtype=np.complex128), z, norm))
    assert out[0][0].size == 1 << n
    assert qcs_b200.fidelity(out[0][0], out[1][0]) >= 1 - FID
    assert np.max(np.abs(out[0][1] - out[1][1])) <= 1e-5
    assert abs(out[0][2] - out[1][2]) <= 1e-5


def test_sampler_and_measurement_c64(gpu_lib, oracle_lib):
    # FP32 amplitudes move P0 by ~1e-7 relative; a draw closer than that to
    # the boundary could flip, which these seeds do not hit
    n = 10
    circ = C.layered_u3_cz(n, 3, seed=2)
    with qcs_b200.Simulator(gpu_lib, n, seed=77, precision=64) as sim:
        sim.run(circ)
        got = [int(v) for v in sim.sample(128)]
    with qcs_b200.Simulator(oracle_lib, n, seed=77) as sim:
        sim.run(circ)
        ref = [int(v) for v in sim.sample(128)]
    assert got == ref
    meas = circ + [("measure", (q,), (q,), (), ()) for q in range(n)]
    _, bits64 = _run(gpu_lib, n, meas, precision=64, seed=5)
    _, bits128 = _run(oracle_lib, n, meas, seed=5)
    assert bits64 == bits128


@pytest.mark.parametrize("prep", ["zero", "flat", "sequential"])
def test_state_preparations_c64(gpu_lib, oracle_lib, prep):
    n = 8
    out = []
    for lib, prec in ((gpu_lib, 64), (oracle_lib, None)):
        with qcs_b200.Simulator(lib, n, precision=prec) as sim:
            sim.set_state(prep)
            out.append(sim.statevector())
    assert np.array_equal(out[0], out[1])
