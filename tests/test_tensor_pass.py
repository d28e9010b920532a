"""Tensor passes (stages as dense 16 x 16 or 8 x 8 matrices on the tensor
cores) against the oracle: forced wherever a pass allows them
(QCS_TENSOR_ALWAYS for 16 x 16 stages, QCS_TENSOR_ALWAYS_8X8 for 8 x 8),
on registers of 12-24 qubits, with every gate kind of at most two targets,
controls on stage, local and chunk qubits, diagonal runs, mid-circuit
measurements (their collapse rides along as a zeroing diagonal), mappings
and state preparations. Tolerance: complex128 amplitudes to 1e-12, clbits
exactly."""

import numpy as np
import pytest

import qcs_b200
from qcs_b200 import GATES, FUSION_GREEDY, TENSOR_ALWAYS, TENSOR_ALWAYS_8X8, TENSOR_AUTO, TENSOR_NEVER
from qcs_b200 import circuits as C

pytestmark = pytest.mark.gpu

TOL = 1e-12
FORCED = [TENSOR_ALWAYS, TENSOR_ALWAYS_8X8]
TWO_TARGET = sorted(g for g, (_, nt) in GATES.items() if nt <= 2)


def _run(lib, n, circ, tensor=None, seed=1, start=None, mapping=None):
    with qcs_b200.Simulator(lib, n, n, seed=seed, mapping=mapping,
                            fusion=FUSION_GREEDY if tensor is not None else None) as sim:
        if tensor is not None:
            sim.set_tensor_passes(tensor)
        if start is not None:
            sim.set_statevector(start)
        sim.run(circ)
        state = sim.statevector()   # flushes the queue
        stats = sim.stats() if tensor is not None else None
        return state, sim.clbits_string(), stats


def _random_state(n, seed):
    rng = np.random.default_rng(seed)
    v = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    return v / np.linalg.norm(v)


@pytest.mark.parametrize("n", [12, 16, 20])
@pytest.mark.parametrize("mode", FORCED)
def test_layered_circuits(gpu_lib, oracle_lib, n, mode):
    for circ in (C.layered_u3_cz_cx_toffoli(n, 6, seed=n), C.u3_random_matching(n, 6, seed=n + 1),
                 C.layered_u3_cz(n, 6, seed=n + 2)):
        got, _, stats = _run(gpu_lib, n, circ, tensor=mode)
        ref, _, _ = _run(oracle_lib, n, circ)
        assert stats["tensor_passes"] > 0
        assert np.max(np.abs(got - ref)) <= TOL
        assert qcs_b200.fidelity(got, ref) >= 1 - 1e-12


@pytest.mark.parametrize("n", [12, 14, 17])
@pytest.mark.parametrize("mode", FORCED)
def test_every_two_target_gate_kind_with_controls(gpu_lib, oracle_lib, n, mode):
    start = _random_state(n, n)
    for i, name in enumerate(TWO_TARGET):
        circ = C.random_circuit(n, 40, seed=n * 977 + i, max_controls=2, gates=[name, "u3", "h"])
        got, _, _ = _run(gpu_lib, n, circ, tensor=mode, start=start)
        ref, _, _ = _run(oracle_lib, n, circ, start=start)
        assert np.max(np.abs(got - ref)) <= TOL, name


@pytest.mark.parametrize("n", [12, 16, 19])
@pytest.mark.parametrize("mode", FORCED)
def test_mixed_random_circuits(gpu_lib, oracle_lib, n, mode):
    circ = C.random_circuit(n, 300, seed=5000 + n, max_controls=3, gates=TWO_TARGET)
    start = _random_state(n, 3)
    got, _, stats = _run(gpu_lib, n, circ, tensor=mode, start=start)
    ref, _, _ = _run(oracle_lib, n, circ, start=start)
    assert np.max(np.abs(got - ref)) <= TOL
    # the same queue without tensor passes
    plain, _, stats0 = _run(gpu_lib, n, circ, tensor=TENSOR_NEVER, start=start)
    assert stats0["tensor_passes"] == 0
    assert np.max(np.abs(got - plain)) <= TOL


@pytest.mark.parametrize("n", [12, 15])
@pytest.mark.parametrize("mode", FORCED)
def test_measurements_and_resets(gpu_lib, oracle_lib, n, mode):
    circ = [("h", (), (q,), (), ()) for q in range(n)]
    circ += C.random_circuit(n, 150, seed=70 + n, max_controls=2, gates=TWO_TARGET, measure_prob=0.08)
    circ += C.layered_u3_cz(n, 3, seed=n)
    circ += [("measure", (q,), (q,), (), ()) for q in range(0, n, 2)]
    circ += C.layered_u3_cz_cx_toffoli(n, 2, seed=n)
    for seed in (11, 12):
        got, gbits, _ = _run(gpu_lib, n, circ, tensor=mode, seed=seed)
        ref, rbits, _ = _run(oracle_lib, n, circ, seed=seed)
        assert gbits == rbits
        assert np.max(np.abs(got - ref)) <= TOL


@pytest.mark.parametrize("mode", FORCED)
def test_mapping_and_qft(gpu_lib, oracle_lib, mode):
    n = 16
    mapping = list(np.random.default_rng(3).permutation(n))
    circ = C.layered_u3_cz_cx_toffoli(n, 5, seed=9) + C.qft(n, seed=2)[0]
    got, _, _ = _run(gpu_lib, n, circ, tensor=mode, mapping=mapping)
    ref, _, _ = _run(oracle_lib, n, circ, mapping=mapping)
    assert np.max(np.abs(got - ref)) <= TOL


def test_twenty_four_qubits_automatic_choice(gpu_lib, oracle_lib):
    n = 24
    circ = C.layered_u3_cz_cx_toffoli(n, 4, seed=21)
    got, _, stats = _run(gpu_lib, n, circ, tensor=TENSOR_AUTO)
    ref, _, _ = _run(oracle_lib, n, circ)
    assert stats["tensor_passes"] > 0
    assert np.max(np.abs(got - ref)) <= TOL
    assert qcs_b200.fidelity(got, ref) >= 1 - 1e-12


@pytest.mark.parametrize("mode", FORCED)
def test_repeated_runs_reuse_matrix_buffer(gpu_lib, oracle_lib, mode):
    """Flushes of different sizes on one simulator (the matrix buffer grows
    between passes) and the |0..0> start of a fresh register."""
    n = 14
    circs = [C.layered_u3_cz(n, 2, seed=1), C.u3_random_matching(n, 12, seed=2), C.layered_u3_cz(n, 1, seed=3)]
    with qcs_b200.Simulator(gpu_lib, n, fusion=FUSION_GREEDY) as sim:
        sim.set_tensor_passes(mode)
        for circ in circs + circs[::-1]:
            sim.set_state("zero")
            sim.run(circ)
            got = sim.statevector()
            ref, _, _ = _run(oracle_lib, n, circ)
            assert np.max(np.abs(got - ref)) <= TOL


def test_tensor_mode_argument_checks(gpu_lib):
    with qcs_b200.Simulator(gpu_lib, 12) as sim:
        with pytest.raises(qcs_b200.QCSError, match="tensor pass mode"):
            sim.set_tensor_passes(4)


def _run64(lib, n, circ, tensor, seed=1, engine=qcs_b200.ENGINE_TCGEN05):
    with qcs_b200.Simulator(lib, n, n, seed=seed, fusion=FUSION_GREEDY, precision=64) as sim:
        sim.set_tensor_passes(tensor)
        sim.set_tensor_engine(engine)
        sim.run(circ)
        state = sim.statevector()
        return state, sim.clbits_string(), sim.stats()


@pytest.mark.parametrize("n", [12, 16, 20])
@pytest.mark.parametrize("mode", FORCED)
def test_complex64_tensor_passes(gpu_lib, oracle_lib, n, mode):
    """complex64 tensor passes (TF32 with a three-term split, FP32
    accumulation): fidelity >= 1 - 1e-6 against the complex128 oracle, as
    for the complex64 register path, and amplitudes within 1e-5."""
    for circ in (C.layered_u3_cz_cx_toffoli(n, 8, seed=n), C.u3_random_matching(n, 8, seed=n + 1),
                 C.random_circuit(n, 200, seed=900 + n, max_controls=2, gates=TWO_TARGET)):
        ref, _, _ = _run(oracle_lib, n, circ)
        got, _, stats = _run64(gpu_lib, n, circ, mode)
        assert stats["tensor_passes"] > 0
        assert qcs_b200.fidelity(got, ref) >= 1 - 1e-6
        assert np.max(np.abs(got - ref)) <= 1e-5
        reg, _, stats0 = _run64(gpu_lib, n, circ, TENSOR_NEVER)
        assert stats0["tensor_passes"] == 0
        assert qcs_b200.fidelity(got, reg) >= 1 - 1e-6


@pytest.mark.parametrize("mode", FORCED)
def test_complex64_measurements(gpu_lib, oracle_lib, mode):
    n = 14
    circ = [("h", (), (q,), (), ()) for q in range(n)]
    circ += C.layered_u3_cz(n, 4, seed=5)
    circ += [("measure", (q,), (q,), (), ()) for q in range(0, n, 3)]
    circ += C.layered_u3_cz_cx_toffoli(n, 3, seed=6)
    ref, rbits, _ = _run(oracle_lib, n, circ, seed=3)
    got, gbits, stats = _run64(gpu_lib, n, circ, mode, seed=3)
    assert stats["tensor_passes"] > 0
    # outcomes follow the same draws unless a probability sits within the
    # complex64 error of a draw (none does for this seed)
    assert gbits == rbits
    assert qcs_b200.fidelity(got, ref) >= 1 - 1e-6


@pytest.mark.parametrize("measure", [False, True])
@pytest.mark.parametrize("mode", FORCED)
def test_complex64_tensor_passes_keep_the_norm(gpu_lib, oracle_lib, measure, mode):
    """Complex64 tensor passes round their FP32 accumulation toward smaller
    magnitudes; each flush that ran them is rescaled to the norm the register
    must have (1, or the kept weight after a measurement, which does not
    renormalise, as in the reference). The raw overlap, not only the
    normalised fidelity, then meets the complex64 bound."""
    n = 20
    circ = C.u3_random_matching(n, 30, seed=7)
    if measure:
        circ = circ[: len(circ) // 2] + [("measure", (3,), (3,), (), ())] + circ[len(circ) // 2:]
    ref, rbits, _ = _run(oracle_lib, n, circ, seed=5)
    got, gbits, stats = _run64(gpu_lib, n, circ, mode, seed=5)
    assert stats["tensor_passes"] > 0
    assert gbits == rbits
    nref = np.vdot(ref, ref).real
    ngot = np.vdot(got, got).real
    assert abs(ngot - nref) <= 1e-6 * nref, (ngot, nref)
    raw = abs(np.vdot(ref, got)) ** 2 / nref ** 2
    assert raw >= 1 - 1e-6, raw


@pytest.mark.parametrize("n", [16, 20])
def test_complex64_tcgen05_passes(gpu_lib, oracle_lib, n):
    """complex64 16 x 16 stages issued as tcgen05.mma (rows in tensor memory,
    TF32 high/low parts, FP32 accumulators in tensor memory) against the
    complex128 oracle, and against the same passes on warp-level mma.sync:
    fidelity >= 1 - 1e-6, amplitudes within 1e-5, as for every complex64
    path. A pass goes to tcgen05 when each of its stages depends on at most
    one local bit outside the stage; the other passes of a circuit stay on
    mma.sync, so the circuits together must have run some on tcgen05."""
    ran = 0
    for circ in (C.layered_u3_cz_cx_toffoli(n, 8, seed=n), C.u3_random_matching(n, 8, seed=n + 1),
                 C.random_circuit(n, 200, seed=900 + n, max_controls=2, gates=TWO_TARGET),
                 C.qft(n, seed=3)[0]):
        ref, _, _ = _run(oracle_lib, n, circ)
        got, _, stats = _run64(gpu_lib, n, circ, TENSOR_ALWAYS)
        ran += stats["tcgen05_passes"]
        assert qcs_b200.fidelity(got, ref) >= 1 - 1e-6
        assert np.max(np.abs(got - ref)) <= 1e-5
        warp, _, stats0 = _run64(gpu_lib, n, circ, TENSOR_ALWAYS, engine=qcs_b200.ENGINE_MMA_SYNC)
        assert stats0["tcgen05_passes"] == 0
        assert qcs_b200.fidelity(got, warp) >= 1 - 1e-6
    assert ran > 0


def test_complex64_tcgen05_measurements_and_norm(gpu_lib, oracle_lib):
    n = 20
    circ = [("h", (), (q,), (), ()) for q in range(n)]
    circ += C.u3_random_matching(n, 10, seed=4)
    circ += [("measure", (q,), (q,), (), ()) for q in range(0, n, 4)]
    circ += C.layered_u3_cz_cx_toffoli(n, 4, seed=8)
    ref, rbits, _ = _run(oracle_lib, n, circ, seed=9)
    got, gbits, stats = _run64(gpu_lib, n, circ, TENSOR_ALWAYS, seed=9)
    assert stats["tensor_passes"] > 0
    assert gbits == rbits
    nref = np.vdot(ref, ref).real
    assert abs(np.vdot(got, got).real - nref) <= 1e-6 * nref
    assert abs(np.vdot(ref, got)) ** 2 / nref ** 2 >= 1 - 1e-6


def test_tensor_engine_argument_checks(gpu_lib):
    with qcs_b200.Simulator(gpu_lib, 12) as sim:
        with pytest.raises(qcs_b200.QCSError, match="tensor engine"):
            sim.set_tensor_engine(2)
