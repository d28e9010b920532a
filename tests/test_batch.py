"""Batches of independent circuits (qcs_b200_batch_*) against the oracle run
circuit by circuit: registers, <Z_q>, parameter updates, the shared plans of
circuits with the same structure, and the argument checks."""

import numpy as np
import pytest

import qcs_b200
from qcs_b200 import GATES
from qcs_b200 import circuits as C

pytestmark = pytest.mark.gpu

TWO_TARGET_GATES = sorted(g for g, (_, nt) in GATES.items() if nt <= 2)


def _oracle_state(oracle_lib, n, circ):
    with qcs_b200.Simulator(oracle_lib, n) as sim:
        sim.run(circ)
        return sim.statevector()


def _z_from_state(v, n):
    p = np.abs(v) ** 2
    idx = np.arange(v.size)
    tot = p.sum()
    return np.array([(tot - 2 * p[(idx >> q) & 1 == 1].sum()) / tot for q in range(n)])


def _mixed_circuits():
    circs = []
    for seed, n in enumerate([9, 10, 11, 12, 13, 14]):
        circs.append((n, C.hea_circuit(n, 3 + seed % 3, seed=seed)))
    # same structure as the first three, other parameters: shared plans
    for seed, n in enumerate([9, 10, 11]):
        circs.append((n, C.hea_circuit(n, 3 + seed % 3, seed=100 + seed)))
    for seed, n in enumerate([9, 12, 13]):
        circs.append((n, C.random_circuit(n, 90, seed=40 + seed, max_controls=2, gates=TWO_TARGET_GATES)))
    circs.append((10, C.layered_u3_cz_cx_toffoli(10, 4, seed=3)))
    circs.append((11, C.u3_random_matching(10, 5, seed=4) + [("h", (), (10,), (), ())]))
    return circs


# batch tensor modes: 0 register passes only, 1 tuned per group (default),
# 2 8 x 8 tensor passes wherever a pass allows them (groups of >= 11 qubits)
TENSOR_MODES = [0, 1, 2]


def _check_tensor_mode(info, mode, widest):
    if mode == 0 or widest < 11:
        assert info["tensor_passes"] == 0
    elif mode == 2:
        assert info["tensor_passes"] > 0
    assert info["tensor_passes"] <= info["passes"]


@pytest.mark.parametrize("tensor", TENSOR_MODES)
@pytest.mark.parametrize("precision", [128, 64])
def test_batch_matches_oracle(gpu_lib, oracle_lib, precision, tensor):
    circs = _mixed_circuits()
    with qcs_b200.Batch(gpu_lib, precision) as b:
        b.set_tensor_passes(tensor)
        for n, circ in circs:
            b.add_circuit(n, circ)
        b.run()
        zs = b.expectation_z()
        info = b.info()
        assert info["circuits"] == len(circs)
        assert info["groups"] == len(circs) - 3   # three circuits reuse a plan
        assert info["launches_per_run"] >= info["passes"] > 0
        _check_tensor_mode(info, tensor, max(n for n, _ in circs))
        for i, (n, circ) in enumerate(circs):
            ref = _oracle_state(oracle_lib, n, circ)
            got = b.statevector(i)
            if precision == 128:
                assert np.max(np.abs(got - ref)) <= 1e-12, i
                assert np.max(np.abs(zs[i] - _z_from_state(ref, n))) <= 1e-12, i
            else:
                fid = abs(np.vdot(got, ref)) ** 2 / (np.vdot(got, got).real * np.vdot(ref, ref).real)
                assert fid >= 1 - 1e-6, i
                assert np.max(np.abs(zs[i] - _z_from_state(ref, n))) <= 1e-5, i


@pytest.mark.parametrize("tensor", [0, 2])
@pytest.mark.parametrize("precision", [128, 64])
def test_batch_phase_runs_and_sign_runs(gpu_lib, oracle_lib, precision, tensor):
    """Batched passes with phase runs (QFT controlled phases: explicit terms,
    since entries differ per register), runs of -1 phases (CZ, CCZ) with
    controls on stage, thread and chunk qubits, and pairs / groups of
    one-qubit gates, against the oracle."""
    diag = ["z", "s", "t", "rz", "p", "rzz", "u1"]
    circs = [(13, C.qft(13, seed=5)[0]), (14, C.qft(14, seed=6)[0])]
    for seed, n in enumerate([12, 14]):
        c = []
        for blk in range(6):
            c += C.random_circuit(n, 4, seed=300 + 10 * seed + blk, max_controls=1, gates=["u3", "h", "ry"])
            c += C.random_circuit(n, 12, seed=400 + 10 * seed + blk, max_controls=2, gates=diag)
        circs.append((n, c))
    with qcs_b200.Batch(gpu_lib, precision) as b:
        b.set_tensor_passes(tensor)
        for n, circ in circs:
            b.add_circuit(n, circ)
        b.run()
        _check_tensor_mode(b.info(), tensor, 14)
        for i, (n, circ) in enumerate(circs):
            ref = _oracle_state(oracle_lib, n, circ)
            got = b.statevector(i)
            if precision == 128:
                assert np.max(np.abs(got - ref)) <= 1e-12, i
            else:
                fid = abs(np.vdot(got, ref)) ** 2 / (np.vdot(got, got).real * np.vdot(ref, ref).real)
                assert fid >= 1 - 1e-6, i


@pytest.mark.parametrize("tensor", [0, 2])
def test_batch_parameter_updates(gpu_lib, oracle_lib, tensor):
    shapes = [(9, 2), (12, 3), (9, 2)]
    with qcs_b200.Batch(gpu_lib, 128) as b:
        b.set_tensor_passes(tensor)
        for k, (n, d) in enumerate(shapes):
            b.add_circuit(n, C.hea_circuit(n, d, seed=k))
        nparams = b.info()["parameters"]
        assert nparams == sum(2 * n * d for n, d in shapes)
        b.run()
        for rnd in range(3):
            rng = np.random.default_rng(rnd)
            params = rng.uniform(-np.pi, np.pi, size=nparams)
            if rnd == 1:
                params[: 2 * 9] = 0.0   # identity rotations in a shared plan
            b.set_parameters(params)
            b.run()
            zs = b.expectation_z()
            off = 0
            for i, (n, d) in enumerate(shapes):
                circ = C.hea_circuit(n, d, seed=i)
                fresh, j = [], off
                for op, p, t, ng, ps in circ:
                    fresh.append((op, tuple(params[j:j + len(p)]), t, ng, ps))
                    j += len(p)
                off = j
                ref = _oracle_state(oracle_lib, n, fresh)
                assert np.max(np.abs(b.statevector(i) - ref)) <= 1e-12
                assert np.max(np.abs(zs[i] - _z_from_state(ref, n))) <= 1e-12


def test_batch_rejects_bad_input(gpu_lib):
    with qcs_b200.Batch(gpu_lib, 128) as b:
        with pytest.raises(qcs_b200.QCSError, match="9 to 30 qubits"):
            b.add_circuit(5, [("h", (), (0,), (), ())])
        with pytest.raises(qcs_b200.QCSError, match="at most two targets"):
            b.add_circuit(10, [("rccx", (), (0, 1, 2), (), ())])
        with pytest.raises(qcs_b200.QCSError, match="out of range"):
            b.add_circuit(10, [("h", (), (10,), (), ())])
        with pytest.raises(qcs_b200.QCSError, match="more than once"):
            b.add_circuit(10, [("x", (), (1,), (), (1,))])
        with pytest.raises(qcs_b200.QCSError, match="no circuits"):
            b.run()
        b.add_circuit(10, [("h", (), (0,), (), ())])
        with pytest.raises(qcs_b200.QCSError, match="run the batch first"):
            b.expectation_z()
        with pytest.raises(qcs_b200.QCSError, match="parameters"):
            b.set_parameters([0.5])
        with pytest.raises(qcs_b200.QCSError, match="tensor mode 3"):
            b.set_tensor_passes(3)
        b.run()
        z = b.expectation_z()[0]
        assert abs(z[0]) < 1e-15 and np.all(np.abs(z[1:] - 1) < 1e-15)
    with pytest.raises(qcs_b200.QCSError, match="precision"):
        qcs_b200.Batch(gpu_lib, 32)


def test_batch_of_identity_circuits(gpu_lib):
    # registers without any gate still start from |0..0>
    with qcs_b200.Batch(gpu_lib, 64) as b:
        b.add_circuit(9, [])
        b.add_circuit(10, [("x", (), (3,), (), ())])
        b.run()
        v = b.statevector(0)
        assert v[0] == 1 and np.count_nonzero(v) == 1
        z = b.expectation_z()
        assert np.all(z[0] == 1.0)
        assert z[1][3] == -1.0 and np.all(np.delete(z[1], 3) == 1.0)


def test_batch_failed_build_releases_memory(gpu_lib):
    """A build that stops part way (here: a circuit whose gate entries exceed
    one register's entry block, found after the register arena is allocated)
    must not leak that arena when run() is retried."""
    import torch

    big = 24   # a 256 MiB complex128 register makes a leaked arena visible
    too_many = [("u3", (0.1 * i, 0.2, 0.3), (i % 9,), (), ()) for i in range(17000)]
    with qcs_b200.Batch(gpu_lib, 128) as b:
        b.add_circuit(big, [("h", (), (0,), (), ())])
        b.add_circuit(9, too_many)
        with pytest.raises(qcs_b200.QCSError, match="too many gate entries"):
            b.run()
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        for _ in range(3):
            with pytest.raises(qcs_b200.QCSError, match="too many gate entries"):
                b.run()
        torch.cuda.synchronize()
        free_after = torch.cuda.mem_get_info()[0]
    assert free_before - free_after < (64 << 20), (free_before, free_after)


@pytest.mark.parametrize("tensor", TENSOR_MODES)
@pytest.mark.parametrize("precision", [128, 64])
def test_batch_multi_chunk_registers(gpu_lib, oracle_lib, precision, tensor):
    """The batch workload's widest registers (15-20 qubits, depth 8: 16 to
    512 chunks per register in the batched pass), including two circuits of
    one structure, against the oracle: states, and <Z_q> of every qubit."""
    widths = [15, 16, 17, 18, 19, 20, 17]
    circs = [(w, C.hea_circuit(w, 8, seed=500 + i)) for i, w in enumerate(widths)]
    with qcs_b200.Batch(gpu_lib, precision) as b:
        b.set_tensor_passes(tensor)
        for n, circ in circs:
            b.add_circuit(n, circ)
        b.run()
        zs = b.expectation_z()
        assert b.info()["groups"] == len(circs) - 1
        _check_tensor_mode(b.info(), tensor, max(widths))
        for i, (n, circ) in enumerate(circs):
            ref = _oracle_state(oracle_lib, n, circ)
            got = b.statevector(i)
            zref = _z_from_state(ref, n)
            if precision == 128:
                assert np.max(np.abs(got - ref)) <= 1e-12, i
                assert np.max(np.abs(zs[i] - zref)) <= 1e-12, i
            else:
                fid = abs(np.vdot(got, ref)) ** 2 / (np.vdot(got, got).real * np.vdot(ref, ref).real)
                assert fid >= 1 - 1e-6, (i, fid)
                assert np.max(np.abs(zs[i] - zref)) <= 1e-5, i
