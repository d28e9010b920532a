"""CPU tests of the oracle: against an independent dense-matrix statement of
every gate, against the reference's documented semantics, and against the
golden fixtures produced by the reference library itself."""

import hashlib
import math
from pathlib import Path

import numpy as np
import pytest

import dense_reference as dr
import golden_cases
import qcs_b200
from qcs_b200 import GATES
from qcs_b200 import circuits as C

GOLDEN = Path(__file__).resolve().parent / "golden" / "reference_golden.npz"


def _random_state(n, seed):
    rng = np.random.default_rng(seed)
    v = rng.normal(size=1 << n) + 1j * rng.normal(size=1 << n)
    return v / np.linalg.norm(v)


@pytest.mark.parametrize("name", sorted(GATES))
def test_oracle_gate_matches_dense_definition(oracle_lib, name):
    n = 5
    circ = C.random_circuit(n, 25, seed=sum(map(ord, name)), max_controls=3, gates=[name])
    start = _random_state(n, 3)
    with qcs_b200.Simulator(oracle_lib, n) as sim:
        sim.set_statevector(start)
        sim.run(circ)
        got = sim.statevector()
    ref = start.copy()
    for op, params, t, neg, pos in circ:
        ref = dr.apply(ref, n, op, params, t, neg, pos)
    assert np.max(np.abs(got - ref)) <= 1e-13


def test_oracle_mixed_random_circuit_with_mapping(oracle_lib):
    n = 6
    circ = C.random_circuit(n, 120, seed=9, max_controls=3)
    start = _random_state(n, 4)
    mapping = [2, 5, 0, 4, 1, 3]
    with qcs_b200.Simulator(oracle_lib, n, mapping=mapping) as sim:
        sim.set_statevector(start)
        sim.run(circ)
        got = sim.statevector()
    ref = start.copy()
    for op, params, t, neg, pos in circ:
        ref = dr.apply(ref, n, op, params, t, neg, pos)
    assert np.max(np.abs(got - ref)) <= 1e-12


def test_oracle_ghz_outcomes_are_all_equal(oracle_lib):
    n = 6
    for seed in range(20):
        with qcs_b200.Simulator(oracle_lib, n, n, seed=seed) as sim:
            sim.gate("h", (), (0,))
            for q in range(1, n):
                sim.gate("x", (), (q,), (), (0,))
            bits = [sim.measure_to_clbit(q, q) for q in range(n)]
            assert len(set(bits)) == 1
            assert sim.clbits_string() == str(bits[0]) * n


def test_oracle_remeasure_is_cached_without_a_draw(oracle_lib):
    # src/qcs.cu:2548-2562: a measured qubit returns its value with no RNG draw,
    # so measuring q twice then r equals measuring q then r.
    a, b = [], []
    for twice in (True, False):
        with qcs_b200.Simulator(oracle_lib, 3, seed=77) as sim:
            for q in range(3):
                sim.gate("h", (), (q,))
            first = sim.measure(0)
            if twice:
                assert sim.measure(0) == first
            (a if twice else b).append((first, sim.measure(1), sim.measure(2)))
    assert a == b


def test_oracle_contradicting_control_skips_gate(oracle_lib):
    # qubit 0 measured as v; a gate controlled on 1-v is cancelled
    with qcs_b200.Simulator(oracle_lib, 2, seed=5) as sim:
        sim.gate("h", (), (0,))
        v = sim.measure(0)
        before = sim.statevector()
        # control on the opposite value: |1> when 0 was measured, |0> otherwise
        neg = () if v == 0 else (0,)
        pos = (0,) if v == 0 else ()
        sim.gate("x", (), (1,), neg, pos)
        after = sim.statevector()
    assert np.array_equal(before, after)


def test_oracle_measurement_is_not_renormalised(oracle_lib):
    with qcs_b200.Simulator(oracle_lib, 1, seed=3) as sim:
        sim.gate("h", (), (0,))
        v = sim.measure(0)
        sv = sim.statevector()
    assert abs(abs(sv[v]) - math.sqrt(0.5)) < 1e-15 and sv[1 - v] == 0


def test_oracle_gate_on_measured_target_unmeasures_it(oracle_lib):
    with qcs_b200.Simulator(oracle_lib, 1, seed=3) as sim:
        sim.gate("h", (), (0,))
        sim.measure(0)
        sim.gate("h", (), (0,))
        # a fresh draw happens now: the state is no longer a basis state
        sv = sim.statevector()
        assert abs(sv[0]) > 0 and abs(sv[1]) > 0


def test_oracle_sample_equals_repeated_measurement(oracle_lib):
    n = 5
    circ = C.layered_u3_cz(n, 4, seed=2)
    with qcs_b200.Simulator(oracle_lib, n, seed=99) as sim:
        sim.run(circ)
        shots = sim.sample(32)
    seq = []
    with qcs_b200.Simulator(oracle_lib, n, n, seed=99) as sim:
        for _ in range(32):
            sim.run(circ)
            seq.append(sum(sim.measure(q) << q for q in range(n)))
            sim.set_state("zero")
            sim.reset_measurement_state()
    assert [int(s) for s in shots] == seq


def test_oracle_errors_are_reported(oracle_lib):
    with qcs_b200.Simulator(oracle_lib, 3) as sim:
        with pytest.raises(qcs_b200.QCSError, match="target"):
            sim.gate("swap", (), (0,))
        with pytest.raises(qcs_b200.QCSError, match="out of range"):
            sim.gate("h", (), (3,))
        with pytest.raises(qcs_b200.QCSError, match="more than once"):
            sim.gate("x", (), (1,), (), (1,))


def test_mlp_oracle_gradient_matches_finite_differences():
    import sys as _sys

    _sys.path.insert(0, str(Path(__file__).resolve().parent.parent / "oracle"))
    import mlp_oracle

    rng = np.random.default_rng(0)
    params = rng.normal(scale=0.3, size=mlp_oracle.NPARAMS)
    x = rng.normal(size=(7, mlp_oracle.IN))
    t = rng.normal(size=7)
    _, g = mlp_oracle.loss_and_gradients(params, x, t)
    idx = rng.choice(mlp_oracle.NPARAMS, size=60, replace=False)
    eps = 1e-6
    for i in idx:
        p1, p2 = params.copy(), params.copy()
        p1[i] += eps
        p2[i] -= eps
        fd = (mlp_oracle.loss_and_gradients(p1, x, t)[0] - mlp_oracle.loss_and_gradients(p2, x, t)[0]) / (2 * eps)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(g[i]))


# ------------------------------------------------------------ golden fixtures


def _golden():
    if not GOLDEN.exists():
        pytest.fail(f"{GOLDEN} is missing: generate it with tests/golden/make_golden.py on a GPU")
    return np.load(GOLDEN)


def _digest(case):
    return hashlib.sha256(repr((case["n"], case["mapping"], case["prep"], case["circuit"])).encode()).hexdigest()[:16]


@pytest.mark.parametrize("case", golden_cases.cases(), ids=lambda c: c["name"])
def test_oracle_matches_reference_golden(oracle_lib, case):
    g = _golden()
    key = case["name"]
    assert str(g[f"{key}/digest"]) == _digest(case), "case definition changed since the fixtures were made"
    with qcs_b200.Simulator(oracle_lib, case["n"], case["num_clbits"], mapping=case["mapping"],
                            seed=golden_cases.SEED) as sim:
        shots, state = golden_cases.run_case(sim, case)
    ref_state = g[f"{key}/state"]
    assert list(g[f"{key}/shots"]) == shots
    scale = max(1.0, float(np.max(np.abs(ref_state))))
    assert np.max(np.abs(state - ref_state)) <= 1e-12 * scale
