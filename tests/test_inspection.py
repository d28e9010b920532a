"""Register inspection extensions: single-amplitude reads and register
comparison (overlap and max difference). Both work in logical order, so they
must agree with the full state read back through get_statevector whatever
the qubit mapping, the relabelled swaps and the precision."""

import numpy as np
import pytest

import qcs_b200
from qcs_b200 import FUSION_GREEDY, FUSION_PLAIN
from qcs_b200 import circuits as C

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", [128, 64])
@pytest.mark.parametrize("mode", [FUSION_PLAIN, FUSION_GREEDY])
def test_amplitudes_match_statevector(gpu_lib, precision, mode):
    n = 14
    mapping = [int(q) for q in np.random.default_rng(3).permutation(n)]
    circ = C.random_circuit(n, 120, seed=9, gates=["u3", "h", "swap", "x", "rzz", "p"])
    with qcs_b200.Simulator(gpu_lib, n, mapping=mapping, fusion=mode, precision=precision) as sim:
        sim.run(circ)
        full = sim.statevector()
        idx = np.random.default_rng(4).integers(0, 1 << n, size=3000, dtype=np.uint64)
        got = sim.amplitudes(idx)
        assert np.array_equal(got, full[idx.astype(np.int64)])
        assert sim.amplitudes([]).size == 0
        with pytest.raises(qcs_b200.QCSError, match="outside"):
            sim.amplitudes([1 << n])


@pytest.mark.parametrize("precision", [128, 64])
def test_compare_matches_host_arithmetic(gpu_lib, precision):
    n = 23   # several staging chunks
    circ = C.layered_u3_cz_cx_toffoli(n, 3, seed=2)
    with qcs_b200.Simulator(gpu_lib, n, fusion=FUSION_PLAIN) as ref, \
            qcs_b200.Simulator(gpu_lib, n, fusion=FUSION_GREEDY, precision=precision,
                               mapping=list(range(n))[::-1]) as sim:
        ref.run(circ)
        sim.run(circ + [("swap", (), (0, 5), (), ()), ("swap", (), (0, 5), (), ())])
        cmp = sim.compare(ref)
        a, b = sim.statevector(), ref.statevector()
        want = np.vdot(a, b)
        assert abs(cmp["overlap"] - want) <= 1e-12 * max(1.0, abs(want)) + 1e-13
        assert cmp["max_abs_diff"] == pytest.approx(float(np.max(np.abs(a - b))), rel=1e-9, abs=1e-300)
        assert cmp["norm_self"] == pytest.approx(np.vdot(a, a).real, rel=1e-12)
        assert cmp["norm_other"] == pytest.approx(np.vdot(b, b).real, rel=1e-12)
        tol = 1e-12 if precision == 128 else 1e-6
        assert 1.0 - cmp["fidelity"] <= tol
        # a register compared with itself
        same = ref.compare(ref)
        assert same["max_abs_diff"] == 0.0
        assert same["overlap"].real == pytest.approx(np.vdot(b, b).real, rel=1e-13)
        assert same["fidelity"] == pytest.approx(1.0, abs=1e-14)


def test_compare_rejects_other_sizes(gpu_lib):
    with qcs_b200.Simulator(gpu_lib, 10) as a, qcs_b200.Simulator(gpu_lib, 11) as b:
        with pytest.raises(qcs_b200.QCSError, match="registers of 10 and 11"):
            a.compare(b)
