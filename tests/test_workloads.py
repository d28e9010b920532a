"""The benchmark workloads and their algorithmic bytes, on the host (no GPU).

The roofline figures of bench.py divide these byte counts by measured
times, so the generators and the accounting are pinned here to the
workload definitions: gate counts by kind and control count, and the
total bytes (2 x 16 B x the amplitudes each gate can change, complex128)
of the 20-qubit CLI circuit (about 14.0 GiB), the 30-qubit layered circuit
(45,600 GiB), the 30-qubit matching circuit (72,000 GiB) and the 33-qubit
QFT (44,288 GiB without the X gates that prepare its basis input).
"""

from collections import Counter

import pytest

from qcs_b200 import circuits as C

GiB = float(1 << 30)


def _kinds(circ):
    return Counter((op, len(neg) + len(pos)) for op, _, _, neg, pos in circ)


def test_layered_30_qubits_depth_40():
    circ = C.layered_u3_cz_cx_toffoli(30, 40, seed=1)
    assert len(circ) == 1820
    assert _kinds(circ) == {("u3", 0): 1200, ("z", 1): 300, ("x", 1): 280, ("x", 2): 40}
    assert C.algorithmic_bytes(circ, 30) / GiB == 45600.0


def test_matching_30_qubits_60_layers():
    circ = C.u3_random_matching(30, 60, seed=1)
    assert _kinds(circ) == {("u3", 0): 1800, ("x", 1): 900}
    # every layer's CX pairs form a perfect matching of the 30 qubits
    cx = [tuple(sorted((targets[0], pos[0]))) for op, _, targets, _, pos in circ if op == "x"]
    for layer in range(60):
        pairs = cx[15 * layer: 15 * (layer + 1)]
        assert sorted(q for p in pairs for q in p) == list(range(30))
    assert C.algorithmic_bytes(circ, 30) / GiB == 72000.0
    assert C.algorithmic_bytes(circ, 30, 8) / GiB == 36000.0


def test_qft_33_qubits():
    circ, x = C.qft(33, seed=1)
    kinds = _kinds(circ)
    assert kinds[("h", 0)] == 33
    assert kinds[("p", 1)] == 33 * 32 // 2
    assert kinds[("swap", 0)] == 16
    assert kinds[("x", 0)] == bin(x).count("1")
    body = [g for g in circ if g[0] != "x"]
    assert C.algorithmic_bytes(body, 33) / GiB == 44288.0


def test_cli_circuit_20_qubits_depth_20():
    circ = C.layered_u3_cz(20, 20, seed=1, measure=True)
    assert _kinds(circ) == {("u3", 0): 400, ("z", 1): 190, ("measure", 0): 20}
    assert C.algorithmic_bytes(circ, 20) / GiB == pytest.approx(14.0, abs=0.05)


@pytest.mark.parametrize("n", [10, 15, 20])
def test_hea_circuit_layers(n):
    circ = C.hea_circuit(n, 8, seed=3)
    assert _kinds(circ) == {("ry", 0): 8 * n, ("rz", 0): 8 * n, ("x", 1): 8 * (n - 1)}
