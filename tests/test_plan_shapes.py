"""Shapes of the fused planner's passes, checked on the host (no GPU).

`qcs_b200_plan_summary_get` plans a gate list as the simulator's greedy fused
mode would and reports passes, stages and pass ops by kind. These tests pin
the plan features the kernel's speed depends on: runs of diagonal gates run
inside the register stages (table-fed factors, integer sign runs), one-qubit
gates are grouped, and small registers fall back to the plain path. The
numerical results of the same plans are checked against the oracle by the
GPU tests.
"""

import numpy as np
import pytest

import qcs_b200
from qcs_b200 import circuits as C


def _summary(lib, n, circ):
    return qcs_b200.plan_summary(lib, n, circ)


def test_qft_runs_are_table_fed_inside_two_stages_per_pass(gpu_lib):
    n = 24
    s = _summary(gpu_lib, n, C.qft(n, seed=1)[0])
    k = s["kinds"]
    assert s["plain_gates"] == 0
    assert s["passes"] <= 4
    assert s["stages"] <= 2 * s["passes"] + 1   # two per pass (4 H gates each), one more for the tail
    assert k["phase_run"] >= 4 * (s["passes"] - 1)
    assert k["term"] == 0                 # every controlled phase is in a table or a per-slot factor
    assert s["table_entries"] > 0
    # ~n^2/2 controlled phases became a few ops per pass
    assert s["ops"] <= 20 * s["passes"]


def test_basis_input_x_gates_move_into_the_qft(gpu_lib):
    # the QFT of a basis state: the input's X gates pass the controlled phases
    # (pattern bits flipped) and end in each qubit's H (a column swap), so the
    # plan is the one of the QFT alone: no X op, no pass for the input
    n = 33
    circ, x = C.qft(n, seed=1)
    assert bin(x).count("1") > 8
    s = _summary(gpu_lib, n, circ)
    bare = _summary(gpu_lib, n, [g for g in circ if g[0] != "x"])
    assert s["kinds"]["x"] == 0
    assert s["passes"] == bare["passes"] <= 4
    assert s["stages"] == bare["stages"]
    # an X that meets a gate it cannot pass (a controlled U3 on its qubit)
    # is placed right before it; one with nothing after it ends the queue
    circ = [("x", (), (3,), (), ()), ("p", (0.3,), (3,), (), (5,)), ("u3", (0.1, 0.2, 0.3), (3,), (), (7,)),
            ("x", (), (9,), (), ()), ("x", (), (4,), (), ()), ("x", (), (4,), (), ())]
    s = _summary(gpu_lib, 12, circ)
    assert s["kinds"]["x"] == 2


def test_layered_circuit_groups_one_qubit_gates_and_runs_signs(gpu_lib):
    n = 20
    s = _summary(gpu_lib, n, C.layered_u3_cz_cx_toffoli(n, 8, seed=2))
    k = s["kinds"]
    assert s["plain_gates"] == 0
    assert k["group4"] > 0 and k["group2"] > 0
    assert k["sign_run"] > 0 and k["sign_term"] >= k["sign_run"]
    assert k["phase"] == 0                # CZ never runs as a predicated phase
    assert k["x"] > 0                     # CX and Toffoli exchanges
    # every U3 went into a group or stands alone: group4 x 4 + group2 x 2 + dense1 >= n x depth
    assert 4 * k["group4"] + 2 * k["group2"] + k["dense1"] >= n * 8


def test_hea_real_rotations_group_and_rz_layers_run_inline(gpu_lib):
    n = 18
    s = _summary(gpu_lib, n, C.hea_circuit(n, 6, seed=3))
    k = s["kinds"]
    assert k["group4_real"] > 0
    assert k["phase_run"] > 0
    assert k["group4"] == 0               # RY is real


def test_two_target_gates_and_small_registers(gpu_lib):
    n = 12
    circ = C.random_circuit(n, 60, seed=4, max_controls=1, gates=["rxx", "ryy", "iswap", "u3"])
    s = _summary(gpu_lib, n, circ)
    assert s["kinds"]["dense2"] > 0
    assert s["plain_gates"] == 0
    small = _summary(gpu_lib, 6, C.random_circuit(6, 40, seed=5))
    assert small["passes"] == 0 and small["plain_gates"] == 40


def test_uncontrolled_swaps_only_relabel(gpu_lib):
    n = 12
    swaps = [("swap", (), (q, n - 1 - q), (), ()) for q in range(n // 2)]
    s = _summary(gpu_lib, n, swaps)
    assert s["passes"] == 0 and s["plain_gates"] == 0 and s["ops"] == 0
    # a gate after the swaps acts on the relabelled qubit
    s2 = _summary(gpu_lib, n, swaps + [("h", (), (0,), (), ())])
    assert s2["passes"] == 1 and s2["kinds"]["dense1_real"] + s2["kinds"]["group4_real"] == 1


def test_bad_gates_are_rejected(gpu_lib):
    with pytest.raises(qcs_b200.QCSError, match="qubit out of range"):
        _summary(gpu_lib, 4, [("h", (), (7,), (), ())])
    with pytest.raises(qcs_b200.QCSError):
        _summary(gpu_lib, 4, [("nosuchgate", (), (0,), (), ())])


def test_measured_workloads_keep_their_pass_counts(gpu_lib):
    # the pass counts behind the measured numbers (one read and write of the
    # register per pass): a planner change that adds passes shows here first
    s = _summary(gpu_lib, 30, C.layered_u3_cz_cx_toffoli(30, 40, seed=1))
    assert s["plain_gates"] == 0 and s["passes"] <= 65
    s = _summary(gpu_lib, 30, C.u3_random_matching(30, 60, seed=1))
    assert s["plain_gates"] == 0 and s["passes"] <= 110
    s = _summary(gpu_lib, 33, C.qft(33, seed=1)[0])
    assert s["plain_gates"] == 0 and s["passes"] <= 4


def test_tensor_pass_choice(gpu_lib):
    # the layered and matching workloads run almost every pass on the FP64
    # tensor cores; the QFT's phase runs reach too many qubits outside their
    # stages (one matrix per assignment of at most 8 of them) and stay on the
    # register path
    s = _summary(gpu_lib, 30, C.layered_u3_cz_cx_toffoli(30, 40, seed=1))
    assert s["tensor_eligible"] == s["passes"] and s["tensor_passes"] >= s["passes"] - 2
    assert s["tensor_matrices"] <= 4096 * s["tensor_passes"]
    # with three dense qubits per stage the estimate favours 8 x 8 stages
    # (half the tensor work per stage, a third more stages)
    assert s["tensor8_passes"] >= 0.9 * s["tensor_passes"]
    assert 3.0 <= s["stages"] / s["passes"] <= 4.5
    s = _summary(gpu_lib, 30, C.u3_random_matching(30, 60, seed=1))
    assert s["tensor_passes"] >= 0.8 * s["passes"]
    s = _summary(gpu_lib, 33, C.qft(33, seed=1)[0])
    assert s["tensor_passes"] == 0
    # passes with fewer than 11 local qubits have no tensor form
    s = _summary(gpu_lib, 10, C.layered_u3_cz(10, 8, seed=1))
    assert s["tensor_eligible"] == 0
