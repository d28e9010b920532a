"""qcs_simulator_get_device_state: the register handed out in logical order.

Uncontrolled SWAPs only relabel qubits in the fused modes (and a mapping
places logical qubits elsewhere), so the register's physical layout can
differ from the logical order. Asking for the device pointer moves the
amplitudes in HBM (physical SWAPs packed into fused passes) until physical
qubit q holds logical qubit q. The device memory, read back raw with the
CUDA runtime, must then equal the oracle's state in logical order, and
later gates must still act on the right qubits.
"""

import ctypes

import numpy as np
import pytest

import qcs_b200
from qcs_b200 import circuits as C

pytestmark = pytest.mark.gpu


def _cudart():
    for name in ("libcudart.so", "libcudart.so.12"):
        try:
            return ctypes.CDLL(name)
        except OSError:
            pass
    return ctypes.CDLL("/usr/local/cuda/lib64/libcudart.so")


def _read_device(ptr, n, bits):
    """Raw device memory of 2^n amplitudes as complex128."""
    rt = _cudart()
    dtype = np.float64 if bits == 128 else np.float32
    host = np.empty(2 << n, dtype=dtype)
    rt.cudaMemcpy.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int]
    assert rt.cudaMemcpy(host.ctypes.data, ptr, host.nbytes, 2) == 0   # device to host
    return host.astype(np.float64).view(np.complex128)


def _scrambled(n, seed):
    """Random gates with uncontrolled SWAPs among them (relabels in the fused
    modes), ending with a reversal of the qubit order."""
    rng = np.random.default_rng(seed)
    circ = []
    for blk in range(6):
        circ += C.random_circuit(n, 30, seed=seed * 10 + blk, max_controls=2, gates=["u3", "h", "rz", "x", "p"])
        for _ in range(3):
            a, b = (int(x) for x in rng.choice(n, size=2, replace=False))
            circ.append(("swap", (), (a, b), (), ()))
    circ += [("swap", (), (q, n - 1 - q), (), ()) for q in range(n // 2)]
    return circ


@pytest.mark.parametrize("fusion", [qcs_b200.FUSION_GREEDY, qcs_b200.FUSION_PLAIN])
@pytest.mark.parametrize("precision", [128, 64])
@pytest.mark.parametrize("n", [14, 22])
def test_device_state_in_logical_order(gpu_lib, oracle_lib, n, precision, fusion):
    circ = _scrambled(n, n + precision)
    tail = C.random_circuit(n, 40, seed=77 + n, max_controls=1, gates=["u3", "ry"])
    with qcs_b200.Simulator(oracle_lib, n) as sim:
        sim.run(circ)
        ref = sim.statevector()
        sim.run(tail)
        ref_tail = sim.statevector()
    tol = 1e-12 if precision == 128 else 2e-6
    with qcs_b200.Simulator(gpu_lib, n, fusion=fusion, precision=precision) as sim:
        sim.run(circ)
        before = sim.stats()["kernel_launches"]
        ptr, bits = sim.device_state()
        assert bits == precision and ptr
        got = _read_device(ptr, n, bits)
        assert np.max(np.abs(got - ref)) <= tol
        if fusion == qcs_b200.FUSION_GREEDY:
            # the relabels left the layout scrambled: the permutation ran
            assert sim.stats()["kernel_launches"] > before
        # the layout is now the logical order: a second call moves nothing
        launches = sim.stats()["kernel_launches"]
        assert sim.device_state()[0] == ptr
        assert sim.stats()["kernel_launches"] == launches
        # later gates act on the logical qubits
        sim.run(tail)
        assert np.max(np.abs(sim.statevector() - ref_tail)) <= tol
        assert np.max(np.abs(_read_device(*sim.device_state()[:1], n, bits) - ref_tail)) <= tol


def test_device_state_with_mapping(gpu_lib, oracle_lib):
    """A mapping given before allocation places the logical qubits elsewhere
    physically; the handed-out register is still in logical order."""
    n = 16
    mapping = list(range(n))[::-1]
    circ = C.random_circuit(n, 120, seed=5, max_controls=2, gates=["u3", "h", "x", "rzz"])
    with qcs_b200.Simulator(oracle_lib, n, mapping=mapping) as sim:
        sim.run(circ)
        ref = sim.statevector()
    with qcs_b200.Simulator(gpu_lib, n, mapping=mapping, fusion=qcs_b200.FUSION_GREEDY) as sim:
        sim.run(circ)
        ptr, bits = sim.device_state()
        assert np.max(np.abs(_read_device(ptr, n, bits) - ref)) <= 1e-12
        assert np.max(np.abs(sim.statevector() - ref)) <= 1e-12
