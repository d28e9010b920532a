"""ctypes binding of the qcs C API (include/qcs.h, include/qcs_b200.h).

The same binding drives any library that exports the reference's C ABI:
the B200 library (rqs-svg_b200/lib/libqcs.so), and -- in the tests only --
the CPU oracle and the reference build. Calls mirror the C functions one to
one (reference src/qcs.cu:3383-3759); a 0 return raises QCSError carrying the
message the library passed to its exception callback.
"""

from __future__ import annotations

import ctypes
import os
import tempfile
from pathlib import Path

import numpy as np

PKG_DIR = Path(__file__).resolve().parent.parent
REPO_DIR = PKG_DIR.parent
LIB_PATH = PKG_DIR / "lib" / "libqcs.so"
CLI_PATH = PKG_DIR / "bin" / "qcs"

bit_num_t = ctypes.c_int16
bit_t = ctypes.c_uint8
event_num_t = ctypes.c_int16
_P = ctypes.c_void_p
_BN = ctypes.POINTER(bit_num_t)
_FP = ctypes.POINTER(ctypes.c_float)

COST_MODEL_PARAMS = 4673
COST_MODEL_SCALING = 14

# name -> (number of double parameters, number of targets)
GATES = {
    "global_phase": (1, 0),
    "h": (0, 1), "x": (0, 1), "y": (0, 1), "z": (0, 1), "s": (0, 1), "sdg": (0, 1),
    "t": (0, 1), "tdg": (0, 1), "sx": (0, 1), "sxdg": (0, 1), "id": (0, 1),
    "rx": (1, 1), "ry": (1, 1), "rz": (1, 1), "u1": (1, 1), "p": (1, 1),
    "u2": (2, 1), "r": (2, 1), "u3": (3, 1), "u": (3, 1), "u4": (4, 1),
    "swap": (0, 2), "iswap": (0, 2), "dcx": (0, 2), "ecr": (0, 2),
    "rxx": (1, 2), "ryy": (1, 2), "rzz": (1, 2), "rzx": (1, 2),
    "xx_plus_yy": (2, 2), "xx_minus_yy": (2, 2),
    "rccx": (0, 3), "rcccx": (0, 4),
}

FUSION_PLAIN, FUSION_GREEDY, FUSION_LEARNED = 0, 1, 2
TENSOR_NEVER, TENSOR_AUTO, TENSOR_ALWAYS, TENSOR_ALWAYS_8X8 = 0, 1, 2, 3
ENGINE_MMA_SYNC, ENGINE_TCGEN05 = 0, 1
# cost-model inputs per pass (QCS_PASS_FEATURES): block width, blocks, gates,
# light ops, target-qubit stride, log2 chunks
PASS_FEATURES = 6


class QCSError(RuntimeError):
    pass


class Stats(ctypes.Structure):
    _fields_ = [
        ("kernel_launches", ctypes.c_uint64),
        ("gates_received", ctypes.c_uint64),
        ("gates_applied", ctypes.c_uint64),
        ("fused_passes", ctypes.c_uint64),
        ("plain_gate_kernels", ctypes.c_uint64),
        ("algorithmic_bytes", ctypes.c_double),
        ("tensor_passes", ctypes.c_uint64),
        ("tensor8_passes", ctypes.c_uint64),
        ("tcgen05_passes", ctypes.c_uint64),
        ("replayed_flushes", ctypes.c_uint64),
    ]


class KernelTimes(ctypes.Structure):
    _fields_ = [
        ("fused_launches", ctypes.c_uint64),
        ("fused_ms", ctypes.c_double),
        ("fused_bytes", ctypes.c_double),
        ("plain_launches", ctypes.c_uint64),
        ("plain_ms", ctypes.c_double),
        ("plain_bytes", ctypes.c_double),
    ]


class BatchGate(ctypes.Structure):
    _fields_ = [
        ("name", ctypes.c_char * 16),
        ("params", ctypes.c_double * 4),
        ("num_targets", ctypes.c_int16),
        ("num_negctrls", ctypes.c_int16),
        ("num_ctrls", ctypes.c_int16),
        ("reserved", ctypes.c_int16),
        ("qubits", ctypes.c_int16 * 12),
    ]


PLAN_KINDS = 24
PLAN_KIND_NAMES = {0: "dense1", 1: "x", 2: "dense2", 3: "cswap", 4: "phase", 5: "diag", 6: "term",
                   7: "dense1_real", 9: "phase_i", 10: "group4", 11: "group4_real", 12: "phase_run",
                   13: "sign_run", 14: "sign_term", 15: "group2"}


class PlanSummary(ctypes.Structure):
    _fields_ = [
        ("passes", ctypes.c_uint32),
        ("plain_gates", ctypes.c_uint32),
        ("stages", ctypes.c_uint32),
        ("ops", ctypes.c_uint32),
        ("kinds", ctypes.c_uint32 * PLAN_KINDS),
        ("table_entries", ctypes.c_uint64),
        ("tensor_passes", ctypes.c_uint32),
        ("tensor_eligible", ctypes.c_uint32),
        ("tensor_matrices", ctypes.c_uint32),
        ("tensor8_passes", ctypes.c_uint32),
    ]


class BatchInfo(ctypes.Structure):
    _fields_ = [
        ("circuits", ctypes.c_uint32),
        ("groups", ctypes.c_uint32),
        ("passes", ctypes.c_uint32),
        ("launches_per_run", ctypes.c_uint32),
        ("amplitudes", ctypes.c_uint64),
        ("parameters", ctypes.c_uint64),
        ("pass_bytes", ctypes.c_double),
        ("last_run_ms", ctypes.c_double),
        ("tensor_passes", ctypes.c_uint32),
        ("reserved", ctypes.c_uint32),
    ]


_CALLBACK = ctypes.CFUNCTYPE(None, ctypes.c_char_p, ctypes.c_size_t)


class Library:
    """One loaded implementation of the qcs C API."""

    def __init__(self, path: str | os.PathLike = LIB_PATH, mode: int = ctypes.RTLD_LOCAL):
        self.path = str(path)
        if not os.path.exists(self.path):
            raise QCSError(f"{self.path} is missing: build it with `make -C rqs-svg_b200`")
        self.lib = ctypes.CDLL(self.path, mode=mode)
        self.last_error = ""

        def _on_error(msg, length):
            self.last_error = ctypes.string_at(msg, length).decode(errors="replace")

        self._cb = _CALLBACK(_on_error)
        self.lib.qcs_set_exception_callback.argtypes = [_CALLBACK]
        self.lib.qcs_set_exception_callback(self._cb)
        self._declare()

    def has(self, name: str) -> bool:
        return hasattr(self.lib, name)

    def _declare(self):
        L = self.lib
        sig = {
            "qcs_simulator_create": [ctypes.POINTER(_P)],
            "qcs_simulator_destroy": [_P],
            "qcs_simulator_allocate_memory": [_P],
            "qcs_simulator_dispose": [_P],
            "qcs_simulator_get_num_procs": [_P, ctypes.POINTER(bit_t)],
            "qcs_simulator_get_proc_num": [_P, ctypes.POINTER(bit_t)],
            "qcs_simulator_get_num_qubits": [_P, ctypes.POINTER(bit_t)],
            "qcs_simulator_get_num_clbits": [_P, ctypes.POINTER(bit_t)],
            "qcs_simulator_set_num_qubits": [_P, bit_num_t],
            "qcs_simulator_set_mapping": [_P, _BN, bit_num_t],
            "qcs_simulator_set_num_clbits": [_P, bit_num_t],
            "qcs_simulator_get_clbits": [_P, ctypes.POINTER(bit_t)],
            "qcs_simulator_get_clbits_string": [_P, ctypes.c_char_p],
            "qcs_simulator_reset": [_P, bit_num_t],
            "qcs_simulator_set_zero_state": [_P],
            "qcs_simulator_set_sequential_state": [_P],
            "qcs_simulator_set_flat_state": [_P],
            "qcs_simulator_set_entangled_state": [_P],
            "qcs_simulator_set_random_state": [_P],
            "qcs_simulator_reset_clbits": [_P],
            "qcs_simulator_reset_measurement_state": [_P],
            "qcs_simulator_reinitialize_mapping": [_P],
            "qcs_simulator_gate_global_phase": [_P, ctypes.c_double, _BN, bit_num_t, _BN, bit_num_t],
            "qcs_simulator_measure": [_P, bit_num_t, ctypes.POINTER(bit_t)],
            "qcs_simulator_measure_to_clbit": [_P, bit_num_t, bit_num_t, ctypes.POINTER(bit_t)],
            "qcs_simulator_read": [_P, bit_num_t, ctypes.POINTER(bit_t)],
            "qcs_simulator_save_statevector": [_P, ctypes.c_char_p],
            "qcs_simulator_event_create": [_P, ctypes.POINTER(bit_t)],
            "qcs_simulator_event_record": [_P, ctypes.c_int],
            "qcs_simulator_event_get_elapsed_time": [_P, event_num_t, event_num_t, ctypes.POINTER(ctypes.c_double)],
            # extensions (absent from the reference build)
            "qcs_simulator_set_fusion": [_P, ctypes.c_int],
            "qcs_simulator_get_fusion": [_P, ctypes.POINTER(ctypes.c_int)],
            "qcs_simulator_set_seed": [_P, ctypes.c_uint32],
            "qcs_simulator_synchronize": [_P],
            "qcs_simulator_get_statevector": [_P, ctypes.POINTER(ctypes.c_double), ctypes.c_uint64],
            "qcs_simulator_set_statevector": [_P, ctypes.POINTER(ctypes.c_double), ctypes.c_uint64],
            "qcs_simulator_expectation_z": [_P, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)],
            "qcs_simulator_sample": [_P, ctypes.c_uint32, ctypes.POINTER(ctypes.c_uint64)],
            "qcs_simulator_get_stats": [_P, ctypes.POINTER(Stats)],
            "qcs_simulator_reset_stats": [_P],
            "qcs_simulator_set_kernel_timing": [_P, ctypes.c_int],
            "qcs_simulator_get_kernel_times": [_P, ctypes.POINTER(KernelTimes)],
            "qcs_b200_zsums_noalloc": [_P, ctypes.c_int, _P, _P],
            "qcs_simulator_set_planner_options": [_P, ctypes.c_int, ctypes.c_int],
            "qcs_simulator_set_tensor_passes": [_P, ctypes.c_int],
            "qcs_simulator_get_tensor_passes": [_P, ctypes.POINTER(ctypes.c_int)],
            "qcs_simulator_set_tensor_engine": [_P, ctypes.c_int],
            "qcs_simulator_get_tensor_engine": [_P, ctypes.POINTER(ctypes.c_int)],
            "qcs_simulator_set_precision": [_P, ctypes.c_int],
            "qcs_simulator_get_precision": [_P, ctypes.POINTER(ctypes.c_int)],
            "qcs_simulator_get_pass_records": [_P, _FP, _FP, ctypes.c_uint32, ctypes.POINTER(ctypes.c_uint32)],
            "qcs_b200_cost_model_create": [ctypes.POINTER(_P), ctypes.c_uint32],
            "qcs_b200_cost_model_destroy": [_P],
            "qcs_b200_cost_model_train": [_P, _FP, _FP, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32,
                                          ctypes.c_float, _FP],
            "qcs_b200_cost_model_predict": [_P, _FP, ctypes.c_uint32, _FP],
            "qcs_b200_cost_model_gradients": [_P, _FP, _FP, ctypes.c_uint32, _FP, _FP],
            "qcs_b200_cost_model_get_params": [_P, _FP, _FP],
            "qcs_b200_cost_model_set_params": [_P, _FP, _FP],
            "qcs_simulator_set_cost_model": [_P, _P],
            "qcs_simulator_get_planner_judge": [_P, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double),
                                                ctypes.POINTER(ctypes.c_double)],
            "qcs_simulator_get_amplitudes": [_P, ctypes.POINTER(ctypes.c_uint64), ctypes.c_uint64,
                                             ctypes.POINTER(ctypes.c_double)],
            "qcs_simulator_compare": [_P, _P] + [ctypes.POINTER(ctypes.c_double)] * 5,
            "qcs_simulator_get_device_state": [_P, ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_int)],
            "qcs_b200_batch_create": [ctypes.POINTER(_P), ctypes.c_int],
            "qcs_b200_batch_destroy": [_P],
            "qcs_b200_batch_add_circuit": [_P, ctypes.c_int, ctypes.POINTER(BatchGate), ctypes.c_uint32,
                                           ctypes.POINTER(ctypes.c_uint32)],
            "qcs_b200_batch_set_parameters": [_P, ctypes.POINTER(ctypes.c_double), ctypes.c_uint64],
            "qcs_b200_batch_run": [_P],
            "qcs_b200_batch_expectation_z": [_P, ctypes.POINTER(ctypes.c_double), ctypes.c_uint64],
            "qcs_b200_batch_get_statevector": [_P, ctypes.c_uint32, ctypes.POINTER(ctypes.c_double), ctypes.c_uint64],
            "qcs_b200_batch_get_info": [_P, ctypes.POINTER(BatchInfo)],
            "qcs_b200_batch_set_tensor_passes": [_P, ctypes.c_int],
            "qcs_b200_plan_summary_get": [ctypes.c_int, ctypes.POINTER(BatchGate), ctypes.c_uint64,
                                          ctypes.POINTER(PlanSummary)],
        }
        for name, (np_, nt) in GATES.items():
            if name == "global_phase":
                continue
            sig[f"qcs_simulator_gate_{name}"] = [_P] + [ctypes.c_double] * np_ + [_BN, bit_num_t, _BN, bit_num_t, _BN, bit_num_t]
        for name, args in sig.items():
            if hasattr(L, name):
                fn = getattr(L, name)
                fn.argtypes = args
                fn.restype = ctypes.c_int

    def call(self, name: str, *args) -> None:
        self.last_error = ""
        ok = getattr(self.lib, name)(*args)
        if ok != 1:
            raise QCSError(f"{name} failed: {self.last_error}")


def _arr(values):
    values = list(values)
    if not values:
        return None, 0
    return (bit_num_t * len(values))(*values), len(values)


class Simulator:
    """A qcs_simulator handle: create, configure, allocate, run, destroy."""

    def __init__(self, lib: Library, num_qubits: int, num_clbits: int = 0, mapping=None,
                 seed: int | None = None, fusion: int | None = None, allocate: bool = True,
                 precision: int | None = None):
        self.lib = lib
        self.n = num_qubits
        self.h = _P()
        lib.call("qcs_simulator_create", ctypes.byref(self.h))
        lib.call("qcs_simulator_set_num_qubits", self.h, num_qubits)
        if precision is not None:
            lib.call("qcs_simulator_set_precision", self.h, precision)
        if num_clbits:
            lib.call("qcs_simulator_set_num_clbits", self.h, num_clbits)
        if mapping is not None:
            arr, cnt = _arr(mapping)
            lib.call("qcs_simulator_set_mapping", self.h, arr, cnt)
        if seed is not None:
            lib.call("qcs_simulator_set_seed", self.h, seed)
        if fusion is not None and lib.has("qcs_simulator_set_fusion"):
            lib.call("qcs_simulator_set_fusion", self.h, fusion)
        if allocate:
            lib.call("qcs_simulator_allocate_memory", self.h)

    # -- lifecycle
    def close(self):
        if self.h:
            self.lib.call("qcs_simulator_destroy", self.h)
            self.h = _P()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- gates
    def gate(self, name: str, params=(), targets=(), negctrls=(), ctrls=()):
        t, nt = _arr(targets)
        ng, nng = _arr(negctrls)
        c, nc = _arr(ctrls)
        if name == "global_phase":
            self.lib.call("qcs_simulator_gate_global_phase", self.h, float(params[0]), ng, nng, c, nc)
        else:
            self.lib.call(f"qcs_simulator_gate_{name}", self.h, *[float(p) for p in params], t, nt, ng, nng, c, nc)

    def run(self, circuit):
        """Replay a circuit: a list of (op, params, targets, negctrls, ctrls);
        op "measure" takes targets=(qubit,) and params=(clbit,)."""
        for op, params, targets, negctrls, ctrls in circuit:
            if op == "measure":
                self.measure_to_clbit(targets[0], int(params[0]))
            else:
                self.gate(op, params, targets, negctrls, ctrls)

    # -- measurement and classical bits
    def measure(self, q: int) -> int:
        r = bit_t()
        self.lib.call("qcs_simulator_measure", self.h, q, ctypes.byref(r))
        return r.value

    def measure_to_clbit(self, q: int, c: int) -> int:
        r = bit_t()
        self.lib.call("qcs_simulator_measure_to_clbit", self.h, q, c, ctypes.byref(r))
        return r.value

    def read(self, c: int) -> int:
        r = bit_t()
        self.lib.call("qcs_simulator_read", self.h, c, ctypes.byref(r))
        return r.value

    def reset(self, q: int):
        self.lib.call("qcs_simulator_reset", self.h, q)

    def clbits_string(self) -> str:
        n = bit_t()
        self.lib.call("qcs_simulator_get_num_clbits", self.h, ctypes.byref(n))
        buf = ctypes.create_string_buffer(n.value + 1)
        self.lib.call("qcs_simulator_get_clbits_string", self.h, buf)
        return buf.value.decode()

    # -- state preparation and bookkeeping
    def set_state(self, kind: str):
        self.lib.call(f"qcs_simulator_set_{kind}_state", self.h)

    def reset_clbits(self):
        self.lib.call("qcs_simulator_reset_clbits", self.h)

    def reset_measurement_state(self):
        self.lib.call("qcs_simulator_reset_measurement_state", self.h)

    def reinitialize_mapping(self):
        self.lib.call("qcs_simulator_reinitialize_mapping", self.h)

    def set_mapping(self, mapping):
        arr, cnt = _arr(mapping)
        self.lib.call("qcs_simulator_set_mapping", self.h, arr, cnt)

    # -- output
    def save_statevector(self, path: str):
        self.lib.call("qcs_simulator_save_statevector", self.h, str(path).encode())

    def statevector(self) -> np.ndarray:
        """State in logical order as complex128 (through save_statevector
        when the library has no get_statevector, as for the reference)."""
        size = 1 << self.n
        if self.lib.has("qcs_simulator_get_statevector"):
            out = np.empty(2 * size, dtype=np.float64)
            self.lib.call("qcs_simulator_get_statevector", self.h,
                          out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), size)
            return out.view(np.complex128)
        with tempfile.TemporaryDirectory() as d:
            p = os.path.join(d, "sv.bin")
            self.save_statevector(p)
            return np.fromfile(p, dtype=np.complex128)

    def set_statevector(self, amps: np.ndarray):
        a = np.ascontiguousarray(amps, dtype=np.complex128).view(np.float64)
        self.lib.call("qcs_simulator_set_statevector", self.h,
                      a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), a.size // 2)

    def expectation_z(self):
        out = np.empty(self.n, dtype=np.float64)
        norm = ctypes.c_double()
        self.lib.call("qcs_simulator_expectation_z", self.h,
                      out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), ctypes.byref(norm))
        return out, norm.value

    def sample(self, shots: int) -> np.ndarray:
        out = np.zeros(shots, dtype=np.uint64)
        self.lib.call("qcs_simulator_sample", self.h, shots,
                      out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)))
        return out

    def synchronize(self):
        self.lib.call("qcs_simulator_synchronize", self.h)

    def amplitudes(self, indices) -> np.ndarray:
        """Amplitudes at the given logical indices (complex128)."""
        idx = np.ascontiguousarray(indices, dtype=np.uint64)
        out = np.empty(2 * idx.size, dtype=np.float64)
        self.lib.call("qcs_simulator_get_amplitudes", self.h, idx.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)),
                      idx.size, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        return out.view(np.complex128)

    def device_state(self):
        """(device pointer, amplitude bits) of the register in logical order
        (the library first moves the amplitudes so that physical qubit q
        holds logical qubit q)."""
        ptr, bits = ctypes.c_void_p(), ctypes.c_int()
        self.lib.call("qcs_simulator_get_device_state", self.h, ctypes.byref(ptr), ctypes.byref(bits))
        return ptr.value, bits.value

    def compare(self, other: "Simulator") -> dict:
        """<self|other>, max |self_i - other_i|, both squared norms and the
        fidelity |<self|other>|^2 / (<self|self> <other|other>), over logical
        indices."""
        v = [ctypes.c_double() for _ in range(5)]
        self.lib.call("qcs_simulator_compare", self.h, other.h, *[ctypes.byref(x) for x in v])
        ovl = complex(v[0].value, v[1].value)
        na, nb = v[3].value, v[4].value
        return {"overlap": ovl, "max_abs_diff": v[2].value, "norm_self": na, "norm_other": nb,
                "fidelity": abs(ovl) ** 2 / (na * nb) if na > 0 and nb > 0 else 0.0}

    def set_fusion(self, mode: int):
        self.lib.call("qcs_simulator_set_fusion", self.h, mode)

    def set_seed(self, seed: int):
        self.lib.call("qcs_simulator_set_seed", self.h, seed)

    # -- events
    def event_create(self) -> int:
        r = bit_t()
        self.lib.call("qcs_simulator_event_create", self.h, ctypes.byref(r))
        return r.value

    def event_record(self, e: int):
        self.lib.call("qcs_simulator_event_record", self.h, e)

    def elapsed(self, a: int, b: int) -> float:
        r = ctypes.c_double()
        self.lib.call("qcs_simulator_event_get_elapsed_time", self.h, a, b, ctypes.byref(r))
        return r.value

    def stats(self) -> dict:
        s = Stats()
        self.lib.call("qcs_simulator_get_stats", self.h, ctypes.byref(s))
        return {f: getattr(s, f) for f, _ in Stats._fields_}

    def reset_stats(self):
        self.lib.call("qcs_simulator_reset_stats", self.h)

    def set_kernel_timing(self, enable: bool):
        self.lib.call("qcs_simulator_set_kernel_timing", self.h, 1 if enable else 0)

    def kernel_times(self) -> dict:
        t = KernelTimes()
        self.lib.call("qcs_simulator_get_kernel_times", self.h, ctypes.byref(t))
        return {f: getattr(t, f) for f, _ in KernelTimes._fields_}

    def set_planner_options(self, max_gates_per_pass: int = 0, local_qubits: int = 0):
        self.lib.call("qcs_simulator_set_planner_options", self.h, max_gates_per_pass, local_qubits)

    def set_tensor_engine(self, engine: int):
        """1: complex64 16 x 16 stages on tcgen05 where allowed (default);
        0: every tensor pass on warp-level mma.sync."""
        self.lib.call("qcs_simulator_set_tensor_engine", self.h, engine)

    def set_tensor_passes(self, mode: int):
        """0: never, 1: where cheaper (default), 2: 16 x 16 stages wherever a
        pass allows, 3: 8 x 8 stages wherever a pass allows."""
        self.lib.call("qcs_simulator_set_tensor_passes", self.h, mode)

    def pass_records(self, capacity: int = 1 << 20):
        feats = np.zeros((capacity, PASS_FEATURES), dtype=np.float32)
        ms = np.zeros(capacity, dtype=np.float32)
        count = ctypes.c_uint32()
        self.lib.call("qcs_simulator_get_pass_records", self.h, _fptr(feats), _fptr(ms), capacity, ctypes.byref(count))
        return feats[: count.value].copy(), ms[: count.value].copy()

    def set_cost_model(self, model):
        self.lib.call("qcs_simulator_set_cost_model", self.h, model.h if model is not None else None)

    def planner_judge(self):
        used = ctypes.c_int()
        g, lrn = ctypes.c_double(), ctypes.c_double()
        self.lib.call("qcs_simulator_get_planner_judge", self.h, ctypes.byref(used), ctypes.byref(g), ctypes.byref(lrn))
        return {"learned_plan": bool(used.value), "greedy_ms": g.value, "learned_ms": lrn.value}


def _fptr(a: np.ndarray):
    assert a.dtype == np.float32 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_FP)


class CostModel:
    """The learned pass-cost model (MLP 4 -> 64 -> 64 -> 1, trained on the GPU)."""

    def __init__(self, lib: Library, seed: int = 1):
        self.lib = lib
        self.h = _P()
        lib.call("qcs_b200_cost_model_create", ctypes.byref(self.h), seed)

    def close(self):
        if self.h:
            self.lib.call("qcs_b200_cost_model_destroy", self.h)
            self.h = _P()

    def train(self, features, targets, epochs=200, batch=256, lr=1e-3) -> float:
        f = np.ascontiguousarray(features, dtype=np.float32)
        t = np.ascontiguousarray(targets, dtype=np.float32)
        loss = ctypes.c_float()
        self.lib.call("qcs_b200_cost_model_train", self.h, _fptr(f), _fptr(t), len(t), epochs, batch, lr,
                      ctypes.byref(loss))
        return loss.value

    def predict(self, features) -> np.ndarray:
        f = np.ascontiguousarray(features, dtype=np.float32)
        out = np.zeros(len(f), dtype=np.float32)
        self.lib.call("qcs_b200_cost_model_predict", self.h, _fptr(f), len(f), _fptr(out))
        return out

    def gradients(self, inputs, targets):
        x = np.ascontiguousarray(inputs, dtype=np.float32)
        t = np.ascontiguousarray(targets, dtype=np.float32)
        g = np.zeros(COST_MODEL_PARAMS, dtype=np.float32)
        loss = ctypes.c_float()
        self.lib.call("qcs_b200_cost_model_gradients", self.h, _fptr(x), _fptr(t), len(t), _fptr(g), ctypes.byref(loss))
        return g, loss.value

    def params(self):
        p = np.zeros(COST_MODEL_PARAMS, dtype=np.float32)
        s = np.zeros(COST_MODEL_SCALING, dtype=np.float32)
        self.lib.call("qcs_b200_cost_model_get_params", self.h, _fptr(p), _fptr(s))
        return p, s

    def set_params(self, params, scaling):
        p = np.ascontiguousarray(params, dtype=np.float32)
        s = np.ascontiguousarray(scaling, dtype=np.float32)
        self.lib.call("qcs_b200_cost_model_set_params", self.h, _fptr(p), _fptr(s))


def plan_summary(lib: "Library", num_qubits: int, circuit) -> dict:
    """How the greedy fused planner would run a circuit (host only, no GPU):
    passes, plain gates, stages, ops, ops by kind name, table entries."""
    arr = Batch.encode(circuit)
    out = PlanSummary()
    lib.call("qcs_b200_plan_summary_get", num_qubits, arr.ctypes.data_as(ctypes.POINTER(BatchGate)),
             ctypes.c_uint64(len(circuit)), ctypes.byref(out))
    kinds = {name: int(out.kinds[i]) for i, name in PLAN_KIND_NAMES.items()}
    return {"passes": out.passes, "plain_gates": out.plain_gates, "stages": out.stages, "ops": out.ops,
            "kinds": kinds, "table_entries": int(out.table_entries), "tensor_passes": out.tensor_passes,
            "tensor_eligible": out.tensor_eligible, "tensor_matrices": out.tensor_matrices,
            "tensor8_passes": out.tensor8_passes}


def fidelity(a: np.ndarray, b: np.ndarray) -> float:
    """|<a|b>|^2 / (<a|a><b|b>)."""
    na = np.vdot(a, a).real
    nb = np.vdot(b, b).real
    if na == 0 or nb == 0:
        return 1.0 if na == nb else 0.0
    return float(abs(np.vdot(a, b)) ** 2 / (na * nb))


class Batch:
    """Many independent circuits run together (qcs_b200_batch_*): circuits
    with the same gates on the same qubits share one plan of fused passes,
    and a run is one replayed CUDA graph."""

    def __init__(self, lib: Library, precision: int = 128):
        self.lib = lib
        self.h = _P()
        self.widths = []
        lib.call("qcs_b200_batch_create", ctypes.byref(self.h), precision)

    def close(self):
        if self.h:
            self.lib.call("qcs_b200_batch_destroy", self.h)
            self.h = _P()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # numpy mirror of qcs_b200_gate (80 bytes, C layout)
    GATE_DTYPE = np.dtype([("name", "S16"), ("params", "<f8", (4,)), ("num_targets", "<i2"),
                           ("num_negctrls", "<i2"), ("num_ctrls", "<i2"), ("reserved", "<i2"),
                           ("qubits", "<i2", (12,))])

    @classmethod
    def encode(cls, circuit) -> np.ndarray:
        """Gate array of a circuit given as (op, params, targets, negctrls, ctrls) tuples."""
        g = len(circuit)
        arr = np.zeros(max(1, g), dtype=cls.GATE_DTYPE)
        if g == 0:
            return arr
        params = np.zeros((g, 4))
        qubits = np.zeros((g, 12), dtype=np.int16)
        counts = np.zeros((g, 3), dtype=np.int16)
        for i, (op, p, targets, neg, pos) in enumerate(circuit):
            params[i, : len(p)] = p
            qs = (*targets, *neg, *pos)
            qubits[i, : len(qs)] = qs
            counts[i] = (len(targets), len(neg), len(pos))
        arr["name"] = [c[0].encode() for c in circuit]
        arr["params"] = params
        arr["qubits"] = qubits
        arr["num_targets"], arr["num_negctrls"], arr["num_ctrls"] = counts[:, 0], counts[:, 1], counts[:, 2]
        return arr

    def add_circuit(self, num_qubits: int, circuit) -> int:
        arr = self.encode(circuit)
        idx = ctypes.c_uint32()
        self.lib.call("qcs_b200_batch_add_circuit", self.h, num_qubits,
                      arr.ctypes.data_as(ctypes.POINTER(BatchGate)), len(circuit), ctypes.byref(idx))
        self.widths.append(num_qubits)
        return idx.value

    def set_parameters(self, params):
        p = np.ascontiguousarray(params, dtype=np.float64)
        self.lib.call("qcs_b200_batch_set_parameters", self.h, p.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), p.size)

    def run(self):
        self.lib.call("qcs_b200_batch_run", self.h)

    def set_tensor_passes(self, mode: int):
        """0: register passes only; 1: tuned per group (default); 2: 8 x 8
        tensor passes wherever a pass allows them."""
        self.lib.call("qcs_b200_batch_set_tensor_passes", self.h, mode)

    def expectation_z(self):
        """<Z_q> per circuit: a list of arrays (one value per qubit)."""
        total = sum(self.widths)
        out = np.empty(total, dtype=np.float64)
        self.lib.call("qcs_b200_batch_expectation_z", self.h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), total)
        return np.split(out, np.cumsum(self.widths)[:-1]) if self.widths else []

    def statevector(self, index: int) -> np.ndarray:
        size = 1 << self.widths[index]
        out = np.empty(2 * size, dtype=np.float64)
        self.lib.call("qcs_b200_batch_get_statevector", self.h, index,
                      out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), size)
        return out.view(np.complex128)

    def info(self) -> dict:
        i = BatchInfo()
        self.lib.call("qcs_b200_batch_get_info", self.h, ctypes.byref(i))
        return {f: getattr(i, f) for f, _ in BatchInfo._fields_}
