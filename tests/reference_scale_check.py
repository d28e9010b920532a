"""Full-size parity check against the reference build (test helper, run by
tests/test_reference_scale.py in a child process with the seed shim
preloaded, so that the reference's measurement engine is seeded like this
library's: src/qcs.cu:1845-1852).

Both libraries run the 30-qubit layered circuit (U3 on every qubit per
layer, CZ on even / CX on odd layers, one Toffoli per layer, depth 40) from
|0..0> on the same GPU. The reference's state vector is read in place, in
chunks, through the device buffer its build recorded (the atlc stand-in
notes the buffers the reference allocates); this library's amplitudes come
through qcs_simulator_get_amplitudes at the same logical indices. Then every
qubit is measured into its clbit in both, with the same seed.

Prints one JSON line: max |a_ref - a_lib|, fidelity, norms, both clbit
strings.
"""

import ctypes
import json
import os
import sys
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(REPO / "rqs-svg_b200"))

import qcs_b200  # noqa: E402
from qcs_b200 import circuits as C  # noqa: E402

REF_SO = REPO / "oracle" / "_ref" / "libqcs_ref.so"


def main():
    n = int(sys.argv[1])
    depth = int(sys.argv[2])
    fusion = {"plain": qcs_b200.FUSION_PLAIN, "greedy": qcs_b200.FUSION_GREEDY}[sys.argv[3]]
    seed = int(os.environ["QCS_REF_SEED"])
    circuit = C.layered_u3_cz_cx_toffoli(n, depth, seed=1)
    meas = [("measure", (q,), (q,), (), ()) for q in range(n)]

    ref_lib = qcs_b200.Library(REF_SO)
    gpu_lib = qcs_b200.Library(qcs_b200.LIB_PATH)
    ref = qcs_b200.Simulator(ref_lib, n, n)
    ref.run(circuit)
    ptr, nbytes = ctypes.c_void_p(), ctypes.c_size_t()
    probe = ref_lib.lib.qcs_ref_stub_largest_buffer
    probe.argtypes = [ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_size_t)]
    found = probe(ctypes.byref(ptr), ctypes.byref(nbytes))
    if not found or nbytes.value != 16 << n:
        raise SystemExit(f"reference state buffer not found (found={found}, bytes={nbytes.value})")
    cudart = ctypes.CDLL("libcudart.so.12")
    cudart.cudaMemcpy.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int]

    lib = qcs_b200.Simulator(gpu_lib, n, n, seed=seed, fusion=fusion)
    lib.run(circuit)

    chunk = 1 << min(n, 24)
    host = np.empty(chunk, dtype=np.complex128)
    max_diff, overlap, norm_ref, norm_lib = 0.0, 0j, 0.0, 0.0
    for start in range(0, 1 << n, chunk):
        # cudaMemcpy on the legacy stream waits for the reference's (blocking) stream
        err = cudart.cudaMemcpy(host.ctypes.data, ptr.value + start * 16, chunk * 16, 2)
        if err != 0:
            raise SystemExit(f"cudaMemcpy failed: {err}")
        mine = lib.amplitudes(np.arange(start, start + chunk, dtype=np.uint64))
        max_diff = max(max_diff, float(np.max(np.abs(mine - host))))
        overlap += np.vdot(host, mine)
        norm_ref += float(np.vdot(host, host).real)
        norm_lib += float(np.vdot(mine, mine).real)

    ref.run(meas)
    lib.run(meas)
    out = {"n": n, "depth": depth, "gates": len(circuit), "fusion": sys.argv[3], "seed": seed,
           "max_abs_diff": max_diff, "fidelity": abs(overlap) ** 2 / (norm_ref * norm_lib),
           "norm_ref": norm_ref, "norm_lib": norm_lib,
           "clbits_ref": ref.clbits_string(), "clbits_lib": lib.clbits_string()}
    lib.close()
    ref.close()
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
