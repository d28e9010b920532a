"""Generate golden fixtures from the reference library.

Runs every case of tests/golden_cases.py through the reference RQS-SVG
library (oracle/_ref/libqcs_ref.so, built from the reference sources by
`make -C oracle ref`) on a GPU, the way bin/qcs drives it, and stores the
final state vectors (as written by its save_statevector) and the clbit
strings of every sample in one compressed .npz.

The reference seeds its measurement engine from std::random_device; the
script re-executes itself with oracle/_ref/libseedshim.so preloaded so that
the seed is golden_cases.SEED.

Usage (on a machine with a GPU and the built reference):
    python tests/golden/make_golden.py --out tests/golden/reference_golden.npz
"""

import argparse
import hashlib
import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parent.parent
sys.path.insert(0, str(REPO / "tests"))
sys.path.insert(0, str(REPO / "rqs-svg_b200"))

import golden_cases  # noqa: E402
import qcs_b200  # noqa: E402

REF_SO = REPO / "oracle" / "_ref" / "libqcs_ref.so"
SHIM_SO = REPO / "oracle" / "_ref" / "libseedshim.so"


def circuit_digest(case) -> str:
    return hashlib.sha256(repr((case["n"], case["mapping"], case["prep"], case["circuit"])).encode()).hexdigest()[:16]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=str(HERE / "reference_golden.npz"))
    ap.add_argument("--only", default=None, help="comma-separated case names")
    args = ap.parse_args()
    if os.environ.get("QCS_REF_SEED") != str(golden_cases.SEED) or str(SHIM_SO) not in os.environ.get("LD_PRELOAD", ""):
        env = dict(os.environ)
        env["QCS_REF_SEED"] = str(golden_cases.SEED)
        env["LD_PRELOAD"] = str(SHIM_SO)
        os.execve(sys.executable, [sys.executable] + sys.argv, env)
    lib = qcs_b200.Library(REF_SO)
    only = set(args.only.split(",")) if args.only else None
    data = {}
    names = []
    for case in golden_cases.cases():
        if only and case["name"] not in only:
            continue
        with qcs_b200.Simulator(lib, case["n"], case["num_clbits"], mapping=case["mapping"]) as sim:
            shots, state = golden_cases.run_case(sim, case)
        key = case["name"]
        names.append(key)
        data[f"{key}/state"] = state
        data[f"{key}/shots"] = np.array(shots, dtype="U64")
        data[f"{key}/digest"] = np.array(circuit_digest(case))
        print(f"{key}: n={case['n']} samples={case['samples']} shots={shots[:4]}", flush=True)
    data["__cases__"] = np.array(names)
    data["__seed__"] = np.array(golden_cases.SEED)
    np.savez_compressed(args.out, **data)
    print(f"wrote {len(names)} cases to {args.out}")


if __name__ == "__main__":
    main()
