"""Parity at the workloads' full sizes against the reference library built
from its own sources for sm_100a, run on the same GPU with the same seed:

- the 30-qubit layered circuit (1820 gates, depth 40): every amplitude to
  1e-12 and fidelity >= 1 - 1e-12, then the 30 measurement outcomes
  (src/qcs.cu:2545-2677) identical, for the fused (default) and the plain
  path;
- the 20-qubit, depth-20 layered U3 + CZ circuit through both drivers
  (`bin/qcs -s 1024` and the reference's own bin/qcs, src/qcs_main.cpp:153-193):
  the clbit strings of all 1024 samples identical and the saved state
  (src/qcs.cu:2494-2543) equal to 1e-12.

Both need the reference build (`make -C oracle ref` where the reference
sources are) and its seed shim; a missing build fails the test.
"""

import json
import os
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np
import pytest

import qcs_b200
from qcs_b200 import circuits as C

pytestmark = pytest.mark.gpu

REPO = Path(__file__).resolve().parent.parent
REF_DIR = REPO / "oracle" / "_ref"
SHIM = REF_DIR / "libseedshim.so"
SEED = 20251203


def _need_reference():
    for f in (REF_DIR / "libqcs_ref.so", SHIM, REF_DIR / "qcs_ref"):
        if not f.exists():
            pytest.fail(f"{f} is missing: run `make -C oracle ref` where the reference sources are")


@pytest.mark.parametrize("fusion", ["greedy", "plain"])
def test_layered_30_qubits_matches_reference_build(fusion):
    _need_reference()
    env = dict(os.environ)
    env.update({"LD_PRELOAD": str(SHIM), "QCS_REF_SEED": str(SEED)})
    r = subprocess.run([sys.executable, str(REPO / "tests" / "reference_scale_check.py"), "30", "40", fusion],
                       capture_output=True, text=True, env=env, timeout=900)
    assert r.returncode == 0, r.stderr[-2000:]
    res = json.loads(r.stdout.strip().splitlines()[-1])
    print(res)
    assert res["gates"] == 1820
    assert res["max_abs_diff"] <= 1e-12, res
    assert res["fidelity"] >= 1 - 1e-12, res
    assert abs(res["norm_ref"] - 1) < 1e-10 and abs(res["norm_lib"] - 1) < 1e-10, res
    assert len(res["clbits_lib"]) == 30
    assert res["clbits_lib"] == res["clbits_ref"], res


def test_cli_1024_samples_at_20_qubits_match_reference_driver():
    _need_reference()
    n, depth, samples = 20, 20, 1024
    circ = C.layered_u3_cz(n, depth, seed=1, measure=True)
    plug = REPO / "rqs-svg_b200" / "examples" / "gatelist.so"
    with tempfile.TemporaryDirectory() as d:
        gl = Path(d) / "c.txt"
        gl.write_text(C.to_gatelist(circ, n, n))
        outs = []
        for exe in (qcs_b200.CLI_PATH, REF_DIR / "qcs_ref"):
            sv = Path(d) / f"{exe.name}.bin"
            env = dict(os.environ)
            env.update({"QCS_GATELIST": str(gl), "LD_PRELOAD": str(SHIM), "QCS_REF_SEED": str(SEED)})
            r = subprocess.run([str(exe), "-s", str(samples), "--output-statevector", str(sv), str(plug)],
                               capture_output=True, text=True, env=env, timeout=900)
            assert r.returncode == 0, r.stderr[-2000:]
            lines = [json.loads(x) for x in r.stdout.splitlines() if x.startswith("{")]
            assert [ln["sample_num"] for ln in lines] == list(range(samples))
            outs.append(([ln["clbits"] for ln in lines], np.fromfile(sv, dtype=np.complex128)))
    mine, theirs = outs
    differing = [i for i, (a, b) in enumerate(zip(mine[0], theirs[0])) if a != b]
    assert not differing, f"samples {differing[:10]} differ"
    assert len(set(mine[0])) > 1   # the shots are not all one outcome
    assert mine[1].size == 1 << n
    assert np.max(np.abs(mine[1] - theirs[1])) <= 1e-12
