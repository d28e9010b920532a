"""bin/qcs end to end on the GPU: per-sample JSON lines, clbit strings under
a pinned seed, --output-statevector, --mapping and --reversed-mapping,
compared with the oracle driven the way the reference driver drives the
library (src/qcs_main.cpp:64-201)."""

import json
import os
import subprocess
import tempfile
from pathlib import Path

import numpy as np
import pytest

import golden_cases
import qcs_b200
from qcs_b200 import circuits as C

pytestmark = pytest.mark.gpu

REPO = Path(__file__).resolve().parent.parent
SHIM = REPO / "oracle" / "_ref" / "libseedshim.so"
GATELIST_SO = REPO / "rqs-svg_b200" / "examples" / "gatelist.so"
GHZ_SO = REPO / "rqs-svg_b200" / "examples" / "ghz.so"


def _run_cli(args, env_extra):
    env = dict(os.environ)
    env.update(env_extra)
    r = subprocess.run([str(qcs_b200.CLI_PATH)] + args, capture_output=True, text=True, env=env, timeout=300)
    assert r.returncode == 0, r.stderr
    return [json.loads(line) for line in r.stdout.splitlines() if line.strip()]


def _oracle_samples(oracle_lib, n, circ, samples, seed, mapping=None):
    case = dict(name="cli", n=n, num_clbits=n, mapping=mapping, prep="zero", circuit=circ, samples=samples)
    with qcs_b200.Simulator(oracle_lib, n, n, mapping=mapping, seed=seed) as sim:
        return golden_cases.run_case(sim, case)


@pytest.mark.parametrize("fusion", ["0", "1"])
def test_cli_samples_and_statevector_match_oracle(oracle_lib, fusion):
    if not SHIM.exists():
        pytest.fail("oracle/_ref/libseedshim.so is missing: run `make -C oracle ref`")
    n, samples, seed = 8, 12, 777
    circ = C.layered_u3_cz(n, 4, seed=3, measure=True)
    with tempfile.TemporaryDirectory() as d:
        gl = Path(d) / "c.txt"
        gl.write_text(C.to_gatelist(circ, n, n))
        sv = Path(d) / "sv.bin"
        lines = _run_cli(["-s", str(samples), "--output-statevector", str(sv), str(GATELIST_SO)],
                         {"QCS_GATELIST": str(gl), "LD_PRELOAD": str(SHIM), "QCS_REF_SEED": str(seed),
                          "QCS_FUSION": fusion})
        shots, state = _oracle_samples(oracle_lib, n, circ, samples, seed)
        assert [ln["sample_num"] for ln in lines] == list(range(samples))
        assert [ln["clbits"] for ln in lines] == shots
        assert all(ln["elapsed_time"] > 0 for ln in lines)
        got = np.fromfile(sv, dtype=np.complex128)
        assert np.max(np.abs(got - state)) <= 1e-12


@pytest.mark.parametrize("reverse", [False, True])
def test_cli_mapping_options(oracle_lib, reverse):
    n = 6
    p2l = [2, 0, 5, 1, 4, 3]
    circ = C.random_circuit(n, 40, seed=8, max_controls=1)
    with tempfile.TemporaryDirectory() as d:
        gl = Path(d) / "c.txt"
        gl.write_text(C.to_gatelist(circ, n, 0))
        sv = Path(d) / "sv.bin"
        args = ["--mapping", ",".join(map(str, p2l))] + (["-r"] if reverse else [])
        _run_cli(args + ["--output-statevector", str(sv), str(GATELIST_SO)], {"QCS_GATELIST": str(gl)})
        mapping = p2l
        if reverse:
            inv = [0] * n
            for p, lq in enumerate(p2l):
                inv[lq] = p
            mapping = inv
        with qcs_b200.Simulator(oracle_lib, n, mapping=mapping) as sim:
            sim.run(circ)
            ref = sim.statevector()
        assert np.max(np.abs(np.fromfile(sv, dtype=np.complex128) - ref)) <= 1e-12


REF_CLI = REPO / "oracle" / "_ref" / "qcs_ref"


@pytest.mark.parametrize("fusion", ["0", "1"])
def test_cli_matches_reference_cli(fusion):
    """Both drivers, same plug-in, same pinned seed: identical JSON clbits on
    every sample and the same saved state."""
    if not REF_CLI.exists():
        pytest.fail("oracle/_ref/qcs_ref is missing: run `make -C oracle ref` where the reference sources are")
    n, samples, seed = 10, 24, 4242
    circ = C.layered_u3_cz(n, 5, seed=11)
    circ += [("measure", (q,), (q,), (), ()) for q in range(0, n, 2)]
    circ += C.random_circuit(n, 30, seed=12, max_controls=1, gates=["u3", "x", "h", "rz"])
    circ += [("measure", (q,), (q,), (), ()) for q in range(n)]
    with tempfile.TemporaryDirectory() as d:
        gl = Path(d) / "c.txt"
        gl.write_text(C.to_gatelist(circ, n, n))
        outs = []
        for exe in (qcs_b200.CLI_PATH, REF_CLI):
            sv = Path(d) / f"{exe.name}.bin"
            env = dict(os.environ)
            env.update({"QCS_GATELIST": str(gl), "LD_PRELOAD": str(SHIM), "QCS_REF_SEED": str(seed),
                        "QCS_FUSION": fusion})
            r = subprocess.run([str(exe), "-s", str(samples), "--output-statevector", str(sv), str(GATELIST_SO)],
                               capture_output=True, text=True, env=env, timeout=300)
            assert r.returncode == 0, r.stderr
            lines = [json.loads(x) for x in r.stdout.splitlines() if x.startswith("{")]
            outs.append(([ln["clbits"] for ln in lines], np.fromfile(sv, dtype=np.complex128)))
        assert outs[0][0] == outs[1][0]
        assert np.max(np.abs(outs[0][1] - outs[1][1])) <= 1e-12


def test_cli_ghz_shots_are_all_zero_or_all_one():
    lines = _run_cli(["-s", "32", str(GHZ_SO)], {"NUM_QUBITS": "16"})
    assert len(lines) == 32
    assert all(ln["clbits"] in ("0" * 16, "1" * 16) for ln in lines)
