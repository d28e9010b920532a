"""CPU checks of the drop-in boundary: libqcs.so loads and exports every
function include/*.h declares; the oracle exports the reference's 64; the CLI
validates its arguments. No call here touches a GPU."""

import re
import subprocess
from pathlib import Path

import pytest

import qcs_b200

REPO = Path(__file__).resolve().parent.parent


def declared(header):
    text = (REPO / "include" / header).read_text()
    # extern "C" functions are the int-returning declarations outside the
    # __cplusplus block of *_cxx functions
    return sorted(set(re.findall(r"^int (qcs_[a-z0-9_]+)\(", text, re.M)) - {
        n for n in re.findall(r"^int (qcs_[a-z0-9_]+_cxx)\(", text, re.M)})


def exported(so):
    out = subprocess.run(["nm", "-D", "--defined-only", str(so)], capture_output=True, text=True, check=True).stdout
    return {line.split()[-1] for line in out.splitlines() if line.strip()}


def test_reference_api_has_64_functions():
    assert len(declared("qcs.h")) == 64


def test_product_exports_every_declared_function():
    syms = exported(qcs_b200.LIB_PATH)
    missing = [f for f in declared("qcs.h") + declared("qcs_b200.h") if f not in syms]
    assert not missing, missing


def test_product_exports_cxx_entry_points():
    syms = exported(qcs_b200.LIB_PATH)
    text = (REPO / "include" / "qcs.h").read_text()
    cxx = re.findall(r"(qcs_[a-z0-9_]+_cxx)\(", text)
    demangled = subprocess.run(["c++filt"], input="\n".join(syms), capture_output=True, text=True).stdout
    missing = [f for f in cxx if f + "(" not in demangled]
    assert not missing, missing


def test_product_exports_nothing_else():
    syms = exported(qcs_b200.LIB_PATH)
    demangled = subprocess.run(["c++filt"], input="\n".join(sorted(syms)), capture_output=True, text=True).stdout.splitlines()
    stray = [s for s in demangled if "qcs" not in s and not s.startswith(("_init", "_fini", "__", "_end", "_edata", "_ITM"))]
    # the static CUDA runtime may contribute no exported symbols either
    assert len(stray) < 5, stray[:20]


def test_product_library_loads_without_gpu():
    lib = qcs_b200.Library(qcs_b200.LIB_PATH)
    assert lib.has("qcs_simulator_gate_rcccx") and lib.has("qcs_simulator_sample")


def test_oracle_exports_reference_api():
    syms = exported(REPO / "oracle" / "liboracle_qcs.so")
    assert all(f in syms for f in declared("qcs.h"))


def test_cli_rejects_missing_circuit():
    r = subprocess.run([str(qcs_b200.CLI_PATH)], capture_output=True, text=True)
    assert r.returncode == 1 and "user circuit shared object path is required" in r.stderr


def test_cli_rejects_nonpositive_samples():
    r = subprocess.run([str(qcs_b200.CLI_PATH), "-s", "0", "x.so"], capture_output=True, text=True)
    assert r.returncode == 1 and "num_samples must be greater than 0" in r.stderr


def test_cli_help_lists_reference_options():
    r = subprocess.run([str(qcs_b200.CLI_PATH), "--help"], capture_output=True, text=True)
    assert r.returncode == 0
    for opt in ("--num-samples", "--mapping", "--reversed-mapping", "--output-statevector"):
        assert opt in r.stdout


def test_python_structs_match_the_c_header(tmp_path):
    """The ctypes mirrors of the extension structs have the C layout."""
    import ctypes

    src = tmp_path / "sizes.c"
    src.write_text(
        '#include <stddef.h>\n#include <stdio.h>\n#include "qcs_b200.h"\n'
        "int main(void) {\n"
        '  printf("%zu %zu %zu %zu %zu %zu %zu\\n", sizeof(qcs_b200_gate), offsetof(qcs_b200_gate, params),\n'
        "         offsetof(qcs_b200_gate, num_targets), offsetof(qcs_b200_gate, qubits),\n"
        "         sizeof(qcs_b200_batch_info), offsetof(qcs_b200_batch_info, amplitudes),\n"
        "         offsetof(qcs_b200_batch_info, last_run_ms));\n"
        "  return 0;\n}\n")
    exe = tmp_path / "sizes"
    inc = Path(__file__).resolve().parent.parent / "include"
    subprocess.run(["gcc", "-std=c11", f"-I{inc}", str(src), "-o", str(exe)], check=True)
    got = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    G, I = qcs_b200.BatchGate, qcs_b200.BatchInfo
    want = [ctypes.sizeof(G), G.params.offset, G.num_targets.offset, G.qubits.offset,
            ctypes.sizeof(I), I.amplitudes.offset, I.last_run_ms.offset]
    assert got == want
