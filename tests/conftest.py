"""Shared fixtures. GPU tests are marked `gpu`; everything else runs on CPU."""

import os
import sys
from pathlib import Path

import pytest

REPO = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(REPO / "rqs-svg_b200"))
sys.path.insert(0, str(REPO / "tests"))

ORACLE_SO = REPO / "oracle" / "liboracle_qcs.so"
PRODUCT_SO = REPO / "rqs-svg_b200" / "lib" / "libqcs.so"
GOLDEN_DIR = REPO / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (runs the CUDA library)")


@pytest.fixture(scope="session")
def oracle_lib():
    import qcs_b200

    if not ORACLE_SO.exists():
        pytest.fail("oracle/liboracle_qcs.so is missing: run `make -C oracle`")
    return qcs_b200.Library(ORACLE_SO)


@pytest.fixture(scope="session")
def gpu_lib():
    """The B200 library. On a GPU test run a missing build or device is a
    failure, never a silent fallback."""
    import qcs_b200

    if not PRODUCT_SO.exists():
        pytest.fail("rqs-svg_b200/lib/libqcs.so is missing: run `make -C rqs-svg_b200`")
    return qcs_b200.Library(PRODUCT_SO)
