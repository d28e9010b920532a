"""The allocation-free squared-norm sums (qcs_b200_zsums_noalloc).

The entry point serves callers that cannot let a library call cudaMalloc
(for example code running inside a framework whose caching allocator owns
the device memory). The caller passes the state and the output in its own
device memory; the scratch is a fixed array inside libqcs.so. Its results
must equal those of the existing entry point (qcs_simulator_expectation_z)
on the same state, call after call, since every call reuses that array.

This file is named so that pytest collects it last.
"""

import ctypes

import numpy as np
import pytest

import qcs_b200
from qcs_b200 import circuits as C

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _noalloc_sums(lib, dev_state, n, dev_out):
    lib.last_error = ""
    ok = lib.lib.qcs_b200_zsums_noalloc(ctypes.c_void_p(dev_state.data_ptr()), n,
                                        ctypes.c_void_p(dev_out.data_ptr()), None)
    return ok


@pytest.mark.parametrize("n", [9, 16, 21])
def test_noalloc_sums_match_expectation_z_twice(gpu_lib, n):
    import torch

    circ = C.layered_u3_cz(n, 3, seed=n) + C.random_circuit(n, 40, seed=n + 1, max_controls=1)
    with qcs_b200.Simulator(gpu_lib, n) as sim:
        sim.run(circ)
        ref_z, ref_norm = sim.expectation_z()
        state = sim.statevector()
    dev_state = torch.from_numpy(np.ascontiguousarray(state).view(np.float64)).cuda()
    dev_out = torch.empty(n + 1, dtype=torch.float64, device="cuda")
    for _ in range(2):
        dev_out.fill_(float("nan"))
        assert _noalloc_sums(gpu_lib, dev_state, n, dev_out) == 1, gpu_lib.last_error
        torch.cuda.synchronize()
        sums = dev_out.cpu().numpy()
        z = (sums[0] - 2.0 * sums[1:]) / sums[0]
        assert abs(sums[0] - ref_norm) <= TOL
        assert np.max(np.abs(z - ref_z)) <= TOL


def test_noalloc_rejects_registers_beyond_its_scratch(gpu_lib):
    import torch

    dev = torch.zeros(4, dtype=torch.float64, device="cuda")
    assert _noalloc_sums(gpu_lib, dev, 41, dev) == 0
    assert "outside [1, 40]" in gpu_lib.last_error
    assert _noalloc_sums(gpu_lib, dev, 0, dev) == 0
