"""Allocation failures inside allocate_memory, made on the host.

QCS_FAIL_ALLOC_AFTER=k makes allocation k of the next allocate_memory call
fail as if the device (or pinned host) memory were exhausted. For every k:
the call returns 0 with a message (the reference's 1/0 + callback
convention, src/qcs.cu:2964-2999), the simulator is left unallocated (other
calls report that allocate_memory must come first instead of launching on
missing buffers), the memory of the allocations made before the failure is
released, and a retry without the hook allocates and runs a circuit whose
state and clbits equal the oracle's. No GPU fault is involved: the failure
is thrown on the host before the allocation it stands for.
"""

import numpy as np
import pytest

import qcs_b200
from qcs_b200 import circuits as C

pytestmark = pytest.mark.gpu

# allocations allocate_memory makes: the state, four device scratch buffers,
# two pinned host buffers, the tensor passes' host-mapped error flag
ALLOCATIONS = 8
N = 22   # a 64 MiB state: a leaked one shows in the free device memory


@pytest.mark.parametrize("k", range(ALLOCATIONS + 1))
def test_failed_allocation_leaves_the_simulator_unallocated(gpu_lib, oracle_lib, monkeypatch, k):
    import torch

    circ = C.layered_u3_cz(N, 2, seed=k + 1) + [("measure", (q,), (q,), (), ()) for q in range(0, N, 5)]
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info()[0]
    with qcs_b200.Simulator(gpu_lib, N, N, seed=11, allocate=False) as sim:
        monkeypatch.setenv("QCS_FAIL_ALLOC_AFTER", str(k))
        if k < ALLOCATIONS:
            with pytest.raises(qcs_b200.QCSError, match=f"injected failure of allocation {k}"):
                gpu_lib.call("qcs_simulator_allocate_memory", sim.h)
            with pytest.raises(qcs_b200.QCSError, match="allocate_memory must be called first"):
                sim.measure(0)
            with pytest.raises(qcs_b200.QCSError, match="allocate_memory must be called first"):
                sim.gate("h", (), (0,))
            torch.cuda.synchronize()
            assert free_before - torch.cuda.mem_get_info()[0] < (32 << 20), k
            monkeypatch.delenv("QCS_FAIL_ALLOC_AFTER")
        gpu_lib.call("qcs_simulator_allocate_memory", sim.h)
        sim.run(circ)
        got, bits = sim.statevector(), sim.clbits_string()
    with qcs_b200.Simulator(oracle_lib, N, N, seed=11) as ref:
        ref.run(circ)
        want, want_bits = ref.statevector(), ref.clbits_string()
    assert bits == want_bits
    assert np.max(np.abs(got - want)) <= 1e-12
    torch.cuda.synchronize()
    assert free_before - torch.cuda.mem_get_info()[0] < (32 << 20), k
