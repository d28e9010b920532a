"""Replica coordination of bench.py on CPU: two gloo ranks (127.0.0.1)
agree on the barrier and on the max-over-ranks timing aggregation, and each
rank's replica computes the same circuit result as the other."""

import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest

REPO = Path(__file__).resolve().parent.parent


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out_dir):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "RANK": str(rank),
                       "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank)})
    sys.path.insert(0, str(REPO))
    sys.path.insert(0, str(REPO / "rqs-svg_b200"))
    import bench
    import qcs_b200
    from qcs_b200 import circuits as C

    bench.WORLD = world
    dist = bench.dist_init("gloo")
    # each replica runs the same small circuit on the CPU oracle
    lib = qcs_b200.Library(REPO / "oracle" / "liboracle_qcs.so")
    with qcs_b200.Simulator(lib, 8, seed=3) as sim:
        sim.run(C.layered_u3_cz(8, 3, seed=1))
        z, norm = sim.expectation_z()
    bench.barrier(dist)
    times = [0.5 + rank, 0.25 * (rank + 1)]   # rank 1 is the slowest
    agg = bench.aggregate_replica_times(dist, times, world)
    np.save(os.path.join(out_dir, f"rank{rank}.npy"), np.array([agg["total_s"], agg["value"], norm] + list(z)))
    dist.destroy_process_group()


def test_two_gloo_replicas_agree(tmp_path):
    import torch.multiprocessing as mp

    port = _free_port()
    mp.start_processes(_worker, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    r0 = np.load(tmp_path / "rank0.npy")
    r1 = np.load(tmp_path / "rank1.npy")
    # slowest rank total = 1.5 + 0.5 = 2.0 s over 2 steps and 2 replicas
    assert r0[0] == pytest.approx(2.0) and r1[0] == pytest.approx(2.0)
    assert r0[1] == pytest.approx(0.5) and r1[1] == pytest.approx(0.5)
    assert np.array_equal(r0[2:], r1[2:])
