"""Host side of `bench.py --gpus N` (replicas): two gloo ranks on the CPU.

The single-mesh path does not shard, so N GPUs run N identical replicas; the bench brackets
the timed steps with barriers, takes the max of the per-rank times and reports all ranks'
tets over that time. These tests run the same helpers with world size 2 on gloo, each rank
evaluating its replica on the oracle, and check that the replicas agree bit for bit, that
the reported time is the slowest rank's and that the throughput counts every rank's work.
"""

import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out_dir):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    sys.path.insert(0, str(ROOT))
    import torch
    import torch.distributed as dist

    import bench
    import oracle
    from litepgo_b200 import workloads

    r, w, local = bench.dist_setup(world)
    assert (r, w, local) == (rank, world, rank)
    assert dist.get_backend() == "gloo"
    g = workloads.gravity_box(4, seed=0)
    u = bench.state(g["X"])
    m = oracle.OracleMesh(g["X"], g["tets"], g["theta"])
    bench.barrier(w)
    E, grad, _ = m.eval(u, True, 1)
    # A rank-dependent "time" so the max is known: rank 1 is the slow one.
    local_seconds = 0.25 + 0.5 * rank
    slowest = bench.max_over_ranks(local_seconds, w)
    bench.barrier(w)
    checks = torch.tensor([E, float(np.sum(grad * np.arange(grad.size)))], dtype=torch.float64)
    gathered = [torch.zeros_like(checks) for _ in range(w)]
    dist.all_gather(gathered, checks)
    T = g["tets"].shape[0]
    rate = bench.whole_job_rate(T * 3, slowest, w)
    np.save(Path(out_dir) / f"rank{rank}.npy",
            np.array([slowest, rate, T] + [float(x) for t in gathered for x in t], dtype=np.float64))
    dist.destroy_process_group()


def test_replicas_two_gloo_ranks(tmp_path):
    import torch.multiprocessing as mp

    world = 2
    mp.start_processes(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    rows = [np.load(tmp_path / f"rank{r}.npy") for r in range(world)]
    for row in rows:
        slowest, rate, T = row[:3]
        assert slowest == 0.75  # max over ranks, not this rank's own time
        assert rate == world * T * 3 / 0.75
        e0, c0, e1, c1 = row[3:]
        assert e0 == e1 and c0 == c1  # identical replicas, identical results
    assert np.array_equal(rows[0], rows[1])


def test_whole_job_rate_single_rank():
    sys.path.insert(0, str(ROOT))
    import bench

    assert bench.whole_job_rate(1000, 2.0, 1) == 500.0
    assert bench.whole_job_rate(1000, 2.0, 4) == 2000.0
