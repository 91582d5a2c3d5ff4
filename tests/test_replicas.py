"""bench.py's multi-GPU path is replicas only: every rank runs its own
iteration, and the job time is the maximum over ranks. The rank logic runs
here as two gloo processes on CPU."""
import os
import sys

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _worker(rank, world, port, q):
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    per_rank_ms = [120.0, 175.5][rank]
    got = bench.max_over_ranks(per_rank_ms, world, "cpu")
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, got))


def test_job_time_is_the_slowest_replica():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 2000
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = dict(q.get(timeout=10) for _ in range(2))
    assert res == {0: 175.5, 1: 175.5}


def test_single_rank_needs_no_collective():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.5, 1, "cpu") == 3.5
