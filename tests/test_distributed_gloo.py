"""Host-side multi-rank logic on CPU (gloo, world_size 2): job sharding is a partition computed
identically on every rank, and the timing reduction is a max over ranks."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from mobileraytracer_b200 import scenes
from mobileraytracer_b200.distributed import job_cost, shard_jobs


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    import torch
    import torch.distributed as dist

    from mobileraytracer_b200.distributed import max_over_ranks, sum_over_ranks
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    jobs = scenes.batched_jobs(64)
    mine = shard_jobs(jobs, world, rank)
    # every rank reports the indices it owns; gather them all
    idx = torch.zeros(64, dtype=torch.int64)
    for j in mine:
        idx[j.index] = rank + 1
    dist.all_reduce(idx)
    t = max_over_ranks(1.5 + rank)
    s = sum_over_ranks(float(len(mine)))
    out[rank] = (idx.tolist(), t, s, sum(job_cost(j) for j in mine))
    dist.barrier()
    dist.destroy_process_group()


def test_sharding_and_timing_over_two_gloo_ranks():
    world = 2
    port = _free_port()
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_worker, args=(world, port, out), nprocs=world, join=True)
    idx0, t0, s0, c0 = out[0]
    idx1, t1, s1, c1 = out[1]
    assert idx0 == idx1
    assert sorted(set(idx0)) == [1, 2]           # every job owned by exactly one rank (1 + rank)
    assert t0 == t1 == 2.5                       # max over ranks
    assert s0 == s1 == 64.0
    assert max(c0, c1) / min(c0, c1) < 1.25      # balanced by estimated cost


def test_single_rank_keeps_everything():
    jobs = scenes.batched_jobs(10)
    assert [j.index for j in shard_jobs(jobs, 1, 0)] == list(range(10))
