"""Multi-GPU plumbing: one process per GPU, torch.distributed for the host-side coordination.

Rendering has no exchange step (pixels, samples and jobs are independent: Renderer.cpp:78-108), so
nothing crosses GPUs on the data path:
  * one frame per rank (replicas: every rank renders its own frame or job list);
  * job streams are sharded across ranks by estimated cost (largest first onto the least-loaded
    rank), each rank keeping the scenes it was given resident on its own GPU;
  * the only collectives are for timing (max over ranks) and for gathering per-job records.
"""
from __future__ import annotations

import heapq
from typing import Sequence


def job_cost(job) -> float:
    """Estimated work of a render job: camera paths x log of the triangle count (traversal depth)."""
    import math
    return float(job.side * job.side * job.spp) * max(1.0, math.log2(max(2, job.n_triangles)))


def shard_jobs(jobs: Sequence, world: int, rank: int) -> list:
    """Jobs assigned to `rank`: longest-processing-time-first onto the least loaded rank.  Every
    rank computes the same assignment from the same list, so no communication is needed."""
    if world <= 1:
        return list(jobs)
    heap = [(0.0, r) for r in range(world)]
    assign = {r: [] for r in range(world)}
    for j in sorted(jobs, key=lambda j: (-job_cost(j), j.index)):
        load, r = heapq.heappop(heap)
        assign[r].append(j)
        heapq.heappush(heap, (load + job_cost(j), r))
    return sorted(assign[rank], key=lambda j: j.index)


def max_over_ranks(value: float, device=None) -> float:
    """Maximum of a per-rank scalar (device time of the timed region)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return value
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value: float, device=None) -> float:
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return value
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())
