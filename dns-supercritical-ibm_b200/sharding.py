"""Host-side multi-GPU plumbing of the projection engine.

One projection fits on one B200, so the engine scales by replicas: every rank
(one process per GPU, ``torch.distributed``) solves its own cases, and the only
collectives are a barrier and the timing reduction.  Independent cases -- the
batched solves and served requests -- are partitioned across ranks by size;
nothing crosses GPUs on the data path.
"""
from __future__ import annotations

import heapq


def partition_cases(points, world: int):
    """Assign cases (their point counts) to ``world`` ranks, largest first onto the least
    loaded rank (longest-processing-time rule; ties go to the lower rank).  Returns, per
    rank, the sorted list of case indices.  Deterministic, so every rank computes the same
    assignment without communication."""
    if world < 1:
        raise ValueError("world must be >= 1")
    heap = [(0, r) for r in range(world)]
    out = [[] for _ in range(world)]
    for idx in sorted(range(len(points)), key=lambda i: (-points[i], i)):
        load, r = heapq.heappop(heap)
        out[r].append(idx)
        heapq.heappush(heap, (load + points[idx], r))
    return [sorted(v) for v in out]


def max_over_ranks(value: float, dist=None, device=None) -> float:
    """Max of a per-rank scalar over all ranks (the rank itself when not distributed).  The
    tensor lives on ``device`` (a CUDA device for NCCL, the CPU for gloo)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device or "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(points_per_rank_step, steps: int, world: int, ms_max: float) -> float:
    """Whole-job Gpts/s: the points of all ranks over the slowest rank's device time."""
    return world * points_per_rank_step * steps / (ms_max / 1e3) / 1e9
