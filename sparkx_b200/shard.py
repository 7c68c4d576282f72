"""Placement of independent graphs across ranks (one process per GPU).

A single graph does not shard: PKT's sub-level barrier would need a cross-GPU
support-decrement exchange per sub-level.  Batches of independent graphs do:
they are partitioned with greedy longest-processing-time-first on an estimate
of each graph's work, with no collective on the data path; only per-rank
timings are reduced (max over ranks).
"""
from __future__ import annotations

import heapq


def work_estimate(n: int, width: int) -> float:
    """Relative cost of one decomposition (CSR slots dominate; vertices add a little)."""
    return float(width) + 0.25 * float(n)


def assign_lpt(works, world: int):
    """Indices of `works` per rank, longest first onto the least-loaded rank.
    Deterministic: ties go to the lower rank / lower index."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(works)), key=lambda i: (-works[i], i))
    heap = [(0.0, r) for r in range(world)]
    heapq.heapify(heap)
    out = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + works[i], r))
    for r in range(world):
        out[r].sort()
    return out


def max_over_ranks(value: float, device=None) -> float:
    """Max of a per-rank scalar (timings are reported as the slowest rank)."""
    import torch
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized():
        return value
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
