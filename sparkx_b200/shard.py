"""Placement of independent graphs across ranks (one process per GPU).

A single graph does not shard: PKT's sub-level barrier would need a cross-GPU
support-decrement exchange per sub-level.  Batches of independent graphs do:
they are partitioned with greedy longest-processing-time-first on an estimate
of each graph's work, with no collective on the data path; only per-rank
timings are reduced (max over ranks).
"""
from __future__ import annotations

import dataclasses
import heapq
import time


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


@dataclasses.dataclass
class ShardedBatch:
    """Outcome of :func:`run_sharded_batch` on one rank."""
    results: list | None       # (truss, stats, status) per graph in input order (on ``dst``; else None)
    local: dict                # this rank's own results, keyed by input index
    parts: list                # LPT placement: input indices per rank
    seconds: float             # slowest rank's decomposition time


def run_sharded_batch(works, load, opts=None, hbm_budget_bytes: int = 0, decompose=None, dst: int = 0,
                      gather: bool = True) -> ShardedBatch:
    """Decompose independent graphs across the ranks of the default process group.

    ``works[i]`` is graph i's work estimate (``work_estimate(n, width)``) and
    ``load(i)`` returns its (offsets, neighbours): every rank sees the same
    placement (LPT on ``works``) and loads only its own graphs, decomposes them
    with one ``run_batch`` call (``decompose``, default the CUDA engine's
    batch entry point: unions under the HBM budget, one launch per wave), and
    the (truss, stats, status) tuples are gathered on rank ``dst`` in input
    order.  No collective touches the decomposition itself: graphs are
    independent, so the only exchanges are the gather of results and the max of
    the per-rank times.  Without an initialised process group this is a
    single-rank run.
    """
    import torch.distributed as dist
    distributed = dist.is_available() and dist.is_initialized()
    rank = dist.get_rank() if distributed else 0
    world = dist.get_world_size() if distributed else 1
    parts = assign_lpt(list(works), world)
    mine = parts[rank]
    if decompose is None:
        from .pkt import run_batch

        def decompose(graphs):
            return run_batch(graphs, opts, hbm_budget_bytes)
    graphs = [load(i) for i in mine]
    t0 = time.perf_counter()
    res = decompose(graphs) if graphs else []
    dt = time.perf_counter() - t0
    local = {i: r for i, r in zip(mine, res)}
    slowest = max_over_ranks(dt) if distributed else dt
    if not gather:
        return ShardedBatch(None, local, parts, slowest)
    if not distributed:
        return ShardedBatch([local[i] for i in range(len(parts[0]))], local, parts, slowest)
    box = [None] * world if rank == dst else None
    dist.gather_object(local, box, dst=dst)
    merged = None
    if rank == dst:
        allres = {}
        for part in box:
            allres.update(part)
        merged = [allres[i] for i in range(len(allres))]
    return ShardedBatch(merged, local, parts, slowest)
