"""Multi-rank host logic on CPU (gloo, world size 2): independent graphs are
sharded with LPT, each rank decomposes its shard (here with the CPU oracle,
the GPU path being covered by the gpu tests), results are gathered and must
equal a single-rank run; timings reduce as max over ranks."""
import os

import numpy as np
import torch.multiprocessing as mp

from sparkx_b200 import shard


def test_lpt_balanced_and_complete():
    works = [100, 1, 1, 50, 50, 99, 3, 7, 7, 60]
    parts = shard.assign_lpt(works, 3)
    assert sorted(i for p in parts for i in p) == list(range(len(works)))
    loads = [sum(works[i] for i in p) for p in parts]
    assert max(loads) - min(loads) <= max(works)
    assert shard.assign_lpt(works, 3) == parts
    assert shard.assign_lpt([5, 5], 4)[2:] == [[], []]


def _worker(rank, world, port, q):
    import torch
    import torch.distributed as dist
    from oracle import oracle as O
    from sparkx_b200 import gen
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    members = [gen.mix_member(i) for i in range(40)]
    members = [m for m in members if m.n <= 20_000][:8]
    graphs = [gen.mix_graph(m) for m in members]
    parts = shard.assign_lpt([shard.work_estimate(g.n, g.width) for g in graphs], world)
    mine = {}
    for i in parts[rank]:
        mine[i] = O.pkt(graphs[i].offsets, graphs[i].neighbours, threads=2)
    gathered = [None] * world
    dist.all_gather_object(gathered, mine)
    slow = shard.max_over_ranks(float(rank + 1))
    if rank == 0:
        merged = {}
        for part in gathered:
            merged.update(part)
        ok = sorted(merged) == list(range(len(graphs)))
        for i, g in enumerate(graphs):
            ok &= bool(np.array_equal(merged[i], O.pkt(g.offsets, g.neighbours)))
        q.put((ok, slow))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_gloo_sharded_batch():
    import random
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + random.randint(0, 2000)
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    ok, slow = q.get(timeout=300)
    for p in procs:
        p.join(timeout=120)
    assert ok
    assert slow == 2.0
