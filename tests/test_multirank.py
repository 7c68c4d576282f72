"""Multi-rank host logic on CPU (gloo, world size 2) through the sharded batch
entry point (shard.run_sharded_batch): independent graphs are placed with
LPT, each rank loads and decomposes only its shard (here the decomposition
call is the CPU oracle, since this host has no GPU; the CUDA batch call it
replaces is covered by the gpu tests), results are gathered on rank 0 in input
order and must equal the oracle's; timings reduce as max over ranks."""
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
    import torch.distributed as dist
    from oracle import oracle as O
    from sparkx_b200 import gen
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    members = [gen.mix_member(i) for i in range(40)]
    members = [m for m in members if m.n <= 20_000][:8]
    works = [shard.work_estimate(m.n, 2 * m.pairs) for m in members]
    loaded = []

    def load(i):  # each rank builds only the graphs placed on it
        loaded.append(i)
        g = gen.mix_graph(members[i])
        return g.offsets, g.neighbours

    def decompose(graphs):  # stands in for the CUDA batch call on a CPU-only host
        return [(O.pkt(off, nbr, threads=2), None, 0) for off, nbr in graphs]

    out = shard.run_sharded_batch(works, load, decompose=decompose)
    ok = sorted(loaded) == out.parts[rank]
    if rank == 0:
        ok &= len(out.results) == len(members)
        for i, m in enumerate(members):
            g = gen.mix_graph(m)
            truss, _, status = out.results[i]
            ok &= status == 0 and bool(np.array_equal(truss, O.pkt(g.offsets, g.neighbours)))
        ok &= out.seconds >= 0.0
    else:
        ok &= out.results is None
    slow = shard.max_over_ranks(float(rank + 1))
    flags = [None] * world
    dist.all_gather_object(flags, ok)
    if rank == 0:
        q.put((all(flags), slow, [len(p) for p in out.parts]))
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
    ok, slow, sizes = q.get(timeout=300)
    for p in procs:
        p.join(timeout=120)
    assert ok
    assert slow == 2.0
    assert sum(sizes) == 8 and min(sizes) >= 1


def test_single_rank_without_process_group():
    from oracle import oracle as O
    from sparkx_b200 import gen
    gs = [gen.rmat(8, 8, seed=s) for s in range(3)]
    out = shard.run_sharded_batch([g.width for g in gs], lambda i: (gs[i].offsets, gs[i].neighbours),
                                  decompose=lambda graphs: [(O.pkt(o, n), None, 0) for o, n in graphs])
    assert out.parts == [[0, 1, 2]]
    for g, (t, _, st) in zip(gs, out.results):
        assert st == 0 and np.array_equal(t, O.pkt(g.offsets, g.neighbours))
