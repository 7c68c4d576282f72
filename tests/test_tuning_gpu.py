"""The tuned knobs change time only: every candidate the autotuner can pick
gives the oracle's truss numbers bit for bit, on single graphs and on batched
unions (whose members now get hub maps of their own); the autotuner stores a
valid choice that later launches with the same key use."""
import itertools

import numpy as np
import pytest

from oracle import oracle as O
from sparkx_b200 import gen
import sparkx_b200.pkt as P

pytestmark = pytest.mark.gpu
O32 = P.PktOptions(out_bits=32, timeout_ms=120_000)

CANDIDATES = [P.PktTuning(merge_ratio=mr, hub_min_degree=h, sample_min=smp, support_kernel=sk, compact_pct=cp,
                          hash_min_degree=hm, sup_hash_min=sh)
              for mr, h, smp, sk, cp, hm, sh in itertools.product((4, 16), (0, 256, 4096), (32, 256), (1, 2),
                                                                  (75, 95), (0, 8, 64), (0, 4, 64))]


@pytest.fixture(scope="module", autouse=True)
def _engine():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    from sparkx_b200 import build
    build.build_engine()
    P.tuning_clear()
    yield
    P.tuning_clear()


def _with_tuning(t, fn):
    """Run fn once to learn its launch key, then again with t stored under that key."""
    fn()
    _, key = P.tuning_last()
    P.tuning_store(key, t)
    try:
        out = fn()
        used, _ = P.tuning_last()
        assert used == t
        return out
    finally:
        P.tuning_clear()


def test_every_candidate_gives_the_same_truss():
    # R-MAT-16 has rows past 1024 and 4096 entries (hub maps) and is big enough to compact
    g = gen.rmat(16, 16, seed=2)
    want = O.fast_truss(g.offsets, g.neighbours)[0]
    for t in CANDIDATES[::13]:
        got, st = _with_tuning(t, lambda: P.run_pkt(g.offsets, g.neighbours, O32))
        assert np.array_equal(got, want), t
        assert (st.hub_maps > 0) == (t.hub_min_degree in (256, 4096)), (t, st.hub_maps)


def test_batched_unions_get_member_hub_maps():
    members = [gen.rmat(13, 16, seed=s) for s in range(3)] + [gen.erdos_renyi(4000, 40000, 5),
                                                              gen.rmat(12, 32, seed=9)]
    want = [O.fast_truss(m.offsets, m.neighbours)[0] for m in members]
    pairs = [(m.offsets, m.neighbours) for m in members]
    for t in (P.PktTuning(hub_min_degree=256), P.PktTuning(hub_min_degree=256, merge_ratio=4, compact_pct=95),
              P.PktTuning(hub_min_degree=0), P.PktTuning(hub_min_degree=1024, hash_min_degree=16),
              P.PktTuning(sup_hash_min=4), P.PktTuning(sup_hash_min=32, support_kernel=2)):
        res = _with_tuning(t, lambda: P.run_batch(pairs, O32))
        for w, (truss, st, status) in zip(want, res):
            assert status == 0 and np.array_equal(truss, w), t


def test_tight_batch_budget_runs_without_the_hash_tables():
    """Unions packed up to a small budget leave no room for the row hash tables
    (32 B per slot): they run without them and give the same truss numbers."""
    members = [gen.rmat(13, 16, seed=s) for s in range(8)]
    want = [O.fast_truss(m.offsets, m.neighbours)[0] for m in members]
    pairs = [(m.offsets, m.neighbours) for m in members]
    for budget in (200 << 20, 260 << 20, 0):  # a union holds 128 MB of staging buffers and hub maps
        res = P.run_batch(pairs, O32, hbm_budget_bytes=budget)
        for w, (truss, st, status) in zip(want, res):
            assert status == 0 and np.array_equal(truss, w), budget


def test_support_hash_on_multigraphs_and_support_only():
    """The hashed out-list probe finds every copy's run the same way the
    search does: weighted supports and the peel over them are unchanged."""
    g = gen.with_parallel_edges(gen.rmat(12, 16, seed=6), 0.25, seed=6)
    want = O.pkt(g.offsets, g.neighbours, threads=4)
    for t in (P.PktTuning(sup_hash_min=4), P.PktTuning(sup_hash_min=16, support_kernel=2)):
        got, _ = _with_tuning(t, lambda: P.run_pkt(g.offsets, g.neighbours, O32))
        assert np.array_equal(got, want), t
    h = gen.rmat(15, 16, seed=8)
    tri = O.triangles(h.offsets, h.neighbours, threads=4)
    for t in (P.PktTuning(sup_hash_min=4), P.PktTuning(sup_hash_min=64)):
        got, _ = _with_tuning(t, lambda: P.run_triangles(h.offsets, h.neighbours))
        assert np.array_equal(got, tri), t


def test_autotune_stores_a_choice_the_next_launch_uses(tmp_path, monkeypatch):
    g = gen.rmat(15, 16, seed=4)
    best, key = P.autotune(g.offsets, g.neighbours, repeats=1)
    assert key == P.tuning_signature(g.offsets)
    assert P.tuning_lookup(key) == (best, True)
    truss, _ = P.run_pkt(g.offsets, g.neighbours, O32)
    assert P.tuning_last() == (best, key)
    assert np.array_equal(truss, O.fast_truss(g.offsets, g.neighbours)[0])
    # a batch sample: the winner goes to its union's key
    members = [gen.mix_graph(gen.mix_member(i)) for i in range(6)]
    best_b, key_b = P.autotune_batch([(m.offsets, m.neighbours) for m in members], repeats=1)
    assert P.tuning_lookup(key_b) == (best_b, True)
    P.tuning_clear()


def test_hash_tables_with_self_loops_and_compaction():
    """Rows that carry self-loop slots (no edge id: kept out of the tables) and
    a peel that compacts its rows many times: the row and out-list tables give
    the oracle's truss numbers at floors from 8 (most rows hashed) upwards."""
    rng = np.random.default_rng(41)
    base = gen.rmat(14, 16, seed=11)
    n = base.n
    src = np.repeat(np.arange(n, dtype=np.int64), np.diff(base.offsets.astype(np.int64)))
    dst = base.neighbours.astype(np.int64)
    keep = src < dst
    edges = list(zip(src[keep].tolist(), dst[keep].tolist()))
    loops = rng.choice(n, size=n // 8, replace=False)
    edges += [(int(v), int(v)) for v in loops]
    g = gen.from_edges(n, edges)
    assert g.self_loops() > 0
    want = O.pkt(g.offsets, g.neighbours, threads=4)
    for t in (P.PktTuning(hash_min_degree=8, compact_pct=95), P.PktTuning(hash_min_degree=8, sup_hash_min=4),
              P.PktTuning(hash_min_degree=64, hub_min_degree=0, sup_hash_min=16)):
        got, _ = _with_tuning(t, lambda: P.run_pkt(g.offsets, g.neighbours, O32))
        assert np.array_equal(got, want), t


def test_relabel_gives_the_same_truss_in_caller_order():
    """Degree-ordered relabelling rebuilds the CSR on new vertex ids and maps
    every result back to the caller's slots: truss numbers (and the triangle
    count) equal the oracle's on graphs with self-loops, isolated vertices,
    skewed and flat degree distributions."""
    rng = np.random.default_rng(43)
    graphs = [gen.rmat(14, 16, seed=12), gen.erdos_renyi(3000, 20000, 7),
              gen.from_edges(6, [(0, 1), (1, 2), (0, 2), (2, 2), (4, 4)]),
              gen.from_edges(9, [(0, 1), (0, 2), (0, 3), (1, 2), (1, 3), (2, 3), (5, 6)])]
    base = gen.rmat(12, 16, seed=13)
    n = base.n
    src = np.repeat(np.arange(n, dtype=np.int64), np.diff(base.offsets.astype(np.int64)))
    dst = base.neighbours.astype(np.int64)
    keep = src < dst
    edges = list(zip(src[keep].tolist(), dst[keep].tolist()))
    edges += [(int(v), int(v)) for v in rng.choice(n, size=n // 10, replace=False)]
    graphs.append(gen.from_edges(n, edges))
    for g in graphs:
        want = O.pkt(g.offsets, g.neighbours, threads=4)
        got, st = _with_tuning(P.PktTuning(relabel=1), lambda: P.run_pkt(g.offsets, g.neighbours, O32))
        assert np.array_equal(got, want)
        plain, st0 = P.run_pkt(g.offsets, g.neighbours, O32)
        assert st.triangles == st0.triangles and st.k_max == st0.k_max
    # a batched union: every member is relabelled within its own id range
    pairs = [(g.offsets, g.neighbours) for g in graphs]
    want = [O.pkt(g.offsets, g.neighbours, threads=4) for g in graphs]
    res = _with_tuning(P.PktTuning(relabel=1), lambda: P.run_batch(pairs, O32))
    for w, (truss, st, status) in zip(want, res):
        assert status == 0 and np.array_equal(truss, w)
