"""Workload generators: CSR invariants, determinism, independence from thread count."""
import hashlib

import numpy as np

from sparkx_b200 import gen
from sparkx_b200.graph import GraphMemoryMap


def sha(g):
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(g.offsets, dtype="<u8").tobytes())
    h.update(np.ascontiguousarray(g.neighbours, dtype="<u4").tobytes())
    return h.hexdigest()


def check_simple_symmetric(g, allow_self=False):
    off = g.offsets.astype(np.int64)
    assert off[0] == 0 and off[-1] == g.width and np.all(np.diff(off) >= 0)
    nbr = g.neighbours.astype(np.int64)
    assert nbr.size == 0 or nbr.max() < g.n
    src = np.repeat(np.arange(g.n), np.diff(off))
    inrow = np.diff(nbr)[np.diff(src) == 0]
    assert np.all(inrow > 0), "rows strictly ascending"
    if not allow_self:
        assert not np.any(src == nbr)
    fwd = set(zip(src.tolist(), nbr.tolist()))
    assert all((v, u) in fwd for (u, v) in fwd)


def test_er_exact_edge_count_and_invariants():
    g = gen.erdos_renyi(2000, 15000, 1)
    assert g.n == 2000 and g.width == 30000
    check_simple_symmetric(g)


def test_rmat_invariants():
    g = gen.rmat(12, 16, seed=2)
    assert g.n == 4096 and 0 < g.width <= 2 * 16 * 4096
    check_simple_symmetric(g)
    deg = np.diff(g.offsets.astype(np.int64))
    assert deg.max() > 20 * deg.mean()  # skewed


def test_debruijn_degree_bound():
    g = gen.debruijn(50_000, 21, 20, 1000, 0.05, 3)
    check_simple_symmetric(g)
    assert np.diff(g.offsets.astype(np.int64)).max() <= 8
    assert g.n >= 49_980


def test_deterministic_and_thread_independent():
    old = gen.set_threads(1)
    a = [sha(gen.rmat(11, 8, seed=9)), sha(gen.erdos_renyi(1000, 5000, 4)), sha(gen.debruijn(20_000, 11, 5, 500, .05, 1))]
    gen.set_threads(4)
    b = [sha(gen.rmat(11, 8, seed=9)), sha(gen.erdos_renyi(1000, 5000, 4)), sha(gen.debruijn(20_000, 11, 5, 500, .05, 1))]
    gen.set_threads(old)
    assert a == b
    assert sha(gen.rmat(11, 8, seed=10)) != a[0]


def test_mix_members():
    ns, ds, kinds = [], [], set()
    for i in range(200):
        m = gen.mix_member(i)
        assert 1000 <= m.n <= 1_000_000 and 4 <= m.avg_degree <= 64
        assert m.seed == 1000 + i
        ns.append(m.n)
        ds.append(m.avg_degree)
        kinds.add(m.kind)
    assert kinds == {"er", "rmat"}
    assert np.median(np.log10(ns)) > 3.8 and np.median(np.log10(ns)) < 5.2  # log-uniform
    assert gen.mix_member(5) == gen.mix_member(5)
    small = next(gen.mix_member(i) for i in range(100) if gen.mix_member(i).n < 3000)
    g = gen.mix_graph(small)
    assert g.n == small.n
    check_simple_symmetric(g)


def test_graph_memory_map_cache_round_trip(tmp_path):
    g = gen.rmat(9, 8, seed=1)
    gm = GraphMemoryMap.from_csr(g, thread_count=16)
    gm.write_cache(str(tmp_path / "off.bin"), str(tmp_path / "nbr.bin"))
    g2 = GraphMemoryMap.open(str(tmp_path / "off.bin"), str(tmp_path / "nbr.bin"))
    assert g2.size() == g.n and g2.width() == g.width
    assert g2.neighbours().dtype == np.uint64
    assert np.array_equal(g2.neighbours(), g.neighbours.astype(np.uint64))
    assert g2.node_degree(3) == int(g.offsets[4] - g.offsets[3])
    assert gm.thread_num() == 16
