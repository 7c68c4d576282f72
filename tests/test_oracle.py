"""The CPU oracle (restatements of the reference's PKT path) against hand-derived
known answers, a brute-force definition and each other."""
import numpy as np
import pytest

from conftest import random_multigraph, book, expected_truss, kats, kn, random_graph
from oracle import oracle as O
from sparkx_b200 import gen


def all_oracles(g, mode=O.MODE_WIDE):
    off, nbr = g.offsets, g.neighbours
    return {
        "pkt_t1": O.pkt(off, nbr, mode=mode, threads=1),
        "pkt_t3": O.pkt(off, nbr, mode=mode, threads=3),
        "pkt_hash": O.pkt(off, nbr, mode=mode, threads=2, hash_map=True),
        "burkhardt": O.burkhardt(off, nbr, mode=mode),
        "fast": O.fast_truss(off, nbr, mode=mode, threads=2)[0],
    }


@pytest.mark.parametrize("name,n,edges,special,default", kats(), ids=[k[0] for k in kats()])
def test_known_answers(name, n, edges, special, default):
    g = gen.from_edges(n, edges)
    exp = expected_truss(g, special, default)
    for impl, t in all_oracles(g).items():
        assert np.array_equal(t, exp), (name, impl, t, exp)
    assert np.array_equal(O.brute_force_truss(g.offsets, g.neighbours), exp)
    assert O.verify(g.offsets, g.neighbours, exp) == -1


def test_random_graphs_agree_with_definition():
    rng = np.random.default_rng(7)
    for _ in range(120):
        g = random_graph(rng)
        bf = O.brute_force_truss(g.offsets, g.neighbours)
        for impl, t in all_oracles(g).items():
            assert np.array_equal(t, bf), impl
        assert O.verify(g.offsets, g.neighbours, bf) == -1


def test_triangles_per_slot_match_definition():
    rng = np.random.default_rng(3)
    for _ in range(40):
        g = random_graph(rng)
        sup = O.triangles(g.offsets, g.neighbours)
        off = g.offsets.astype(np.int64)
        nb = [set(int(x) for x in g.neighbours[off[u]:off[u + 1]]) - {u} for u in range(g.n)]
        for u in range(g.n):
            for s in range(off[u], off[u + 1]):
                v = int(g.neighbours[s])
                want = 0 if v == u else len(nb[u] & nb[v])
                assert sup[s] == want


def test_edge_index_reciprocals():
    g = gen.rmat(10, 8, seed=5)
    eo, er = O.edge_index(g.offsets, g.neighbours, threads=3)
    off = g.offsets.astype(np.int64)
    for u in range(g.n):
        row = g.neighbours[off[u]:off[u + 1]]
        assert eo[u] == off[u] + int(np.searchsorted(row, u, side="right"))
    src = np.repeat(np.arange(g.n), np.diff(off))
    assert np.array_equal(er[er], np.arange(g.width))
    assert np.array_equal(g.neighbours[er], src.astype(np.uint32))


def test_verify_rejects_wrong_assignments():
    g = kn(5)
    good = np.full(g.width, 5, dtype=np.uint32)
    assert O.verify(g.offsets, g.neighbours, good) == -1
    bad = good.copy()
    bad[3] = 4  # asymmetric
    assert O.verify(g.offsets, g.neighbours, bad) >= 0
    assert O.verify(g.offsets, g.neighbours, np.full(g.width, 6, dtype=np.uint32)) >= 0


def test_invalid_inputs_rejected():
    off = np.array([0, 1, 3, 4, 4], dtype=np.uint64)
    with pytest.raises(O.OracleError):
        O.edge_index(off, np.array([1, 0, 2, 3], dtype=np.uint32))  # asymmetric
    with pytest.raises(O.OracleError):
        O.edge_index(np.array([0, 2, 3, 4], dtype=np.uint64), np.array([1, 1, 0, 0], dtype=np.uint32))
    with pytest.raises(O.OracleError):
        O.edge_index(np.array([0, 2, 4, 6], dtype=np.uint64), np.array([2, 1, 0, 2, 0, 1], dtype=np.uint32))


def test_u8_mode_wraps_support_like_the_reference():
    # spine support 256 wraps to 0: the reference marks it processed at level 0
    # (truss 2) and never charges its triangles, so the pages keep truss 3
    g = book(256)
    sup = O.triangles(g.offsets, g.neighbours, mode=O.MODE_U8)
    wide = O.triangles(g.offsets, g.neighbours)
    assert wide.max() == 256 and sup.max() == 1
    res = all_oracles(g, mode=O.MODE_U8)
    spine = [s for s in range(g.width) if g.neighbours[s] in (0, 1) and s < g.offsets[2]]
    for impl, t in res.items():
        assert all(t[s] == 2 for s in spine if (s < g.offsets[1] and g.neighbours[s] == 1)
                   or (s >= g.offsets[1] and g.neighbours[s] == 0)), impl
    base = res["pkt_t1"]
    for impl, t in res.items():
        assert np.array_equal(t, base), impl
    for impl, t in all_oracles(g).items():
        assert (t == 3).all(), impl
    # below 256 the two widths agree
    g2 = book(200)
    assert np.array_equal(O.pkt(g2.offsets, g2.neighbours, mode=O.MODE_U8),
                          O.pkt(g2.offsets, g2.neighbours))


def test_u8_level_overflow_is_an_error():
    # K_257: support 255 everywhere -> level 255 -> the reference's u8 level
    # counter overflows (pkt.rs:508-516)
    g = kn(257)
    with pytest.raises(O.OracleError):
        O.pkt(g.offsets, g.neighbours, mode=O.MODE_U8, threads=4)
    t = O.pkt(g.offsets, g.neighbours, threads=4)
    assert (t == 257).all()


def test_medium_graphs_three_way():
    for g in (gen.erdos_renyi(3000, 30000, 11), gen.rmat(12, 16, seed=4), gen.debruijn(20000, 7, 20, 500, 0.05, 9)):
        base = O.pkt(g.offsets, g.neighbours, threads=4)
        assert np.array_equal(base, O.burkhardt(g.offsets, g.neighbours))
        assert np.array_equal(base, O.fast_truss(g.offsets, g.neighbours, threads=4)[0])
        assert O.verify(g.offsets, g.neighbours, base, threads=4) == -1


@pytest.mark.parametrize("name", ["arr_rmat10", "arr_dbg_k6", "arr_er"])
def test_oracle_against_committed_vectors(name):
    import os
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", f"{name}.npz"))
    off, nbr = z["offsets"], z["neighbours"]
    assert np.array_equal(O.pkt(off, nbr, threads=2), z["truss_mode0"])
    assert np.array_equal(O.burkhardt(off, nbr), z["truss_mode0"])
    assert np.array_equal(z["brute_force"], z["truss_mode0"])
    if "truss_mode1" in z:
        assert np.array_equal(O.pkt(off, nbr, mode=O.MODE_U8), z["truss_mode1"])


def test_generators_reproduce_fixture_graphs():
    import hashlib
    import json
    import os
    fx = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "fixtures.json")))
    for name in ("rmat16", "cfg1_er_100k_1m", "dbg_small"):
        p = fx[name]["params"]
        if p["fn"] == "er":
            g = gen.erdos_renyi(p["n"], p["m"], p["seed"])
        elif p["fn"] == "rmat":
            g = gen.rmat(p["scale"], p["ef"], seed=p["seed"])
        else:
            g = gen.debruijn(p["seq_len"], p["k"], p["copies"], p["seg_len"], p["mut_rate"], p["seed"])
        h = hashlib.sha256()
        h.update(np.ascontiguousarray(g.offsets, dtype="<u8").tobytes())
        h.update(np.ascontiguousarray(g.neighbours, dtype="<u4").tobytes())
        assert h.hexdigest() == fx[name]["csr_sha256"], name


def _clustering_definition(g):
    """Local coefficients from the definition: edges among u's neighbours over C(d, 2), d the
    number of distinct neighbours (a self-loop counts as one, as the reference's row HashSet
    does), and the reference's transitivity: triangles / sum of C(d, 2)."""
    off = g.offsets.astype(np.int64)
    nbrs = [set(int(x) for x in g.neighbours[off[u]:off[u + 1]]) for u in range(g.n)]
    local, possible, tri_total = [], 0.0, 0
    for u in range(g.n):
        d = len(nbrs[u])
        others = nbrs[u] - {u}
        links = sum(1 for a in others for b in others if a < b and b in nbrs[a])
        p = d * (d - 1) / 2.0 if d > 1 else 0.0
        possible += p
        tri_total += links
        local.append(links / p if p > 0 else 0.0)
    return np.array(local), (tri_total / 3) / possible if possible else float("nan")


def test_clustering_known_answers():
    # K3 and K4: every neighbour pair linked; the reference's transitivity is T / sum C(d, 2)
    for n in (3, 4):
        local, trans, avg = O.clustering(kn(n).offsets, kn(n).neighbours)
        assert np.array_equal(local, np.ones(n)) and avg == 1.0
        assert trans == pytest.approx(1.0 / 3.0, rel=1e-15)
    path = gen.from_edges(3, [(0, 1), (1, 2)])
    local, trans, avg = O.clustering(path.offsets, path.neighbours)
    assert np.array_equal(local, np.zeros(3)) and trans == 0.0 and avg == 0.0
    # a self-loop widens u's neighbourhood (d counts u) without adding triangles
    g = gen.from_edges(3, [(0, 1), (1, 2), (0, 2), (0, 0)])
    local, _, _ = O.clustering(g.offsets, g.neighbours)
    assert local[0] == pytest.approx(1.0 / 3.0, rel=1e-15) and local[1] == 1.0


def test_clustering_matches_definition():
    rng = np.random.default_rng(11)
    for _ in range(60):
        g = random_graph(rng)
        local, trans, avg = O.clustering(g.offsets, g.neighbours)
        want_local, want_trans = _clustering_definition(g)
        assert np.allclose(local, want_local, rtol=1e-15, atol=0)
        if np.isnan(want_trans):
            assert np.isnan(trans)
        else:
            assert trans == pytest.approx(want_trans, rel=1e-14)
        assert avg == pytest.approx(want_local.sum() / g.n, rel=1e-14)


def test_clustering_faithful_mode_reproduces_the_reference_zeroing():
    """Defect D4: clustering_coefficient.rs:130-135 zeroes the supports before reading them,
    so the reference's coefficients are all 0 (transitivity NaN without any possible pair).
    The faithful mode pins that output; the default mode (what the GPU engine returns) keeps
    the intended values."""
    g = kn(5)
    local, trans, avg = O.clustering(g.offsets, g.neighbours, faithful=True)
    assert np.array_equal(local, np.zeros(5)) and trans == 0.0 and avg == 0.0
    local, trans, avg = O.clustering(g.offsets, g.neighbours)
    assert np.array_equal(local, np.ones(5)) and avg == 1.0
    path = gen.from_edges(2, [(0, 1)])
    _, trans, _ = O.clustering(path.offsets, path.neighbours, faithful=True)
    assert np.isnan(trans)


def _core_definition(g):
    """Textbook core numbers: repeatedly remove a vertex of minimum remaining degree; its core
    is the largest minimum seen so far (graphs without self-loops)."""
    off = g.offsets.astype(np.int64)
    adj = [set(int(x) for x in g.neighbours[off[u]:off[u + 1]]) for u in range(g.n)]
    deg = {u: len(adj[u]) for u in range(g.n)}
    core, level = {}, 0
    while deg:
        u = min(deg, key=lambda x: (deg[x], x))
        level = max(level, deg[u])
        core[u] = level
        for v in adj[u]:
            if v in deg:
                deg[v] -= 1
        del deg[u]
    return np.array([core[u] for u in range(g.n)])


def test_kcore_known_answers():
    assert list(O.kcore(*(lambda g: (g.offsets, g.neighbours))(gen.from_edges(3, [(0, 1), (1, 2)])))) == [1, 1, 1]
    assert list(O.kcore(kn(5).offsets, kn(5).neighbours)) == [4] * 5
    g = gen.from_edges(5, [(0, 1), (0, 2), (0, 3), (1, 2)])  # triangle, a pendant, an isolated vertex
    assert list(O.kcore(g.offsets, g.neighbours)) == [2, 2, 2, 1, 0]
    # u8 degrees: K300's degree 299 wraps to 43, so every vertex is peeled at level 43
    assert set(O.kcore(kn(300).offsets, kn(300).neighbours, mode=O.MODE_U8)) == {43}


def test_kcore_matches_definition():
    rng = np.random.default_rng(17)
    for _ in range(60):
        g = random_graph(rng, self_loop_p=0.0)
        assert np.array_equal(O.kcore(g.offsets, g.neighbours), _core_definition(g))


# ---- multigraphs (the reference's OneOrMany paths) -------------------------------------

def test_multigraph_known_answers():
    # a triangle whose edge (0, 1) is doubled: two triangles of copies; a copy of (0, 1) lies in
    # one, (1, 2) and (0, 2) in two each -> every edge is in the 3-truss, none in the 4-truss
    g = gen.from_multi_edges(3, [(0, 1), (0, 1), (1, 2), (0, 2)])
    assert np.array_equal(O.triangles(g.offsets, g.neighbours), [1, 1, 2, 1, 1, 2, 2, 2])
    for f in (O.pkt, O.burkhardt, lambda o, n: O.fast_truss(o, n)[0], O.brute_force_truss):
        assert np.array_equal(f(g.offsets, g.neighbours), np.full(8, 3))
    # every pair doubled: each copy lies in 2 * 2 = 4 triangles -> the 6-truss
    g = gen.from_multi_edges(3, [(0, 1), (1, 2), (0, 2)] * 2)
    for f in (O.pkt, O.burkhardt, lambda o, n: O.fast_truss(o, n)[0], O.brute_force_truss):
        assert np.array_equal(f(g.offsets, g.neighbours), np.full(12, 6))
    # parallel self-loops: truss 2 each, their own reciprocals
    g = gen.from_multi_edges(3, [(0, 1), (1, 2), (0, 2), (1, 1), (1, 1)])
    _, er = O.edge_index(g.offsets, g.neighbours)
    loops = [s for s in range(g.width) if g.neighbours[s] == 1 and 2 <= s < 6]
    assert all(er[s] == s for s in loops) and len(loops) == 2
    t = O.pkt(g.offsets, g.neighbours)
    assert all(t[s] == 2 for s in loops)
    assert O.verify(g.offsets, g.neighbours, t) == -1


def test_multigraph_edge_index_pairs_copies():
    rng = np.random.default_rng(31)
    for _ in range(40):
        g = random_multigraph(rng)
        eo, er = O.edge_index(g.offsets, g.neighbours, threads=3)
        off = g.offsets.astype(np.int64)
        row = np.repeat(np.arange(g.n), np.diff(off))
        er = er.astype(np.int64)
        assert np.array_equal(er[er], np.arange(g.width))            # an involution
        assert np.array_equal(row[er], g.neighbours.astype(np.int64))  # joins a copy of the same pair
        assert np.array_equal(g.neighbours[er].astype(np.int64), row)


def test_multigraph_restatements_agree_with_definition():
    rng = np.random.default_rng(32)
    for i in range(60):
        g = random_multigraph(rng)
        want_sup = O.support_definition(g.offsets, g.neighbours)
        assert np.array_equal(O.triangles(g.offsets, g.neighbours, hash_map=bool(i & 1)), want_sup)
        want = O.brute_force_truss(g.offsets, g.neighbours)
        assert np.array_equal(O.pkt(g.offsets, g.neighbours, threads=1 + i % 4, hash_map=bool(i & 1)), want)
        assert np.array_equal(O.burkhardt(g.offsets, g.neighbours, hash_map=bool(i & 2)), want)
        t, tri, _ = O.fast_truss(g.offsets, g.neighbours, threads=2)
        assert np.array_equal(t, want)
        assert tri * 6 == int(want_sup.sum())
        assert O.verify(g.offsets, g.neighbours, want) == -1


def test_multigraph_verifier_rejects_wrong_assignments():
    g = gen.from_multi_edges(4, [(0, 1), (0, 1), (1, 2), (0, 2), (2, 3), (1, 3)])
    t = O.brute_force_truss(g.offsets, g.neighbours)
    assert O.verify(g.offsets, g.neighbours, t) == -1
    for s in range(g.width):
        if g.neighbours[s] == s:
            continue
        bad = t.copy()
        bad[s] += 1
        assert O.verify(g.offsets, g.neighbours, bad) >= 0


def test_multigraph_larger_graphs_pkt_equals_fast_peel():
    for seed, frac in ((1, 0.2), (2, 0.5)):
        g = gen.with_parallel_edges(gen.rmat(11, 8, seed=seed), frac, max_extra=3, seed=seed)
        want = O.fast_truss(g.offsets, g.neighbours)[0]
        assert np.array_equal(O.pkt(g.offsets, g.neighbours, threads=4), want)
        assert O.verify(g.offsets, g.neighbours, want, threads=4) == -1


def test_every_pinned_truss_is_certified_by_the_verifier():
    """Each fixture's mode-0 truss carries two independent oracles or a verifier pass; the two
    largest (R-MAT-22 and the R-MAT-24 tail, pinned by the independent peel alone) carry a pass
    of the corrected verifier (symmetry, support >= k - 2 inside the k-truss, local
    maximality), recorded by tests/golden/make_golden.py."""
    import json
    import os
    with open(os.path.join(os.path.dirname(__file__), "golden", "fixtures.json")) as f:
        fx = json.load(f)
    for name, entry in fx.items():
        m0 = entry["modes"]["0"]
        assert m0.get("verified") is True or len(m0["oracles"]) >= 2, name
    for name in ("cfg2_rmat22", "cfg5_rmat24_tail", "rmat20"):
        assert fx[name]["modes"]["0"].get("verified") is True, name
    assert set(fx["rmat20"]["modes"]["0"]["oracles"]) == {"pkt", "fast"}
