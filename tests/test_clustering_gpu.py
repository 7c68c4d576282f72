"""GPU clustering coefficients and the Burkhardt-API facade against the oracle.

Local coefficients are compared exactly (the same integer counts and the same IEEE divisions on
both sides); the transitivity and the average are sums of doubles whose order differs between
the GPU reduction and the oracle, so they are compared to a relative 1e-12."""
import numpy as np
import pytest

from conftest import kn, random_graph
from oracle import oracle as O
from sparkx_b200 import AlgoBurkhardtEtAl, ClusteringCoefficient, GraphMemoryMap, gen
from sparkx_b200 import pkt as P

pytestmark = pytest.mark.gpu

RTOL = 1e-12


def _check(g, mode=P.SUPPORT_WIDE, oracle_mode=O.MODE_WIDE):
    local, trans, avg, st = P.run_clustering(g.offsets, g.neighbours, P.PktOptions(support_mode=mode))
    want_local, want_trans, want_avg = O.clustering(g.offsets, g.neighbours, mode=oracle_mode)
    assert np.array_equal(local, want_local)
    for got, want in ((trans, want_trans), (avg, want_avg)):
        if np.isnan(want):
            assert np.isnan(got)
        else:
            assert got == pytest.approx(want, rel=RTOL, abs=0)
    return st


def test_clustering_known_answers():
    for n in (3, 4, 6):
        _check(kn(n))
    _check(gen.from_edges(3, [(0, 1), (1, 2)]))
    _check(gen.from_edges(3, [(0, 1), (1, 2), (0, 2), (0, 0)]))


def test_clustering_random_graphs():
    rng = np.random.default_rng(21)
    for _ in range(25):
        _check(random_graph(rng))


def test_clustering_rmat_and_u8_counts():
    g = gen.rmat(12, 16, seed=3)
    st = _check(g)
    assert st.triangles > 0
    # dense graph: slot supports past 255 wrap in u8 mode, as the reference's AtomicU8 counts
    dense = kn(40)
    _check(dense, P.SUPPORT_U8, O.MODE_U8)
    _check(gen.rmat(10, 32, seed=9), P.SUPPORT_U8, O.MODE_U8)


def test_clustering_api():
    g = gen.rmat(11, 8, seed=4)
    cc = ClusteringCoefficient.new(GraphMemoryMap.from_csr(g.as_u64()))
    want_local, want_trans, want_avg = O.clustering(g.offsets, g.neighbours)
    assert cc.get_node_clusteringcoefficient(5) == want_local[5]
    assert cc.get_graph_transitivity() == pytest.approx(want_trans, rel=RTOL)
    assert cc.get_average_clustering_coefficient() == pytest.approx(want_avg, rel=RTOL)


def test_burkhardt_api_and_k_truss_facade(tmp_path, monkeypatch):
    monkeypatch.setattr(P, "CACHE_DIR", str(tmp_path))
    g = gen.rmat(11, 8, seed=6)
    gm = GraphMemoryMap.from_csr(g.as_u64())
    want = O.burkhardt(g.offsets, g.neighbours)
    a = AlgoBurkhardtEtAl.new(gm, P.PktOptions(out_bits=32))
    assert np.array_equal(a.k_trusses(), want)
    assert a.trussness(3) == want[3]
    assert np.array_equal(gm.k_truss_pkt().k_trusses(), gm.k_truss().k_trusses())
    assert np.array_equal(gm.k_truss_bea().k_trusses(), want.astype(np.uint8))
