"""GPU parity on multigraphs (parallel edges, the reference's OneOrMany paths:
impl_csc.rs:154-215, triangles.rs:172-224, pkt.rs:373-395).

The engine deduplicates the rows, runs the weighted support and peel and maps
every caller slot back to its pair; the oracle restates the reference's
copy-by-copy code.  Bit-exact against the oracle's PKT restatement (small
graphs) and its independent weighted peel (larger ones), in every entry point
that takes host graphs, plus the device entry point and a batch that mixes
simple graphs and multigraphs."""
import numpy as np
import pytest

from conftest import random_multigraph
from oracle import oracle as O
from sparkx_b200 import gen
from sparkx_b200.pkt import LOOP_HOST, PktError, PktOptions, run_batch, run_clustering, run_pkt, run_triangles
import sparkx_b200.pkt as P

pytestmark = pytest.mark.gpu
O32 = PktOptions(out_bits=32, timeout_ms=120_000)


@pytest.fixture(scope="module", autouse=True)
def _engine():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    from sparkx_b200 import build
    build.build_engine()
    yield


def test_multigraph_known_answers():
    # doubled edge on a triangle: all 3; every pair doubled: each copy in 4 triangles -> 6
    g = gen.from_multi_edges(3, [(0, 1), (0, 1), (1, 2), (0, 2)])
    t, st = run_pkt(g.offsets, g.neighbours, O32)
    assert (t == 3).all() and st.triangles == 2 and st.m == 3
    g = gen.from_multi_edges(3, [(0, 1), (1, 2), (0, 2)] * 2)
    t, st = run_pkt(g.offsets, g.neighbours.astype(np.uint64))  # u8 output, the reference layout
    assert t.dtype == np.uint8 and (t == 6).all() and st.triangles == 8
    # parallel self-loops keep truss 2
    g = gen.from_multi_edges(4, [(0, 1), (1, 2), (0, 2), (1, 1), (1, 1), (2, 3), (2, 3)])
    t, st = run_pkt(g.offsets, g.neighbours, O32)
    assert np.array_equal(t, O.brute_force_truss(g.offsets, g.neighbours))
    assert st.self_loops == 2


def test_random_multigraphs_match_oracle_both_loops():
    rng = np.random.default_rng(41)
    host = PktOptions(out_bits=32, loop=LOOP_HOST, timeout_ms=60_000)
    for i in range(80):
        g = random_multigraph(rng, n_max=50)
        ref = O.pkt(g.offsets, g.neighbours)
        t, _ = run_pkt(g.offsets, g.neighbours, O32)
        assert np.array_equal(t, ref), i
        t2, _ = run_pkt(g.offsets, g.neighbours, host)
        assert np.array_equal(t2, ref), i


def test_multigraph_supports_and_u8_mode():
    rng = np.random.default_rng(42)
    graphs = [random_multigraph(rng) for _ in range(20)]
    graphs.append(gen.with_parallel_edges(gen.rmat(12, 16, seed=3), 0.3, max_extra=3, seed=3))
    for g in graphs:
        sup, st = run_triangles(g.offsets, g.neighbours.astype(np.uint64))
        ref = O.triangles(g.offsets, g.neighbours)
        assert np.array_equal(sup, ref)
        assert st.triangles * 6 == int(ref.astype(np.int64).sum())
        sup8, _ = run_triangles(g.offsets, g.neighbours.astype(np.uint64), PktOptions(support_mode=P.SUPPORT_U8))
        assert np.array_equal(sup8, O.triangles(g.offsets, g.neighbours, mode=O.MODE_U8))
        try:
            ref8 = O.pkt(g.offsets, g.neighbours, mode=O.MODE_U8, threads=4)
        except O.OracleError:
            continue
        t8, _ = run_pkt(g.offsets, g.neighbours, PktOptions(out_bits=32, support_mode=P.SUPPORT_U8))
        assert np.array_equal(t8, ref8)


def test_multigraph_clustering_counts_distinct_neighbours():
    rng = np.random.default_rng(43)
    for _ in range(15):
        g = random_multigraph(rng)
        local, trans, avg, _ = run_clustering(g.offsets, g.neighbours)
        want_local, want_trans, want_avg = O.clustering(g.offsets, g.neighbours)
        assert np.array_equal(local, want_local)
        if np.isnan(want_trans):
            assert np.isnan(trans)
        else:
            assert trans == pytest.approx(want_trans, rel=1e-12)
        assert avg == pytest.approx(want_avg, rel=1e-12)


def test_larger_multigraphs_match_the_weighted_peel():
    # R-MAT and de Bruijn bases with parallel copies on a share of their edges;
    # large enough for hub maps, compaction and many sub-levels
    cases = [gen.with_parallel_edges(gen.rmat(15, 16, seed=2), 0.2, max_extra=3, seed=7),
             gen.with_parallel_edges(gen.debruijn(400_000, 21, 100, 2_000, 0.05, 3), 0.5, max_extra=2, seed=8)]
    for g in cases:
        want, tri, _ = O.fast_truss(g.offsets, g.neighbours)
        t, st = run_pkt(g.offsets, g.neighbours.astype(np.uint64), O32)
        assert np.array_equal(t, want)
        assert st.triangles == tri
    # the PKT restatement itself on the smaller one (minutes on the CPU at the larger)
    small = gen.with_parallel_edges(gen.rmat(13, 16, seed=5), 0.3, max_extra=3, seed=9)
    t, _ = run_pkt(small.offsets, small.neighbours, O32)
    assert np.array_equal(t, O.pkt(small.offsets, small.neighbours, threads=8))


def test_multigraph_device_entry_and_batch():
    import torch
    rng = np.random.default_rng(44)
    g = gen.with_parallel_edges(gen.rmat(11, 16, seed=4), 0.4, max_extra=2, seed=4)
    want = O.pkt(g.offsets, g.neighbours, threads=4)
    d_off = torch.from_numpy(g.offsets.view(np.int64)).cuda()
    d_nbr = torch.from_numpy(g.neighbours.view(np.int32)).cuda()
    d_out = torch.empty(g.width, dtype=torch.int32, device="cuda")
    P.run_pkt_device(d_off.data_ptr(), g.n + 1, d_nbr.data_ptr(), g.width, d_out.data_ptr(), O32,
                     torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert np.array_equal(d_out.cpu().numpy().view(np.uint32), want)
    # a union mixing simple graphs and multigraphs: every member as alone
    members = [gen.rmat(10, 8, seed=1), g, random_multigraph(rng), gen.erdos_renyi(3000, 20000, 2),
               random_multigraph(rng)]
    res = run_batch([(m.offsets, m.neighbours) for m in members], O32)
    for m, (t, st, status) in zip(members, res):
        assert status == 0
        assert np.array_equal(t, O.pkt(m.offsets, m.neighbours, threads=4))


def test_multigraph_asymmetric_copies_are_invalid():
    # (0, 1) three times in row 0, twice in row 1
    off = np.array([0, 3, 5, 5], np.uint64)
    nbr = np.array([1, 1, 1, 0, 0], np.uint32)
    with pytest.raises(PktError) as ei:
        run_pkt(off, nbr, O32)
    assert ei.value.status == P.E_INVALID_CSR
    t, _ = run_pkt(gen.from_multi_edges(2, [(0, 1)] * 3).offsets, gen.from_multi_edges(2, [(0, 1)] * 3).neighbours,
                   O32)
    assert (t == 2).all()
