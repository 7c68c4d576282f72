"""GPU parity: the CUDA engine through its C ABI against the CPU oracle and the
committed golden fixtures.  Bit-exact everywhere (integer work)."""
import hashlib
import json
import os

import numpy as np
import pytest

from conftest import book, expected_truss, kats, kn, random_graph
from oracle import oracle as O
from sparkx_b200 import gen
from sparkx_b200.graph import GraphMemoryMap
from sparkx_b200.pkt import (AlgoPKT, LOOP_HOST, PktError, PktOptions, Triangles, run_pkt, run_pkt_device,
                             run_triangles)
import sparkx_b200.pkt as P

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
FIX = os.path.join(HERE, "golden", "fixtures.json")
O32 = PktOptions(out_bits=32, timeout_ms=120_000)


@pytest.fixture(scope="module", autouse=True)
def _engine():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    from sparkx_b200 import build
    build.build_engine()
    yield


def fixtures():
    with open(FIX) as f:
        return json.load(f)


def csr_sha(g):
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(g.offsets, dtype="<u8").tobytes())
    h.update(np.ascontiguousarray(g.neighbours, dtype="<u4").tobytes())
    return h.hexdigest()


def truss_sha(t):
    return hashlib.sha256(np.ascontiguousarray(t, dtype="<u4").tobytes()).hexdigest()


@pytest.mark.parametrize("name,n,edges,special,default", kats(), ids=[k[0] for k in kats()])
def test_known_answers(name, n, edges, special, default):
    g = gen.from_edges(n, edges)
    exp = expected_truss(g, special, default)
    t, st = run_pkt(g.offsets, g.neighbours, O32)
    assert np.array_equal(t, exp)
    t8, _ = run_pkt(g.offsets, g.neighbours.astype(np.uint64))
    assert t8.dtype == np.uint8 and np.array_equal(t8, exp.astype(np.uint8))


def test_random_graphs_both_loops():
    rng = np.random.default_rng(11)
    host = PktOptions(out_bits=32, loop=LOOP_HOST, timeout_ms=60_000)
    for _ in range(120):
        g = random_graph(rng, n_max=70)
        ref = O.pkt(g.offsets, g.neighbours)
        t, _ = run_pkt(g.offsets, g.neighbours, O32)
        assert np.array_equal(t, ref)
        t2, _ = run_pkt(g.offsets, g.neighbours, host)
        assert np.array_equal(t2, ref)


def test_triangles_per_slot():
    for g in (gen.erdos_renyi(20000, 200000, 5), gen.rmat(14, 16, seed=2), book(300)):
        ref = O.triangles(g.offsets, g.neighbours)
        sup, st = run_triangles(g.offsets, g.neighbours.astype(np.uint64))
        assert np.array_equal(sup, ref)
        assert st.triangles == int(ref.astype(np.int64).sum()) // 6
        sup8, _ = run_triangles(g.offsets, g.neighbours.astype(np.uint64), PktOptions(support_mode=P.SUPPORT_U8))
        assert np.array_equal(sup8, O.triangles(g.offsets, g.neighbours, mode=O.MODE_U8))


def test_invalid_inputs_return_status():
    cases = {
        "id_out_of_range": (np.array([0, 1, 3, 4, 4], np.uint64), np.array([1, 0, 9, 1], np.uint32), P.E_INVALID_CSR),
        "asymmetric": (np.array([0, 1, 3, 4, 4], np.uint64), np.array([1, 0, 2, 3], np.uint32), P.E_INVALID_CSR),
        # a parallel edge (0, 1) listed twice in row 0 but once in row 1
        "multigraph_asymmetric": (np.array([0, 2, 4, 5], np.uint64), np.array([1, 1, 0, 2, 1], np.uint32),
                                  P.E_INVALID_CSR),
        "unsorted": (np.array([0, 2, 4, 6], np.uint64), np.array([2, 1, 0, 2, 0, 1], np.uint32), P.E_INVALID_CSR),
        "offsets_not_zero": (np.array([1, 2, 3], np.uint64), np.array([1, 0], np.uint32), P.E_INVALID_CSR),
        "offsets_decreasing": (np.array([0, 2, 1, 2], np.uint64), np.array([1, 0], np.uint32), P.E_INVALID_CSR),
    }
    for name, (off, nbr, code) in cases.items():
        with pytest.raises(PktError) as ei:
            run_pkt(off, nbr, O32)
        assert ei.value.status == code, name
    # the engine stays usable after every failure
    g = kn(6)
    t, _ = run_pkt(g.offsets, g.neighbours, O32)
    assert (t == 6).all()


def test_u8_output_overflow_and_wide_output():
    g = kn(260)
    with pytest.raises(PktError) as ei:
        run_pkt(g.offsets, g.neighbours)
    assert ei.value.status == P.E_OVERFLOW_U8
    t, st = run_pkt(g.offsets, g.neighbours, O32)
    assert (t == 260).all() and st.k_max == 260
    # the reference's u8 counters: level 255 overflows its u8 level counter
    with pytest.raises(PktError) as ei:
        run_pkt(kn(257).offsets, kn(257).neighbours, PktOptions(out_bits=32, support_mode=P.SUPPORT_U8))
    assert ei.value.status == P.E_OVERFLOW_U8


def test_u8_support_mode_matches_reference_wrap():
    for g in (book(256), book(300), gen.rmat(12, 16, seed=2), gen.rmat(14, 16, seed=2)):
        try:
            ref = O.pkt(g.offsets, g.neighbours, mode=O.MODE_U8, threads=4)
        except O.OracleError:
            continue
        t, _ = run_pkt(g.offsets, g.neighbours, PktOptions(out_bits=32, support_mode=P.SUPPORT_U8))
        assert np.array_equal(t, ref)


def test_device_api_matches_host_api():
    import torch
    g = gen.rmat(16, 16, seed=2)
    host, _ = run_pkt(g.offsets, g.neighbours.astype(np.uint64))
    d_off = torch.from_numpy(g.offsets.view(np.int64)).cuda()
    d_nbr = torch.from_numpy(g.neighbours.view(np.int32)).cuda()
    d_out = torch.empty(g.width, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream()
    st = run_pkt_device(d_off.data_ptr(), g.n + 1, d_nbr.data_ptr(), g.width, d_out.data_ptr(), PktOptions(),
                        stream.cuda_stream)
    torch.cuda.synchronize()
    assert np.array_equal(d_out.cpu().numpy(), host)
    assert st.waves > 0 and st.launches > st.waves  # one wave kernel per wave, plus preparation


def test_algopkt_api(tmp_path, monkeypatch):
    monkeypatch.setattr(P, "CACHE_DIR", str(tmp_path))
    g = gen.rmat(12, 16, seed=3)
    gm = GraphMemoryMap.from_csr(g.as_u64(), thread_count=16)
    algo = AlgoPKT.new(gm)
    ref = O.pkt(g.offsets, g.neighbours)
    assert np.array_equal(algo.k_trusses(), ref.astype(np.uint8))
    assert algo.trussness(7) == ref[7]
    with pytest.raises(AssertionError):
        algo.trussness(g.width)
    again = AlgoPKT.get_or_compute(gm)  # served from the result file
    assert np.array_equal(again.k_trusses(), algo.k_trusses())
    algo.drop_cache()
    tri = Triangles.new(gm)
    assert np.array_equal(tri.all_triangles(), O.triangles(g.offsets, g.neighbours))


def test_timeout_returns_status_and_engine_recovers():
    g = gen.rmat(18, 16, seed=2)
    with pytest.raises(PktError) as ei:
        run_pkt(g.offsets, g.neighbours, PktOptions(out_bits=32, timeout_ms=1))
    assert ei.value.status == P.E_TIMEOUT
    t, _ = run_pkt(g.offsets, g.neighbours, O32)
    fx = fixtures()["rmat18"]
    assert truss_sha(t) == fx["modes"]["0"]["truss_sha256"]


def test_self_loops_and_isolated():
    edges = [(0, 1), (1, 2), (0, 2), (2, 2), (5, 5), (3, 4)]
    g = gen.from_edges(8, edges)
    t, st = run_pkt(g.offsets, g.neighbours, O32)
    assert np.array_equal(t, O.brute_force_truss(g.offsets, g.neighbours))
    assert st.self_loops == 2
    t0, _ = run_pkt(np.zeros(5, np.uint64), np.zeros(0, np.uint32), O32)
    assert t0.size == 0


@pytest.mark.parametrize("name", ["dbg_small", "rmat16", "rmat18", "cfg1_er_100k_1m", "cfg3_debruijn", "cfg2_rmat22",
                                  "cfg5_rmat24_tail"])
def test_golden_workloads(name):
    fx = fixtures()[name]
    p = fx["params"]
    if p["fn"] == "er":
        g = gen.erdos_renyi(p["n"], p["m"], p["seed"])
    elif p["fn"] == "rmat":
        g = gen.rmat(p["scale"], p["ef"], seed=p["seed"])
    else:
        g = gen.debruijn(p["seq_len"], p["k"], p["copies"], p["seg_len"], p["mut_rate"], p["seed"])
    assert csr_sha(g) == fx["csr_sha256"], "generator output changed"
    t, st = run_pkt(g.offsets, g.neighbours, O32)
    want = fx["modes"]["0"]
    assert st.triangles == fx["triangles"]
    hist = {str(i): int(c) for i, c in enumerate(np.bincount(t.astype(np.int64))) if c}
    assert hist == want["hist"]
    assert truss_sha(t) == want["truss_sha256"]
    assert st.k_max == want["k_max"]
    u8 = fx["modes"].get("1")
    if u8 and "truss_sha256" in u8:
        t8, _ = run_pkt(g.offsets, g.neighbours, PktOptions(out_bits=32, support_mode=P.SUPPORT_U8))
        assert truss_sha(t8) == u8["truss_sha256"]


@pytest.mark.parametrize("name", ["arr_rmat10", "arr_dbg_k6", "arr_er"])
def test_golden_arrays(name):
    z = np.load(os.path.join(HERE, "golden", f"{name}.npz"))
    t, _ = run_pkt(z["offsets"], z["neighbours"], O32)
    assert np.array_equal(t, z["truss_mode0"])
    if "truss_mode1" in z:
        t8, _ = run_pkt(z["offsets"], z["neighbours"], PktOptions(out_bits=32, support_mode=P.SUPPORT_U8))
        assert np.array_equal(t8, z["truss_mode1"])


def test_golden_mix_members():
    fx = fixtures()
    names = sorted(k for k in fx if k.startswith("cfg4_mix_"))
    assert len(names) >= 8
    for name in names:
        f = fx[name]
        g = gen.mix_graph(gen.mix_member(f["params"]["index"]))
        assert csr_sha(g) == f["csr_sha256"]
        t, st = run_pkt(g.offsets, g.neighbours, O32)
        assert truss_sha(t) == f["modes"]["0"]["truss_sha256"], name
        assert st.triangles == f["triangles"]


def test_batch_matches_solo_runs_and_oracle():
    from sparkx_b200.pkt import run_batch
    rng = np.random.default_rng(5)
    graphs = [random_graph(rng, n_max=50) for _ in range(60)]
    graphs += [gen.mix_graph(gen.mix_member(i)) for i in range(12) if gen.mix_member(i).n < 30_000]
    graphs += [gen.rmat(13, 16, seed=7), kn(30), gen.from_edges(3, [])]
    res = run_batch([(g.offsets, g.neighbours) for g in graphs], O32)
    for g, (t, st, status) in zip(graphs, res):
        assert status == 0
        ref = O.pkt(g.offsets, g.neighbours, threads=2)
        assert np.array_equal(t, ref)
        solo, sst = run_pkt(g.offsets, g.neighbours, O32)
        assert np.array_equal(t, solo)
        assert st.triangles == sst.triangles and st.k_max == sst.k_max


def test_batch_isolates_bad_members_and_budget():
    from sparkx_b200.pkt import run_batch
    good = gen.rmat(11, 8, seed=1)
    bad_sym = (np.array([0, 1, 3, 4, 4], np.uint64), np.array([1, 0, 2, 3], np.uint32))
    bad_range = (np.array([0, 1, 2], np.uint64), np.array([1, 7], np.uint32))
    multi = (np.array([0, 2, 4, 5], np.uint64), np.array([1, 1, 0, 2, 1], np.uint32))
    res = run_batch([(good.offsets, good.neighbours), bad_sym, bad_range, multi,
                     (good.offsets, good.neighbours.astype(np.uint64))], O32)
    assert [r[2] for r in res] == [0, P.E_INVALID_CSR, P.E_INVALID_CSR, P.E_INVALID_CSR, 0]
    ref = O.pkt(good.offsets, good.neighbours)
    assert np.array_equal(res[0][0], ref) and np.array_equal(res[4][0], ref)
    # a tiny budget forces one graph per union; a graph larger than the budget fails alone
    gs = [gen.rmat(10, 8, seed=s) for s in range(4)]
    res = run_batch([(g.offsets, g.neighbours) for g in gs], O32, hbm_budget_bytes=300 << 20)
    for g, r in zip(gs, res):
        assert r[2] == 0 and np.array_equal(r[0], O.pkt(g.offsets, g.neighbours))
    res = run_batch([(gs[0].offsets, gs[0].neighbours)], O32, hbm_budget_bytes=1 << 20)
    assert res[0][2] == P.E_OOM


@pytest.mark.parametrize("loop", [P.LOOP_GRAPH, LOOP_HOST])
def test_compaction_in_both_loops(loop):
    """Graphs above the compaction threshold rebuild the working rows mid-peel;
    host-launched waves must resume the planned wave unchanged after each rebuild."""
    fx = fixtures()
    for name in ("rmat16", "rmat18"):
        p = fx[name]["params"]
        g = gen.rmat(p["scale"], p["ef"], seed=p["seed"])
        t, st = run_pkt(g.offsets, g.neighbours, PktOptions(out_bits=32, loop=loop, timeout_ms=120_000))
        assert truss_sha(t) == fx[name]["modes"]["0"]["truss_sha256"]
        assert st.compactions >= 1


@pytest.mark.parametrize("kernel", [1, 2])
def test_support_kernel_forms_agree(kernel):
    """Balanced (edge) and vertex (shared-memory hash) support forms give the same
    per-slot support and the same truss numbers."""
    for g in (gen.rmat(14, 16, seed=2), gen.erdos_renyi(20000, 300000, 9), kn(90), book(300),
              gen.debruijn(20000, 7, 20, 500, 0.05, 9)):
        ref = O.triangles(g.offsets, g.neighbours)
        sup, st = run_triangles(g.offsets, g.neighbours.astype(np.uint64), PktOptions(support_kernel=kernel))
        assert np.array_equal(sup, ref)
        t, _ = run_pkt(g.offsets, g.neighbours, PktOptions(out_bits=32, support_kernel=kernel))
        assert np.array_equal(t, O.pkt(g.offsets, g.neighbours, threads=4))


def test_sharded_batch_single_rank_uses_the_engine():
    """shard.run_sharded_batch without a process group: one rank, the CUDA batch call, the
    same results as the oracle (the gloo tests cover placement and the gather on CPU)."""
    from sparkx_b200 import shard
    gs = [gen.rmat(10, 8, seed=s) for s in range(3)] + [gen.erdos_renyi(5000, 30000, 9)]
    out = shard.run_sharded_batch([shard.work_estimate(g.n, g.width) for g in gs],
                                  lambda i: (gs[i].offsets, gs[i].neighbours), opts=O32)
    assert out.parts == [[0, 1, 2, 3]]
    for g, (t, st, status) in zip(gs, out.results):
        assert status == 0 and np.array_equal(t, O.pkt(g.offsets, g.neighbours))


def test_gpu_truss_passes_the_verifier_on_rmat18():
    """The corrected verifier (the definition, no peel involved) accepts the GPU's R-MAT-18
    decomposition and rejects it with one slot changed."""
    g = gen.rmat(18, 16, seed=2)
    t, _ = run_pkt(g.offsets, g.neighbours, O32)
    assert O.verify(g.offsets, g.neighbours, t, threads=os.cpu_count() or 1) == -1
    bad = t.copy()
    s = int(np.argmax(t))
    bad[s] += 1
    assert O.verify(g.offsets, g.neighbours, bad, threads=os.cpu_count() or 1) >= 0
