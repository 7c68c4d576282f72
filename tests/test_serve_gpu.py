"""Continuous-batching service: every request's result equals its solo
decomposition (and the oracle), whatever else is in flight."""
import time

import numpy as np
import pytest

from conftest import kn, random_graph
from oracle import oracle as O
from sparkx_b200 import gen
import sparkx_b200.pkt as P
from sparkx_b200.serve import PktServer

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _engine():
    import torch
    assert torch.cuda.is_available(), "needs a CUDA device"
    from sparkx_b200 import build
    build.build_engine()


def workload():
    rng = np.random.default_rng(23)
    gs = [random_graph(rng, n_max=60) for _ in range(25)]
    gs += [gen.mix_graph(gen.mix_member(i)) for i in range(20) if gen.mix_member(i).n < 40_000]
    gs += [gen.rmat(13, 16, seed=3), gen.rmat(14, 16, seed=4), kn(40), gen.from_edges(5, [])]
    return gs


def test_alone_equals_in_mix():
    gs = workload()
    solo = [P.run_pkt(g.offsets, g.neighbours, P.PktOptions(out_bits=32))[0] for g in gs]
    with PktServer(8 << 30) as srv:
        tickets = [srv.submit(g.offsets, g.neighbours) for g in gs]
        res = [srv.wait(t, timeout_ms=120_000) for t in tickets]
    for g, r, s in zip(gs, res, solo):
        assert r.status == P.OK
        assert np.array_equal(r.truss, s)
        assert r.latency_ms > 0
    for g, r in list(zip(gs, res))[:12]:
        assert np.array_equal(r.truss, O.pkt(g.offsets, g.neighbours, threads=2))


def test_staggered_arrivals_overlap():
    gs = workload()
    with PktServer(8 << 30) as srv:
        first = [srv.submit(g.offsets, g.neighbours) for g in gs[:10]]
        time.sleep(0.01)
        second = [srv.submit(g.offsets, g.neighbours) for g in gs[10:]]
        out = {t: srv.wait(t, timeout_ms=120_000) for t in first + second}
    for g, t in zip(gs, first + second):
        assert out[t].status == P.OK
        assert np.array_equal(out[t].truss, P.run_pkt(g.offsets, g.neighbours, P.PktOptions(out_bits=32))[0])


def test_errors_cancel_and_budget():
    good = gen.rmat(12, 16, seed=5)
    bad = (np.array([0, 1, 3, 4, 4], np.uint64), np.array([1, 0, 2, 3], np.uint32))
    with PktServer(1 << 30) as srv:
        tb = srv.submit(*bad)
        tg = [srv.submit(good.offsets, good.neighbours) for _ in range(30)]
        cancelled = srv.cancel(tg[-1])
        rb = srv.wait(tb, timeout_ms=60_000)
        assert rb.status == P.E_INVALID_CSR
        for t in tg[:-1]:
            r = srv.wait(t, timeout_ms=60_000)
            assert r.status == P.OK and np.array_equal(r.truss, O.pkt(good.offsets, good.neighbours))
        last = srv.wait(tg[-1], timeout_ms=60_000)
        assert last.status == (P.E_CANCELLED if cancelled else P.OK)
        big = gen.rmat(20, 16, seed=1)  # needs more than a quarter of a 1 GiB budget
        r = srv.wait(srv.submit(big.offsets, big.neighbours), timeout_ms=60_000)
        assert r.status == P.E_OOM


def _one_lane_server(budget):
    import os
    old = os.environ.get("SPARX_SERVE_LANES")
    os.environ["SPARX_SERVE_LANES"] = "1"
    try:
        return PktServer(budget)
    finally:
        if old is None:
            del os.environ["SPARX_SERVE_LANES"]
        else:
            os.environ["SPARX_SERVE_LANES"] = old


def test_requests_join_a_running_union_mid_peel():
    """One lane: a long request starts a union; requests submitted while its peel runs join
    it at a wave boundary (the server counts them), finish before it, and every result
    equals the solo decomposition and the oracle."""
    big = gen.rmat(20, 16, seed=7)  # ~0.1 s of peel: the others arrive while it runs
    rng = np.random.default_rng(29)
    small = [random_graph(rng, n_max=60) for _ in range(10)]
    small += [gen.mix_graph(gen.mix_member(i)) for i in range(8) if gen.mix_member(i).n < 20_000]
    small.append(gen.with_parallel_edges(gen.rmat(9, 8, seed=2), 0.3, seed=2))  # a multigraph: not joined
    with _one_lane_server(16 << 30) as srv:
        tb = srv.submit(big.offsets, big.neighbours)
        time.sleep(0.02)  # the big request's union is running
        ts = [srv.submit(g.offsets, g.neighbours) for g in small]
        rs = [srv.wait(t, timeout_ms=120_000) for t in ts]
        rb = srv.wait(tb, timeout_ms=120_000)
        info = srv.info()
    assert rb.status == P.OK
    assert np.array_equal(rb.truss, P.run_pkt(big.offsets, big.neighbours, P.PktOptions(out_bits=32))[0])
    for g, r in zip(small, rs):
        assert r.status == P.OK
        assert np.array_equal(r.truss, O.pkt(g.offsets, g.neighbours, threads=2))
    assert info["joined"] >= 1, info
    # joined members leave as soon as they finish: the small ones do not wait for the big one
    assert min(r.latency_ms for r in rs) < rb.latency_ms


def test_invalid_request_is_isolated_from_a_running_union():
    good = gen.rmat(12, 16, seed=5)
    bad = (np.array([0, 1, 3, 4, 4], np.uint64), np.array([1, 0, 2, 3], np.uint32))
    big = gen.rmat(19, 16, seed=8)
    with _one_lane_server(8 << 30) as srv:
        tb = srv.submit(big.offsets, big.neighbours)
        time.sleep(0.01)
        tx = srv.submit(*bad)
        tg = [srv.submit(good.offsets, good.neighbours) for _ in range(5)]
        assert srv.wait(tx, timeout_ms=60_000).status == P.E_INVALID_CSR
        want = O.pkt(good.offsets, good.neighbours)
        for t in tg:
            r = srv.wait(t, timeout_ms=60_000)
            assert r.status == P.OK and np.array_equal(r.truss, want)
        assert srv.wait(tb, timeout_ms=60_000).status == P.OK


def test_large_request_runs_with_row_hash_tables():
    """A request of more than 2^26 slots (R-MAT-22, 128 M) runs in a served union
    that takes no joins, and so gets the row hash tables: its truss equals the
    pinned fixture, and requests submitted while it runs are decomposed in the
    other lanes and equal the oracle's."""
    import hashlib
    import json
    import os
    fx = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "fixtures.json")))["cfg2_rmat22"]
    big = gen.rmat(22, 16, seed=2)
    rng = np.random.default_rng(31)
    small = [random_graph(rng, n_max=60) for _ in range(6)] + [gen.rmat(12, 16, seed=9)]
    with PktServer(48 << 30) as srv:
        tb = srv.submit(big.offsets, big.neighbours)
        time.sleep(0.05)
        ts = [srv.submit(g.offsets, g.neighbours) for g in small]
        rs = [srv.wait(t, timeout_ms=120_000) for t in ts]
        rb = srv.wait(tb, timeout_ms=300_000)
    assert rb.status == P.OK
    sha = hashlib.sha256(np.ascontiguousarray(rb.truss, dtype="<u4").tobytes()).hexdigest()
    assert sha == fx["modes"]["0"]["truss_sha256"]
    for g, r in zip(small, rs):
        assert r.status == P.OK
        assert np.array_equal(r.truss, O.pkt(g.offsets, g.neighbours, threads=2))
