"""The allocation-free entry point (sparx_pkt_run_device_noalloc), checked
against the regular device entry point and against the oracle.

Callers such as a service whose device memory is all pre-reserved by its own
pool, or a request path that must not wait for or fail on cudaMalloc, cannot
let the library allocate a workspace; this entry point keeps its scratch in a
fixed static device array instead.  The test calls it twice in a row (the
array keeps the previous call's contents, so the second call checks that
everything that must start at zero is reset), the second time on a freshly
created non-default stream, and compares each result with
sparx_pkt_run_device and with the oracle's PKT bit for bit.  Collected last on
purpose; it also passes alone in a fresh process."""
import ctypes

import numpy as np
import pytest

from conftest import kn, random_graph
from oracle import oracle as O
from sparkx_b200 import gen
import sparkx_b200.pkt as P

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    assert torch.cuda.is_available(), "needs a CUDA device"
    from sparkx_b200 import build
    build.build_engine()
    return torch


def device_csr(torch, g):
    d_off = torch.from_numpy(np.ascontiguousarray(g.offsets).view(np.int64)).cuda()
    d_nbr = torch.from_numpy(np.ascontiguousarray(g.neighbours, dtype=np.uint32).view(np.int32)).cuda()
    return d_off, d_nbr


def via_regular_entry(torch, g):
    d_off, d_nbr = device_csr(torch, g)
    out = torch.empty(max(1, g.width), dtype=torch.int32, device="cuda")
    P.run_pkt_device(d_off.data_ptr(), g.n + 1, d_nbr.data_ptr(), g.width, out.data_ptr(),
                     P.PktOptions(out_bits=32), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    return out.cpu().numpy().view(np.uint32)[: g.width]


def via_noalloc(torch, g, stream=None):
    d_off, d_nbr = device_csr(torch, g)
    out = torch.full((max(1, g.width),), -1, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()  # inputs written on torch's stream are complete
    L = P.lib()
    s = stream if stream is not None else torch.cuda.current_stream()
    rc = L.sparx_pkt_run_device_noalloc(d_off.data_ptr(), g.n + 1, d_nbr.data_ptr(), g.width, out.data_ptr(),
                                         torch.cuda.current_device(), s.cuda_stream)
    assert rc == 0, (rc, L.sparx_last_error())
    torch.cuda.synchronize()
    return out.cpu().numpy().view(np.uint32)[: g.width]


def test_noalloc_matches_regular_entry_twice_in_a_row(torch_cuda):
    torch = torch_cuda
    rng = np.random.default_rng(17)
    graphs = [gen.rmat(12, 16, seed=2), kn(30), random_graph(rng, n_max=60, self_loop_p=1.0),
              gen.erdos_renyi(20_000, 120_000, 3)]
    for g in graphs:
        ref = via_regular_entry(torch, g)
        want = O.pkt(g.offsets, g.neighbours)
        assert np.array_equal(ref, want)
        first = via_noalloc(torch, g)
        second = via_noalloc(torch, g, stream=torch.cuda.Stream())  # a new non-default stream
        assert np.array_equal(first, want)
        assert np.array_equal(second, want)


def test_noalloc_rejects_graphs_beyond_its_scratch(torch_cuda):
    torch = torch_cuda
    g = gen.rmat(18, 16, seed=2)  # 7.6 M slots > the fixed scratch
    d_off, d_nbr = device_csr(torch, g)
    out = torch.empty(g.width, dtype=torch.int32, device="cuda")
    L = P.lib()
    rc = L.sparx_pkt_run_device_noalloc(d_off.data_ptr(), g.n + 1, d_nbr.data_ptr(), g.width, out.data_ptr(),
                                         torch.cuda.current_device(), None)
    assert rc == P.E_TOO_LARGE
    assert b"scratch" in L.sparx_last_error()
    # still usable afterwards
    small = gen.rmat(10, 8, seed=4)
    assert np.array_equal(via_noalloc(torch, small), via_regular_entry(torch, small))
