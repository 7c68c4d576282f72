"""GPU k-core decomposition against the oracle's restatement of the reference's peel
(k_core/liu_et_al.rs:190-420).  Core numbers are integers: compared exactly."""
import numpy as np
import pytest

from conftest import kn, random_graph
from oracle import oracle as O
from sparkx_b200 import AlgoLiuEtAl, GraphMemoryMap, gen
from sparkx_b200 import pkt as P

pytestmark = pytest.mark.gpu


def _check(g, mode=P.SUPPORT_WIDE, oracle_mode=O.MODE_WIDE, out_bits=32):
    cores, st = P.run_kcore(g.offsets, g.neighbours, P.PktOptions(support_mode=mode, out_bits=out_bits))
    want = O.kcore(g.offsets, g.neighbours, mode=oracle_mode)
    assert np.array_equal(cores.astype(np.int64), want)
    assert st.k_max == (int(want.max()) if want.size else 0)
    return st


def test_kcore_known_answers():
    _check(gen.from_edges(3, [(0, 1), (1, 2)]))
    _check(gen.from_edges(5, [(0, 1), (0, 2), (0, 3), (1, 2)]))
    for n in (2, 3, 7):
        _check(kn(n))
    _check(gen.from_edges(4, [(0, 0), (0, 1), (1, 2), (2, 2)]))  # self-loops count in the degree


def test_kcore_random_graphs():
    rng = np.random.default_rng(31)
    for _ in range(25):
        _check(random_graph(rng), out_bits=8)


def test_kcore_rmat_and_u8_degrees():
    st = _check(gen.rmat(14, 16, seed=8))
    assert st.levels > 1 and st.waves >= st.levels
    _check(gen.erdos_renyi(5000, 40000, 12))
    # degrees past 255 wrap in u8 mode, as the reference's AtomicU8 degrees do
    _check(kn(300), P.SUPPORT_U8, O.MODE_U8)
    _check(gen.rmat(12, 32, seed=2), P.SUPPORT_U8, O.MODE_U8, out_bits=8)


def test_kcore_u8_output_overflow():
    with pytest.raises(P.PktError) as e:
        P.run_kcore(kn(300).offsets, kn(300).neighbours, P.PktOptions(out_bits=8))
    assert e.value.status == P.E_OVERFLOW_U8
    cores, _ = P.run_kcore(kn(300).offsets, kn(300).neighbours, P.PktOptions(out_bits=32))
    assert set(cores.tolist()) == {299}


def test_algoliu_api(tmp_path, monkeypatch):
    monkeypatch.setattr(P, "CACHE_DIR", str(tmp_path))
    g = gen.rmat(11, 8, seed=5)
    gm = GraphMemoryMap.from_csr(g.as_u64())
    a = AlgoLiuEtAl.new(gm)
    want = O.kcore(g.offsets, g.neighbours)
    assert np.array_equal(a.k_cores(), want.astype(np.uint8))
    assert a.coreness(4) == want[4]
    again = AlgoLiuEtAl.get_or_compute(gm)
    assert np.array_equal(again.k_cores(), a.k_cores())
    a.drop_cache()
    assert np.array_equal(gm.k_core_lea().k_cores(), a.k_cores())


def test_kcore_level_loop_on_device_and_host_agree():
    """The device-resident level loop (CUDA-graph WHILE node, the default) and host-launched
    waves (SPARX_LOOP_HOST) give the oracle's core numbers, on graphs with many levels and
    multigraph rows (a parallel edge counts once per copy in the reference's degree)."""
    rng = np.random.default_rng(37)
    graphs = [gen.rmat(15, 16, seed=9), gen.with_parallel_edges(gen.rmat(11, 16, seed=3), 0.3, seed=3)]
    graphs += [random_graph(rng) for _ in range(5)]
    for g in graphs:
        want = O.kcore(g.offsets, g.neighbours)
        for loop in (P.LOOP_GRAPH, P.LOOP_HOST):
            cores, st = P.run_kcore(g.offsets, g.neighbours, P.PktOptions(out_bits=32, loop=loop))
            assert np.array_equal(cores.astype(np.int64), want), loop
            assert st.k_max == (int(want.max()) if want.size else 0)
