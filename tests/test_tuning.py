"""The tuning cache on the CPU: the degree signature, store / lookup / clear,
and the text file the autotuner writes (no GPU: nothing here launches work)."""
import numpy as np
import pytest

from sparkx_b200 import build, gen
import sparkx_b200.pkt as P


@pytest.fixture(scope="module", autouse=True)
def _lib():
    build.build_engine()
    P.lib()
    yield
    P.tuning_clear()


def _signature(g):
    d = np.diff(g.offsets.astype(np.int64))
    d = d[d > 0]
    b = np.floor(np.log2(d)).astype(np.int64) + 1
    slots = np.bincount(b, weights=d, minlength=34)
    heavy = slots[9:].sum()
    total = slots.sum()
    return (int(np.log2(g.width)) if g.width else 0, int(b.max()) if b.size else 0,
            int(min(7, 8 * heavy // total)) if total else 0)


def test_signature_matches_the_degree_histogram():
    for g in (gen.rmat(12, 16, seed=2), gen.erdos_renyi(5000, 40000, 1), gen.rmat(14, 8, seed=3),
              gen.from_edges(3, [(0, 1)])):
        assert P.tuning_signature(g.offsets) == _signature(g)


def test_store_lookup_save_load(tmp_path):
    P.tuning_clear()
    key = (20, 12, 1)
    t, found = P.tuning_lookup(key)
    assert not found and t == P.PktTuning()
    mine = P.PktTuning(merge_ratio=4, hub_min_degree=512, sample_min=128, support_kernel=2, compact_pct=75,
                       hash_min_degree=32, sup_hash_min=16, relabel=1)
    P.tuning_store(key, mine)
    assert P.tuning_lookup(key) == (mine, True)
    path = str(tmp_path / "tune.txt")
    P.tuning_save(path)
    P.tuning_clear()
    assert not P.tuning_lookup(key)[1]
    P.tuning_load(path)
    assert P.tuning_lookup(key) == (mine, True)
    with pytest.raises(P.PktError):
        P.tuning_store(key, P.PktTuning(compact_pct=5))   # out of range
    with pytest.raises(P.PktError):
        P.tuning_store(key, P.PktTuning(hub_min_degree=100))
    with pytest.raises(P.PktError):
        P.tuning_store(key, P.PktTuning(sup_hash_min=2))
    with pytest.raises(P.PktError):
        P.tuning_store(key, P.PktTuning(relabel=2))
    P.tuning_clear()


def test_defaults_depend_on_the_key():
    """Unskewed keys with a largest degree of 64..255 default to the vertex form
    of the support pass; other keys keep the edge form; large skewed keys relabel."""
    P.tuning_clear()
    assert P.tuning_lookup((24, 7, 0)) == (P.PktTuning(support_kernel=2), False)
    assert P.tuning_lookup((27, 8, 0)) == (P.PktTuning(support_kernel=2), False)
    for key in ((24, 6, 0), (24, 9, 0), (24, 7, 1), (25, 3, 0), (27, 20, 1)):
        assert P.tuning_lookup(key) == (P.PktTuning(), False), key
    # large skewed keys (2^26 slots or more, a quarter of them in rows of degree >= 256) relabel
    for key in ((27, 20, 4), (26, 18, 5), (28, 19, 2)):
        assert P.tuning_lookup(key) == (P.PktTuning(relabel=1), False), key
    for key in ((25, 17, 4), (22, 12, 2), (20, 15, 7)):
        assert P.tuning_lookup(key) == (P.PktTuning(), False), key
