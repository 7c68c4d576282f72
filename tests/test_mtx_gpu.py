"""MatrixMarket ingestion on the GPU (sparx_mtx_to_csr) against the oracle's
restatement of the reference parser, bit-exact, and into the PKT engine."""
import os

import numpy as np
import pytest

from oracle import oracle as O
from sparkx_b200 import gen
from sparkx_b200.graph import GraphMemoryMap
import sparkx_b200.pkt as P
from test_mtx import SYM

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _engine():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    from sparkx_b200 import build
    build.build_engine()
    yield


TEXTS = [
    SYM,
    b"%%MatrixMarket MATRIX Coordinate integer General\n3 3 4\n1 2 7\n1 2 9\n3 1 5\n2 2 1\n",
    b"%%MatrixMarket matrix coordinate pattern skew-symmetric\n2 2 2\n2 1\n2 1\n",
    b"%%MatrixMarket matrix coordinate pattern symmetric\n3 3 2\n2\n+3 +1\n",
    b"%%MatrixMarket matrix coordinate pattern symmetric\n5 5 0\n",                   # no entries
    b"%%MatrixMarket matrix coordinate pattern symmetric\r\n3 3 2\r\n2 1\r\n3 2\r\n",   # CRLF
    b"%%MatrixMarket matrix coordinate pattern symmetric\n3 3 2\n2 1\n3 2",              # no final newline
]


@pytest.mark.parametrize("i", range(len(TEXTS)))
def test_small_texts_match_the_oracle(i):
    want = O.mtx_to_csr(TEXTS[i])
    got = P.mtx_to_csr(TEXTS[i])
    assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1])


@pytest.mark.parametrize("txt", [
    b"%%MatrixMarket matrix coordinate pattern symmetric\n2 2 1\n0 1\n",
    b"%%MatrixMarket matrix coordinate pattern symmetric\n2 2 1\n3 1\n",
    b"%%MatrixMarket matrix coordinate pattern symmetric\n2 2 1\n2 x\n",
    b"%%MatrixMarket matrix coordinate real symmetric\n2 2 1\n2 1\n",
    b"%%MatrixMarket matrix coordinate pattern symmetric\n2 3 1\n2 1\n",
])
def test_malformed_texts_return_parse_status(txt):
    with pytest.raises(P.PktError) as ei:
        P.mtx_to_csr(txt)
    assert ei.value.status == P.E_PARSE


def test_large_round_trip_and_random_order():
    # R-MAT-16 written as a symmetric pattern file, then with its entry lines shuffled
    g = gen.rmat(16, 16, seed=2)
    txt = O.csr_to_mtx(g.offsets, g.neighbours)
    off, nbr = P.mtx_to_csr(txt)
    assert np.array_equal(off, g.offsets) and np.array_equal(nbr, g.neighbours.astype(np.uint64))
    lines = txt.split(b"\n")
    k = next(i for i, l in enumerate(lines) if l.startswith(str(g.n).encode() + b" "))
    entries = [l for l in lines[k + 1:] if l]
    rng = np.random.default_rng(3)
    order = rng.permutation(len(entries))
    shuffled = b"\n".join(lines[:k + 1] + [entries[i] for i in order]) + b"\n"
    off2, nbr2 = P.mtx_to_csr(shuffled)
    assert np.array_equal(off2, g.offsets) and np.array_equal(nbr2, g.neighbours.astype(np.uint64))


def test_mtx_file_into_pkt(tmp_path):
    # a multigraph file (repeated entries) through GraphMemoryMap.from_mtx_file and AlgoPKT
    m = gen.with_parallel_edges(gen.rmat(11, 16, seed=6), 0.3, max_extra=2, seed=6)
    path = os.path.join(tmp_path, "g.mtx")
    with open(path, "wb") as f:
        f.write(O.csr_to_mtx(m.offsets, m.neighbours, field="integer"))
    g = GraphMemoryMap.from_mtx_file(path)
    assert np.array_equal(g.offsets(), m.offsets)
    truss, _ = P.run_pkt(g.offsets(), g.neighbours(), P.PktOptions(out_bits=32))
    assert np.array_equal(truss, O.pkt(m.offsets, m.neighbours, threads=4))
