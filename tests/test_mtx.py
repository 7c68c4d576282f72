"""MatrixMarket ingestion: the oracle's restatement of the reference parser
(graph/cache/parser_mtx) on hand-written texts (no GPU)."""
import numpy as np
import pytest

from oracle import oracle as O
from sparkx_b200 import gen

SYM = b"""%%MatrixMarket matrix coordinate pattern symmetric
% a comment
%
4 4 5

2 1
3 1
3 2
   4 4
4 3
"""


def test_symmetric_pattern_with_comments_blank_lines_and_a_self_loop():
    off, nbr = O.mtx_to_csr(SYM)
    assert off.tolist() == [0, 2, 4, 7, 9]
    assert nbr.tolist() == [1, 2, 0, 2, 0, 1, 3, 2, 3]


def test_general_keeps_direction_integer_field_and_duplicates():
    txt = b"%%MatrixMarket MATRIX Coordinate integer General\n3 3 4\n1 2 7\n1 2 9\n3 1 5\n2 2 1\n"
    off, nbr = O.mtx_to_csr(txt)
    assert off.tolist() == [0, 2, 3, 4]
    assert nbr.tolist() == [1, 1, 1, 0]
    # skew-symmetric mirrors like symmetric; duplicates stay (parallel edges)
    off, nbr = O.mtx_to_csr(b"%%MatrixMarket matrix coordinate pattern skew-symmetric\n2 2 2\n2 1\n2 1\n")
    assert off.tolist() == [0, 2, 4] and nbr.tolist() == [1, 1, 0, 0]


@pytest.mark.parametrize("txt", [
    b"%%MatrixMarket matrix coordinate real symmetric\n2 2 1\n2 1\n",     # field
    b"%%MatrixMarket matrix array pattern symmetric\n2 2 1\n2 1\n",        # not coordinate
    b"%MatrixMarket matrix coordinate pattern symmetric\n2 2 1\n2 1\n",    # header
    b"%%MatrixMarket matrix coordinate pattern symmetric\n2 3 1\n2 1\n",   # not square
    b"%%MatrixMarket matrix coordinate pattern symmetric\n2 2 1\n0 1\n",   # 0-based index
    b"%%MatrixMarket matrix coordinate pattern symmetric\n2 2 1\n3 1\n",   # out of range
    b"%%MatrixMarket matrix coordinate pattern symmetric\n2 2 1\n2 x\n",   # not a number
    b"%%MatrixMarket matrix coordinate pattern symmetric\n% only comments\n",
])
def test_malformed_texts_are_errors(txt):
    with pytest.raises(O.OracleError):
        O.mtx_to_csr(txt)


def test_short_lines_are_skipped_and_plus_signs_parse():
    txt = b"%%MatrixMarket matrix coordinate pattern symmetric\n3 3 2\n2\n+3 +1\n"
    off, nbr = O.mtx_to_csr(txt)
    assert off.tolist() == [0, 1, 1, 2] and nbr.tolist() == [2, 0]


def test_round_trip_of_a_generated_graph():
    g = gen.rmat(9, 8, seed=4)
    off, nbr = O.mtx_to_csr(O.csr_to_mtx(g.offsets, g.neighbours))
    assert np.array_equal(off, g.offsets) and np.array_equal(nbr, g.neighbours.astype(np.uint64))
    m = gen.from_multi_edges(4, [(0, 1), (0, 1), (1, 2), (2, 2), (2, 3)])
    off, nbr = O.mtx_to_csr(O.csr_to_mtx(m.offsets, m.neighbours, field="integer"))
    assert np.array_equal(off, m.offsets) and np.array_equal(nbr, m.neighbours.astype(np.uint64))
