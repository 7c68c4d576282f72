import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")
    config.addinivalue_line("markers", "slow: long-running case")


@pytest.fixture(scope="session", autouse=True)
def _native_build():
    """Host-side libraries (generators, oracle) are built on demand; the CUDA
    engine is built by __graft_entry__.build() / python -m sparkx_b200.build."""
    from oracle import oracle as O
    from sparkx_b200 import build
    O.build()
    build.build_graphgen()
    yield


def kn(n):
    from sparkx_b200 import gen
    return gen.from_edges(n, [(i, j) for i in range(n) for j in range(i + 1, n)])


def book(pages):
    """Spine (0, 1) plus `pages` vertices adjacent to both: the spine lies in
    `pages` triangles, every page edge in one."""
    from sparkx_b200 import gen
    edges = [(0, 1)]
    for p in range(2, pages + 2):
        edges += [(0, p), (1, p)]
    return gen.from_edges(pages + 2, edges)


def random_graph(rng, n_max=40, self_loop_p=0.2):
    from sparkx_b200 import gen
    n = int(rng.integers(1, n_max))
    p = rng.uniform(0.03, 0.9)
    edges = [(i, j) for i in range(n) for j in range(i + 1, n) if rng.random() < p]
    if n and rng.random() < self_loop_p:
        v = int(rng.integers(0, n))
        edges.append((v, v))
    return gen.from_edges(n, edges)


def random_multigraph(rng, n_max=30):
    """A random graph whose edges repeat (parallel copies, up to four of a pair) and
    which may carry repeated self-loops."""
    from sparkx_b200 import gen
    n = int(rng.integers(2, n_max))
    p = rng.uniform(0.05, 0.8)
    edges = []
    for i in range(n):
        for j in range(i + 1, n):
            if rng.random() < p:
                edges += [(i, j)] * int(rng.choice([1, 1, 1, 2, 3, 4]))
    for _ in range(int(rng.integers(0, 3))):
        v = int(rng.integers(0, n))
        edges += [(v, v)] * int(rng.integers(1, 3))
    return gen.from_multi_edges(n, edges)


# Hand-derived known answers: (name, n, edges, expected truss per undirected edge)
def kats():
    out = []
    for n in range(2, 8):
        out.append((f"K{n}", n, [(i, j) for i in range(n) for j in range(i + 1, n)], None, n))
    out.append(("triangle", 3, [(0, 1), (1, 2), (0, 2)], None, 3))
    out.append(("path", 5, [(0, 1), (1, 2), (2, 3), (3, 4)], None, 2))
    out.append(("star", 6, [(0, i) for i in range(1, 6)], None, 2))
    out.append(("two_triangles_sharing_edge", 4, [(0, 1), (0, 2), (1, 2), (1, 3), (2, 3)], None, 3))
    k4_pendant = [(i, j) for i in range(4) for j in range(i + 1, 4)] + [(3, 4)]
    out.append(("K4_plus_pendant", 5, k4_pendant, {(3, 4): 2}, 4))
    out.append(("isolated_vertices", 6, [(0, 1), (1, 2), (0, 2)], None, 3))
    out.append(("self_loop_on_triangle", 3, [(0, 1), (1, 2), (0, 2), (1, 1)], {(1, 1): 2}, 3))
    out.append(("empty", 4, [], None, 2))
    # K5 sharing an edge with a triangle: K5 edges 5, the triangle's two other edges 3
    k5 = [(i, j) for i in range(5) for j in range(i + 1, 5)]
    out.append(("K5_with_triangle", 6, k5 + [(0, 5), (1, 5)], {(0, 5): 3, (1, 5): 3}, 5))
    return out


def expected_truss(csr, special, default):
    import numpy as np
    off = csr.offsets.astype(np.int64)
    exp = np.full(csr.width, default, dtype=np.uint32)
    for u in range(csr.n):
        for s in range(off[u], off[u + 1]):
            v = int(csr.neighbours[s])
            key = (min(u, v), max(u, v))
            if special and key in special:
                exp[s] = special[key]
    return exp
