"""Synthetic CSR workloads for PKT k-truss (host-side C++ generators).

The graphs come back in the layout the reference's graph store memory-maps
(``graph/mod.rs:482-489``): ``offsets`` u64[n+1] and neighbour ids sorted
ascending within each row, both directions of every undirected edge present.
Self-loops and duplicates are removed.  Draws are counter based (splitmix64),
so a graph depends only on its parameters and seed, never on thread count.
"""
from __future__ import annotations

import ctypes
import dataclasses
import math

import numpy as np

from ._native import load_library

_RMAT_ABC = (0.57, 0.19, 0.19)


class _MixMember(ctypes.Structure):
    _fields_ = [
        ("kind", ctypes.c_uint32),
        ("scale", ctypes.c_uint32),
        ("n", ctypes.c_uint64),
        ("pairs", ctypes.c_uint64),
        ("avg_degree", ctypes.c_double),
        ("seed", ctypes.c_uint64),
    ]


def _lib():
    lib = load_library("libsparx_graphgen.so")
    if not getattr(lib, "_sgx_typed", False):
        vp = ctypes.c_void_p
        u64 = ctypes.c_uint64
        lib.sgx_gen_er.restype = vp
        lib.sgx_gen_er.argtypes = [u64, u64, u64]
        lib.sgx_gen_rmat.restype = vp
        lib.sgx_gen_rmat.argtypes = [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_double,
                                     ctypes.c_double, ctypes.c_double, u64, ctypes.c_int]
        lib.sgx_gen_debruijn.restype = vp
        lib.sgx_gen_debruijn.argtypes = [u64, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32,
                                         ctypes.c_double, u64]
        lib.sgx_mix_describe.restype = ctypes.c_int
        lib.sgx_mix_describe.argtypes = [u64, u64, ctypes.c_double, ctypes.c_double,
                                         ctypes.c_double, ctypes.c_double,
                                         ctypes.POINTER(_MixMember)]
        lib.sgx_gen_mix_member.restype = vp
        lib.sgx_gen_mix_member.argtypes = [ctypes.POINTER(_MixMember), ctypes.c_double,
                                           ctypes.c_double, ctypes.c_double]
        lib.sgx_graph_dims.restype = None
        lib.sgx_graph_dims.argtypes = [vp, ctypes.POINTER(u64), ctypes.POINTER(u64)]
        lib.sgx_graph_copy.restype = ctypes.c_int
        lib.sgx_graph_copy.argtypes = [vp, vp, vp, ctypes.c_int]
        lib.sgx_graph_free.restype = None
        lib.sgx_graph_free.argtypes = [vp]
        lib.sgx_set_threads.restype = ctypes.c_int
        lib.sgx_set_threads.argtypes = [ctypes.c_int]
        lib._sgx_typed = True
    return lib


@dataclasses.dataclass
class Csr:
    """Symmetric CSR: ``offsets`` u64[n+1], ``neighbours`` u32 or u64 [width]."""

    offsets: np.ndarray
    neighbours: np.ndarray
    name: str = ""

    @property
    def n(self) -> int:
        return int(self.offsets.shape[0]) - 1

    @property
    def width(self) -> int:
        return int(self.neighbours.shape[0])

    @property
    def m(self) -> int:
        """Undirected edges (self-loop slots counted once)."""
        return (self.width + self.self_loops()) // 2

    def self_loops(self) -> int:
        rows = np.repeat(np.arange(self.n, dtype=np.uint64), np.diff(self.offsets).astype(np.int64))
        return int(np.count_nonzero(rows == self.neighbours.astype(np.uint64)))

    def as_u64(self) -> "Csr":
        return Csr(self.offsets, self.neighbours.astype(np.uint64, copy=False), self.name)

    def as_u32(self) -> "Csr":
        if self.n >= 2**32:
            raise ValueError("vertex ids do not fit u32")
        return Csr(self.offsets, self.neighbours.astype(np.uint32, copy=False), self.name)


def _take(handle, name: str, bits: int = 32) -> Csr:
    lib = _lib()
    if not handle:
        raise RuntimeError(f"graph generator failed for {name}")
    try:
        n = ctypes.c_uint64()
        w = ctypes.c_uint64()
        lib.sgx_graph_dims(handle, ctypes.byref(n), ctypes.byref(w))
        off = np.empty(n.value + 1, dtype=np.uint64)
        nbr = np.empty(w.value, dtype=np.uint32 if bits == 32 else np.uint64)
        rc = lib.sgx_graph_copy(handle, off.ctypes.data, nbr.ctypes.data, bits)
        if rc:
            raise RuntimeError("sgx_graph_copy failed")
    finally:
        lib.sgx_graph_free(handle)
    return Csr(off, nbr, name)


def set_threads(t: int) -> int:
    """Host threads used by the generators (OpenMP); returns the active count."""
    return _lib().sgx_set_threads(int(t))


def erdos_renyi(n: int, m: int, seed: int, bits: int = 32) -> Csr:
    """n vertices, the first m distinct unordered pairs u != v in draw order."""
    return _take(_lib().sgx_gen_er(n, m, seed), f"er-n{n}-m{m}-s{seed}", bits)


def rmat(scale: int, edge_factor: int = 16, a: float = 0.57, b: float = 0.19, c: float = 0.19,
         seed: int = 2, permute: bool = True, bits: int = 32) -> Csr:
    """R-MAT with 2^scale vertices and edge_factor * 2^scale generated pairs."""
    h = _lib().sgx_gen_rmat(scale, edge_factor, a, b, c, seed, int(permute))
    return _take(h, f"rmat-{scale}-ef{edge_factor}-s{seed}", bits)


def debruijn(seq_len: int = 20_000_000, k: int = 21, copies: int = 1000, seg_len: int = 10_000,
             mut_rate: float = 0.05, seed: int = 3, bits: int = 32) -> Csr:
    """Distinct k-mers of a seeded sequence plus mutated segment copies;
    an undirected edge joins k-mers overlapping by k-1 bases."""
    h = _lib().sgx_gen_debruijn(seq_len, k, copies, seg_len, mut_rate, seed)
    return _take(h, f"dbg-L{seq_len}-k{k}-c{copies}-s{seed}", bits)


@dataclasses.dataclass
class MixMember:
    index: int
    kind: str           # "er" | "rmat"
    n: int
    pairs: int
    avg_degree: float
    seed: int
    scale: int


def mix_member(index: int, base_seed: int = 1000, n_lo: float = 1e3, n_hi: float = 1e6,
               d_lo: float = 4.0, d_hi: float = 64.0) -> MixMember:
    """Description of member ``index`` of the batched mix (seed base_seed + index)."""
    d = _MixMember()
    rc = _lib().sgx_mix_describe(index, base_seed, n_lo, n_hi, d_lo, d_hi, ctypes.byref(d))
    if rc:
        raise ValueError("bad mix parameters")
    return MixMember(index, "rmat" if d.kind == 1 else "er", int(d.n), int(d.pairs),
                     float(d.avg_degree), int(d.seed), int(d.scale))


def mix_graph(member: MixMember, bits: int = 32) -> Csr:
    d = _MixMember(1 if member.kind == "rmat" else 0, member.scale, member.n, member.pairs,
                   member.avg_degree, member.seed)
    h = _lib().sgx_gen_mix_member(ctypes.byref(d), *_RMAT_ABC)
    return _take(h, f"mix-{member.index}-{member.kind}-n{member.n}", bits)


def from_edges(n: int, edges, bits: int = 32) -> Csr:
    """Symmetric CSR from an undirected edge list (tests; duplicates removed,
    self-loops kept so callers can exercise them)."""
    pairs = set()
    for u, v in edges:
        pairs.add((u, v))
        pairs.add((v, u))
    rows = [[] for _ in range(n)]
    for u, v in pairs:
        rows[u].append(v)
    off = np.zeros(n + 1, dtype=np.uint64)
    nbr = []
    for u in range(n):
        r = sorted(rows[u])
        nbr.extend(r)
        off[u + 1] = off[u] + len(r)
    return Csr(off, np.asarray(nbr, dtype=np.uint32 if bits == 32 else np.uint64), "edges")


def log_uniform_mean(lo: float, hi: float) -> float:
    return (hi - lo) / math.log(hi / lo)


def from_multi_edges(n: int, edges, bits: int = 32) -> Csr:
    """Symmetric multigraph CSR from an undirected edge list in which repeats
    are parallel edges: every (u, v), u != v, adds slot v to row u and slot u to
    row v; a self-loop (u, u) adds one slot u to row u (its own reciprocal, as
    in the reference's edge index).  Rows sorted ascending, copies side by side
    (the layout the reference's GGCAT cache gives parallel edges)."""
    rows = [[] for _ in range(n)]
    for u, v in edges:
        rows[u].append(v)
        if u != v:
            rows[v].append(u)
    off = np.zeros(n + 1, dtype=np.uint64)
    nbr = []
    for u in range(n):
        r = sorted(rows[u])
        nbr.extend(r)
        off[u + 1] = off[u] + len(r)
    return Csr(off, np.asarray(nbr, dtype=np.uint32 if bits == 32 else np.uint64), "multi-edges")


def with_parallel_edges(g: Csr, frac: float, max_extra: int = 2, seed: int = 0) -> Csr:
    """A multigraph from a simple graph: each undirected edge (self-loops
    excepted) gets, with probability ``frac``, between 1 and ``max_extra``
    extra copies (seeded), added to both of its rows."""
    rng = np.random.default_rng(seed)
    off = g.offsets.astype(np.int64)
    nbr = g.neighbours.astype(np.int64)
    src = np.repeat(np.arange(g.n, dtype=np.int64), np.diff(off))
    up = src < nbr
    a, b = src[up], nbr[up]
    extra = np.where(rng.random(a.shape[0]) < frac, rng.integers(1, max_extra + 1, a.shape[0]), 0)
    ea, eb = np.repeat(a, extra), np.repeat(b, extra)
    rs = np.concatenate([src, ea, eb])
    cs = np.concatenate([nbr, eb, ea])
    order = np.lexsort((cs, rs))
    rs, cs = rs[order], cs[order]
    new_off = np.zeros(g.n + 1, dtype=np.uint64)
    np.cumsum(np.bincount(rs, minlength=g.n), out=new_off[1:])
    return Csr(new_off, cs.astype(np.uint32 if g.neighbours.dtype == np.uint32 else np.uint64),
               f"{g.name}-parallel{frac}")
