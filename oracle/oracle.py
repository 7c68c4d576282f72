"""ORACLE — test infrastructure only (the checker, never the product path).

Python side of the CPU restatement in ``pkt_oracle.cpp`` plus a brute-force
truss decomposition straight from the definition.  Only ``tests/``,
``__graft_entry__.smoke()`` and the CPU-baseline legs of ``bench.py`` may
import this module.

Parity is unpinned by the reference: the Rust reference cannot be built here
and ships no truss/support golden vectors (see ``pkt_oracle.cpp``).  The
restatements are pinned by hand-derived known answers and by agreement with
``brute_force_truss`` (below) on random graphs.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

MODE_WIDE = 0
MODE_U8 = 1

ERRORS = {0: "ok", 1: "invalid CSR", 2: "multigraph", 3: "level overflow (u8)", 4: "queue full"}


class OracleError(RuntimeError):
    pass


def build(force: bool = False) -> str:
    path = os.path.join(_HERE, "liboracle.so")
    src = os.path.join(_HERE, "pkt_oracle.cpp")
    if force or not os.path.exists(path) or os.path.getmtime(path) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", _HERE, "liboracle.so"], check=True)
    return path


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        vp, u64, i32 = ctypes.c_void_p, ctypes.c_uint64, ctypes.c_int
        L.orc_validate.restype = i32
        L.orc_validate.argtypes = [u64, vp, vp]
        L.orc_edge_index.restype = i32
        L.orc_edge_index.argtypes = [u64, vp, vp, vp, vp, i32]
        L.orc_triangles.restype = i32
        L.orc_triangles.argtypes = [u64, vp, vp, vp, vp, i32, i32, i32, vp]
        L.orc_pkt.restype = i32
        L.orc_pkt.argtypes = [u64, vp, vp, vp, vp, i32, i32, i32, vp, vp]
        L.orc_burkhardt.restype = i32
        L.orc_burkhardt.argtypes = [u64, vp, vp, vp, vp, i32, i32, vp]
        L.orc_verify.restype = u64
        L.orc_verify.argtypes = [u64, vp, vp, vp, vp, i32]
        L.orc_fast_truss.restype = i32
        L.orc_fast_truss.argtypes = [u64, vp, vp, i32, i32, vp, vp, vp]
        _LIB = L
    return _LIB


def _csr(off, nbr):
    off = np.ascontiguousarray(off, dtype=np.uint64)
    nbr = np.ascontiguousarray(nbr, dtype=np.uint32)
    return off, nbr, len(off) - 1


def _check(rc):
    if rc:
        raise OracleError(ERRORS.get(rc, f"error {rc}"))


def edge_index(off, nbr, threads=1):
    """(eo, er) as in graph/impl_csc.rs:87-263."""
    off, nbr, n = _csr(off, nbr)
    eo = np.zeros(n, dtype=np.uint64)
    er = np.zeros(len(nbr), dtype=np.uint64)
    _check(lib().orc_edge_index(n, off.ctypes.data, nbr.ctypes.data, eo.ctypes.data,
                                er.ctypes.data, threads))
    return eo, er


def triangles(off, nbr, mode=MODE_WIDE, threads=1, hash_map=False, eo_er=None):
    """Per-slot triangle support as in k_truss/triangles.rs:144-243."""
    off, nbr, n = _csr(off, nbr)
    eo, er = eo_er if eo_er is not None else edge_index(off, nbr, threads)
    sup = np.zeros(len(nbr), dtype=np.uint32)
    _check(lib().orc_triangles(n, off.ctypes.data, nbr.ctypes.data, eo.ctypes.data,
                               er.ctypes.data, threads, mode, int(hash_map), sup.ctypes.data))
    return sup


def kcore(off, nbr, mode=MODE_WIDE):
    """Core numbers as k_core/liu_et_al.rs:190-420 computes them, peeled sequentially (the
    result does not depend on the order).  degree = row length, reduced mod 256 in MODE_U8
    (AtomicU8, :258); degree-0 vertices are dead with core 0 (:259-265); from k = 1 (:295),
    every live vertex with degree <= k is peeled with core k (:303-312); peeling u decrements a
    neighbour's degree only while it exceeds k, and a neighbour whose degree was k + 1 is
    peeled at the same level (:339-372); an empty level raises k (:316-327).  In MODE_U8 a
    level past 255 is the reference's overflow error (never reached: degrees stay below 256)."""
    off = np.ascontiguousarray(off, dtype=np.int64)
    nbr = np.ascontiguousarray(nbr, dtype=np.int64)
    n = len(off) - 1
    d = np.diff(off)
    deg = (d & 0xFF) if mode == MODE_U8 else d.copy()
    alive = d != 0
    core = np.zeros(n, dtype=np.int64)
    remaining = int(alive.sum())
    k = 1
    while remaining > 0:
        front = np.nonzero(alive & (deg <= k))[0]
        if front.size == 0:
            if mode == MODE_U8 and k == 255:
                raise OracleError("overflow when adding to k")
            k += 1
            continue
        alive[front] = False
        stack = [int(u) for u in front]
        while stack:
            u = stack.pop()
            core[u] = k
            remaining -= 1
            for v in nbr[off[u]:off[u + 1]]:
                if deg[v] > k:
                    deg[v] -= 1
                    if deg[v] == k and alive[v]:
                        alive[v] = False
                        stack.append(int(v))
    return core


def clustering(off, nbr, mode=MODE_WIDE, threads=1, faithful=False):
    """Local clustering coefficients, transitivity and their average, with the
    definitions of k_truss/clustering_coefficient.rs:93-190 but the INTENDED
    triangle counts (default), or the reference's actual output (faithful=True).

    Reference defect D4: compute() builds the supports with Triangles::new
    (clustering_coefficient.rs:105) and then, before reading them, overwrites
    every slot's counter with AtomicU8::new(0) (:130-135).  The reference
    therefore reads zero supports: every local coefficient is 0, the average is
    0 and the transitivity is 0 / 2 / (sum of possible pairs), i.e. 0 (NaN when
    no vertex has two neighbours).  It also sums a thread's slot supports into
    `total_triangles_t`, whose type is inferred from the u8 load (:129,144), so
    with real supports that running sum would wrap modulo 256.  faithful=True
    returns exactly that zero output; the default computes what the code means:

    For u with d distinct neighbours (the row's HashSet, :140-155):
    possible = d(d-1)/2 if d > 1 else 0; t = ceil(row support sum / 2); local = t / possible
    when possible is a normal float, else 0 (:160-172).  transitivity = (sum of all slot
    supports // 3) / 2 / sum(possible) (:157,178-181), summed without the u8 wrap and with one
    worker (the reference divides by 3 per worker thread, :157, so its value would depend on
    the thread count); average = sum(local) / n (:177).  Slot supports come from
    ``triangles`` (AtomicU8 counts in MODE_U8)."""
    off = np.ascontiguousarray(off, dtype=np.int64)
    nbr = np.ascontiguousarray(nbr, dtype=np.int64)
    n = len(off) - 1
    sup = triangles(off.astype(np.uint64), nbr.astype(np.uint64), mode=mode, threads=threads)
    sup = sup.astype(np.uint64)
    if faithful:
        sup[:] = 0  # clustering_coefficient.rs:130-135 zeroes the counters before reading them
    if mode == MODE_U8:
        sup &= np.uint64(0xFF)
    rows = np.repeat(np.arange(n), np.diff(off))
    same = np.zeros(len(nbr), dtype=bool)
    if len(nbr) > 1:
        same[1:] = (nbr[1:] == nbr[:-1]) & (rows[1:] == rows[:-1])
    deg = np.diff(off) - np.bincount(rows[same], minlength=n) if n else np.zeros(0, np.int64)
    possible = np.where(deg > 1, deg.astype(np.float64) * (deg - 1).astype(np.float64) / 2.0, 0.0)
    cs = np.concatenate([[0], np.cumsum(sup, dtype=np.uint64)]).astype(np.uint64)
    row_sum = cs[off[1:]] - cs[off[:-1]]
    tri = ((row_sum + np.uint64(1)) // np.uint64(2)).astype(np.float64)
    local = np.zeros(n, dtype=np.float64)
    pos = possible > 0
    local[pos] = tri[pos] / possible[pos]
    total_triangles = int(sup.sum()) // 3
    with np.errstate(divide="ignore", invalid="ignore"):
        transitivity = float(np.float64(total_triangles) / 2.0 / np.float64(possible.sum()))
        average = float(np.float64(local.sum()) / np.float64(n))
    return local, transitivity, average


def pkt(off, nbr, mode=MODE_WIDE, threads=1, hash_map=False, return_stats=False):
    """Truss per slot (u32) by the PKT restatement of k_truss/pkt.rs:216-563."""
    off, nbr, n = _csr(off, nbr)
    eo, er = edge_index(off, nbr, threads)
    sup = triangles(off, nbr, mode, threads, hash_map, (eo, er))
    truss = np.zeros(len(nbr), dtype=np.uint32)
    st = np.zeros(3, dtype=np.uint64)
    _check(lib().orc_pkt(n, off.ctypes.data, nbr.ctypes.data, er.ctypes.data, sup.ctypes.data,
                         threads, mode, int(hash_map), truss.ctypes.data, st.ctypes.data))
    if return_stats:
        return truss, {"levels": int(st[0]), "sublevels": int(st[1]), "max_level": int(st[2])}
    return truss


def burkhardt(off, nbr, mode=MODE_WIDE, hash_map=False):
    """Truss per slot by the restatement of k_truss/burkhardt_et_al.rs:186-380."""
    off, nbr, n = _csr(off, nbr)
    eo, er = edge_index(off, nbr)
    sup = triangles(off, nbr, mode, 1, hash_map, (eo, er))
    truss = np.zeros(len(nbr), dtype=np.uint32)
    _check(lib().orc_burkhardt(n, off.ctypes.data, nbr.ctypes.data, er.ctypes.data,
                               sup.ctypes.data, mode, int(hash_map), truss.ctypes.data))
    return truss


def verify(off, nbr, truss, threads=1):
    """Corrected k_truss/mod.rs:30-216; returns -1 if the assignment passes,
    else the first failing slot."""
    off, nbr, n = _csr(off, nbr)
    _, er = edge_index(off, nbr, threads)
    t = np.ascontiguousarray(truss, dtype=np.uint32)
    r = lib().orc_verify(n, off.ctypes.data, nbr.ctypes.data, er.ctypes.data, t.ctypes.data,
                         threads)
    return int(r) - 1


def fast_truss(off, nbr, mode=MODE_WIDE, threads=None):
    """Independent exact peel for large graphs: (truss per slot, triangles, levels)."""
    off, nbr, n = _csr(off, nbr)
    threads = threads or os.cpu_count() or 1
    truss = np.zeros(len(nbr), dtype=np.uint32)
    tri = ctypes.c_uint64()
    lev = ctypes.c_uint64()
    _check(lib().orc_fast_truss(n, off.ctypes.data, nbr.ctypes.data, threads, mode,
                                truss.ctypes.data, ctypes.byref(tri), ctypes.byref(lev)))
    return truss, int(tri.value), int(lev.value)


def brute_force_truss(off, nbr):
    """Truss per slot straight from the definition: the k-truss is the largest
    subgraph in which every edge lies in >= k-2 triangles; an edge's truss is
    the largest such k.  In a multigraph a triangle is one choice of a copy of
    each of its three pairs, so a copy of (u, v) lies in sum over common
    neighbours w of mu(u, w) * mu(v, w) of them, and all copies of a pair share
    its truss.  Pure Python: small graphs only."""
    off = np.asarray(off, dtype=np.int64)
    nbr = np.asarray(nbr, dtype=np.int64)
    n = len(off) - 1
    mu = {}
    for u in range(n):
        for s in range(off[u], off[u + 1]):
            v = int(nbr[s])
            if v > u:
                mu[(u, v)] = mu.get((u, v), 0) + 1
    truss = {e: 2 for e in mu}
    live = set(mu)
    k = 3
    while live:
        # peel to the k-truss of the current live graph
        ladj = {}
        for (u, v) in live:
            ladj.setdefault(u, {})[v] = mu[(u, v)]
            ladj.setdefault(v, {})[u] = mu[(u, v)]
        changed = True
        while changed:
            changed = False
            for (u, v) in list(live):
                au, av = ladj[u], ladj[v]
                sup = sum(c * av[w] for w, c in au.items() if w in av and w != u and w != v)
                if sup < k - 2:
                    live.discard((u, v))
                    del au[v]
                    del av[u]
                    changed = True
        for e in live:
            truss[e] = k
        k += 1
    out = np.zeros(len(nbr), dtype=np.uint32)
    for u in range(n):
        for s in range(off[u], off[u + 1]):
            v = int(nbr[s])
            out[s] = 2 if v == u else truss[(min(u, v), max(u, v))]
    return out


def support_definition(off, nbr):
    """Triangles per slot from the definition (multigraph-aware): a copy of (u, v)
    lies in sum over w != u, v of mu(u, w) * mu(v, w) triangles.  Small graphs."""
    off = np.asarray(off, dtype=np.int64)
    nbr = np.asarray(nbr, dtype=np.int64)
    n = len(off) - 1
    cnt = [dict() for _ in range(n)]
    for u in range(n):
        for s in range(off[u], off[u + 1]):
            v = int(nbr[s])
            if v != u:
                cnt[u][v] = cnt[u].get(v, 0) + 1
    out = np.zeros(len(nbr), dtype=np.uint64)
    for u in range(n):
        for s in range(off[u], off[u + 1]):
            v = int(nbr[s])
            if v != u:
                out[s] = sum(c * cnt[v][w] for w, c in cnt[u].items() if w in cnt[v] and w != v)
    return out


def _mtx_usize(tok: str) -> int:
    """Rust's usize::from_str: an optional '+', then ASCII digits (64-bit)."""
    t = tok[1:] if tok.startswith("+") else tok
    if not t or not all("0" <= c <= "9" for c in t):
        raise OracleError(f"not an unsigned integer: {tok!r}")
    v = int(t)
    if v >= 1 << 64:
        raise OracleError(f"integer overflow: {tok!r}")
    return v


def mtx_to_csr(data: bytes):
    """CSR (offsets u64[n+1], neighbours u64[width]) from MatrixMarket text, restating
    GraphCache::from_mtx_file (graph/cache/parser_mtx/mod.rs:34-162): the header checks and size
    line of parse_mtx_header (producers.rs:139-176), the entry lines of
    parallel_no_labels_parse_mtx_with (producers.rs:217-240: blank and '%' lines skipped, a line
    with fewer than two tokens skipped, 1-based indices, 0 or >= nrows an error, the mirror of
    (i, j) added unless the header says general or i == j), degree count and scatter
    (mod.rs:74-155) and the per-row sort (impl_sort.rs:10-51).  Duplicates stay.  The reference
    stops reading once its threads have seen nnz entries (checked per thread chunk); a text with
    exactly nnz entries is read in full, as here, where every entry line is read."""
    text = data.decode("latin-1")
    lines = text.split("\n")
    if not lines or not lines[0].startswith("%%MatrixMarket"):
        raise OracleError("invalid MatrixMarket header")
    toks = lines[0].split()
    if len(toks) < 5:
        raise OracleError("malformed MatrixMarket header")
    low = [t.lower() for t in toks]
    if (low[1] != "matrix" or low[2] != "coordinate" or low[3] not in ("pattern", "integer")
            or low[4] not in ("symmetric", "skew-symmetric", "general")):
        raise OracleError("unsupported MatrixMarket header")
    symmetric = low[4] != "general"
    k = 1
    while True:
        if k >= len(lines):
            raise OracleError("unexpected end before the size line")
        t = lines[k].strip()
        k += 1
        if not t or t.startswith("%"):
            continue
        parts = t.split()
        if len(parts) < 3:
            raise OracleError("malformed size line")
        nr, nc = _mtx_usize(parts[0]), _mtx_usize(parts[1])
        _mtx_usize(parts[2])
        if nr != nc:
            raise OracleError("nrows != ncols")
        n = nr
        break
    rows = [[] for _ in range(n)]
    for line in lines[k:]:
        t = line.strip()
        if not t or t.startswith("%"):
            continue
        parts = t.split()
        if len(parts) < 2:
            continue
        i1, j1 = _mtx_usize(parts[0]), _mtx_usize(parts[1])
        if i1 == 0 or j1 == 0:
            raise OracleError("MatrixMarket indices are 1-based")
        i, j = i1 - 1, j1 - 1
        if i >= n or j >= n:
            raise OracleError("entry out of bounds")
        rows[i].append(j)
        if symmetric and i != j:
            rows[j].append(i)
    off = np.zeros(n + 1, dtype=np.uint64)
    nbr = []
    for u in range(n):
        r = sorted(rows[u])
        nbr.extend(r)
        off[u + 1] = off[u] + len(r)
    return off, np.asarray(nbr, dtype=np.uint64)


def csr_to_mtx(offsets, neighbours, field: str = "pattern", comments: bool = True) -> bytes:
    """A symmetric MatrixMarket text listing each undirected pair once per copy (i >= j, the
    lower triangle), from which mtx_to_csr rebuilds the same CSR (test input)."""
    off = np.asarray(offsets, dtype=np.int64)
    nbr = np.asarray(neighbours, dtype=np.int64)
    n = len(off) - 1
    src = np.repeat(np.arange(n, dtype=np.int64), np.diff(off))
    low = src >= nbr
    i, j = src[low] + 1, nbr[low] + 1
    head = f"%%MatrixMarket matrix coordinate {field} symmetric\n"
    if comments:
        head += "% written by the oracle for a round-trip test\n%\n"
    head += f"{n} {n} {i.shape[0]}\n"
    if field == "integer":
        body = "\n".join(f"{a} {b} 1" for a, b in zip(i.tolist(), j.tolist()))
    else:
        body = "\n".join(f"{a} {b}" for a, b in zip(i.tolist(), j.tolist()))
    return (head + body + ("\n" if body else "")).encode()
