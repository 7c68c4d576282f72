"""``AlgoPKT`` / ``Triangles`` over the CUDA engine (``libsparx_pkt.so``).

Mirrors the reference's PKT entry point (``src/k_truss/pkt.rs:29-123``):

* ``AlgoPKT.new(g)``                 pkt.rs:45-52   (threads argument of the
  ``AlgoPKT.new_with_conf(g, threads)`` pkt.rs:85-95   reference is accepted and
                                                    ignored: the GPU does the work)
* ``AlgoPKT.get_or_compute(g)``      pkt.rs:61-76   (re-uses the cached result file)
* ``trussness(e)``                   pkt.rs:104-107 (asserts ``e < g.width()``)
* ``k_trusses()``                    pkt.rs:112-114 (u8 per CSR slot)
* ``drop_cache()``                   pkt.rs:117-122 (removes the result file)

and ``Triangles`` (``src/k_truss/triangles.rs:16-69``): support per CSR slot.

Errors are raised as ``PktError`` carrying the C status, the way the reference
returns ``Box<dyn Error>`` (e.g. the u8 level overflow at pkt.rs:508-516).
The native library is mandatory; there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import dataclasses
import os

import numpy as np

from ._native import load_library
from .graph import GraphMemoryMap

OK = 0
E_INVALID_CSR = 1
E_MULTIGRAPH = 2
E_OVERFLOW_U8 = 3
E_OOM = 4
E_TIMEOUT = 5
E_CUDA = 6
E_TOO_LARGE = 7
E_ARG = 8
E_NOT_FOUND = 9
E_CANCELLED = 10
E_PARSE = 11

SUPPORT_WIDE = 0
SUPPORT_U8 = 1
LOOP_GRAPH = 0
LOOP_HOST = 1

CACHE_DIR = os.environ.get("SPARX_CACHE_DIR", "./.cache")


class _Opts(ctypes.Structure):
    _fields_ = [
        ("struct_size", ctypes.c_uint32),
        ("support_mode", ctypes.c_uint32),
        ("out_bits", ctypes.c_uint32),
        ("device", ctypes.c_int32),
        ("loop", ctypes.c_uint32),
        ("support_kernel", ctypes.c_uint32),
        ("timeout_ms", ctypes.c_uint64),
    ]


class _Stats(ctypes.Structure):
    _fields_ = [
        ("n", ctypes.c_uint64), ("width", ctypes.c_uint64), ("m", ctypes.c_uint64),
        ("self_loops", ctypes.c_uint64), ("triangles", ctypes.c_uint64),
        ("max_support", ctypes.c_uint64), ("k_max", ctypes.c_uint32), ("levels", ctypes.c_uint32),
        ("waves", ctypes.c_uint32), ("launches", ctypes.c_uint32),
        ("ms_upload", ctypes.c_double), ("ms_orient", ctypes.c_double),
        ("ms_support", ctypes.c_double), ("ms_peel", ctypes.c_double),
        ("ms_finalize", ctypes.c_double), ("ms_download", ctypes.c_double),
        ("ms_total", ctypes.c_double),
        ("support_elements", ctypes.c_uint64), ("peel_elements", ctypes.c_uint64),
        ("peel_hits", ctypes.c_uint64), ("peel_scanned", ctypes.c_uint64),
        ("peel_edges", ctypes.c_uint64), ("compactions", ctypes.c_uint32), ("hub_maps", ctypes.c_uint32),
        ("merge_iters", ctypes.c_uint64), ("lane_iters", ctypes.c_uint64), ("merge_chunks", ctypes.c_uint64),
    ]


class _GraphView(ctypes.Structure):
    _fields_ = [
        ("offsets", ctypes.c_void_p), ("n_plus_1", ctypes.c_uint64),
        ("neighbours", ctypes.c_void_p), ("width", ctypes.c_uint64),
        ("neighbour_bits", ctypes.c_uint32), ("reserved", ctypes.c_uint32),
        ("truss_out", ctypes.c_void_p),
    ]


class _Tuning(ctypes.Structure):
    _fields_ = [(name, ctypes.c_uint32) for name in
                ("struct_size", "merge_ratio", "hub_min_degree", "sample_min", "support_kernel", "compact_pct",
                 "hash_min_degree", "sup_hash_min", "relabel")]


EXPORTS = [
    "sparx_pkt_default_opts", "sparx_strerror", "sparx_last_error", "sparx_pkt_run",
    "sparx_pkt_run_u32", "sparx_pkt_run_device", "sparx_triangles_run", "sparx_clustering_run",
    "sparx_kcore_run",
    "sparx_pkt_run_batch",
    "sparx_pkt_run_device_noalloc",
    "sparx_server_create", "sparx_server_submit", "sparx_server_poll", "sparx_server_wait",
    "sparx_server_cancel", "sparx_server_destroy",
]


def lib():
    L = load_library("libsparx_pkt.so")
    if getattr(L, "_sparx_typed", False):
        return L
    vp, u64, i32 = ctypes.c_void_p, ctypes.c_uint64, ctypes.c_int
    P = ctypes.POINTER
    L.sparx_pkt_default_opts.restype = i32
    L.sparx_pkt_default_opts.argtypes = [P(_Opts)]
    L.sparx_strerror.restype = ctypes.c_char_p
    L.sparx_strerror.argtypes = [i32]
    L.sparx_last_error.restype = ctypes.c_char_p
    L.sparx_last_error.argtypes = []
    for name in ("sparx_pkt_run", "sparx_pkt_run_u32", "sparx_triangles_run"):
        f = getattr(L, name)
        f.restype = i32
        f.argtypes = [vp, u64, vp, u64, vp, P(_Opts), P(_Stats)]
    L.sparx_kcore_run.restype = i32
    L.sparx_kcore_run.argtypes = [vp, u64, vp, u64, vp, P(_Opts), P(_Stats)]
    L.sparx_clustering_run.restype = i32
    L.sparx_clustering_run.argtypes = [vp, u64, vp, u64, vp, P(ctypes.c_double), P(ctypes.c_double),
                                       P(_Opts), P(_Stats)]
    L.sparx_pkt_run_device.restype = i32
    L.sparx_pkt_run_device.argtypes = [vp, u64, vp, u64, vp, P(_Opts), P(_Stats), vp]
    if hasattr(L, "sparx_pkt_run_device_noalloc"):
        L.sparx_pkt_run_device_noalloc.restype = i32
        L.sparx_pkt_run_device_noalloc.argtypes = [vp, u64, vp, u64, vp, ctypes.c_int, vp]
    if hasattr(L, "sparx_pkt_run_batch"):
        L.sparx_pkt_run_batch.restype = i32
        L.sparx_pkt_run_batch.argtypes = [P(_GraphView), u64, u64, P(_Opts), P(ctypes.c_int), P(_Stats)]
    L.sparx_mtx_to_csr.restype = i32
    L.sparx_mtx_to_csr.argtypes = [ctypes.c_char_p, u64, vp, u64, vp, u64, P(u64), P(u64), P(_Opts)]
    key3 = P(ctypes.c_uint32)
    for name, args in (("sparx_tuning_default", [P(_Tuning)]),
                       ("sparx_tuning_signature", [vp, u64, key3]),
                       ("sparx_tuning_lookup", [key3, P(_Tuning), P(ctypes.c_int)]),
                       ("sparx_tuning_store", [key3, P(_Tuning)]),
                       ("sparx_tuning_clear", []),
                       ("sparx_tuning_last", [P(_Tuning), key3]),
                       ("sparx_tuning_save", [ctypes.c_char_p]),
                       ("sparx_tuning_load", [ctypes.c_char_p]),
                       ("sparx_autotune", [vp, u64, vp, u64, P(_Opts), ctypes.c_uint32, P(_Tuning), key3]),
                       ("sparx_autotune_batch", [P(_GraphView), u64, u64, P(_Opts), ctypes.c_uint32, P(_Tuning),
                                                 key3])):
        f = getattr(L, name)
        f.restype = i32
        f.argtypes = args
    L._sparx_typed = True
    return L


class PktError(RuntimeError):
    def __init__(self, status: int, detail: str = ""):
        self.status = status
        msg = lib().sparx_strerror(status).decode()
        super().__init__(f"{msg} (status {status})" + (f": {detail}" if detail else ""))


@dataclasses.dataclass
class PktOptions:
    support_mode: int = SUPPORT_WIDE   # SUPPORT_U8 reproduces the reference's u8 counters
    out_bits: int = 8                  # 8: reference layout (u8 per slot); 32: u32
    device: int = -1
    loop: int = LOOP_GRAPH
    support_kernel: int = 0
    timeout_ms: int = 0

    def c(self) -> _Opts:
        o = _Opts()
        lib().sparx_pkt_default_opts(ctypes.byref(o))
        o.support_mode = self.support_mode
        o.out_bits = self.out_bits
        o.device = self.device
        o.loop = self.loop
        o.support_kernel = self.support_kernel
        if self.timeout_ms:
            o.timeout_ms = self.timeout_ms
        return o


@dataclasses.dataclass
class PktStats:
    n: int = 0
    width: int = 0
    m: int = 0
    self_loops: int = 0
    triangles: int = 0
    max_support: int = 0
    k_max: int = 0
    levels: int = 0
    waves: int = 0
    launches: int = 0
    ms_upload: float = 0.0
    ms_orient: float = 0.0
    ms_support: float = 0.0
    ms_peel: float = 0.0
    ms_finalize: float = 0.0
    ms_download: float = 0.0
    ms_total: float = 0.0
    support_elements: int = 0
    peel_elements: int = 0
    peel_hits: int = 0
    peel_scanned: int = 0
    peel_edges: int = 0
    compactions: int = 0
    hub_maps: int = 0
    merge_iters: int = 0
    lane_iters: int = 0
    merge_chunks: int = 0

    @classmethod
    def from_c(cls, s: _Stats) -> "PktStats":
        return cls(**{f.name: getattr(s, f.name) for f in dataclasses.fields(cls)})


def _check(rc: int):
    if rc != OK:
        raise PktError(rc, lib().sparx_last_error().decode())


def _arrays(g: GraphMemoryMap):
    off = np.ascontiguousarray(g.offsets(), dtype=np.uint64)
    nbr = np.ascontiguousarray(g.neighbours())
    return off, nbr


def run_pkt(offsets: np.ndarray, neighbours: np.ndarray, opts: PktOptions | None = None):
    """Truss per CSR slot (u8 or u32 per ``opts.out_bits``) and stats."""
    opts = opts or PktOptions()
    off = np.ascontiguousarray(offsets, dtype=np.uint64)
    nbr = np.ascontiguousarray(neighbours)
    out = np.empty(nbr.shape[0], dtype=np.uint8 if opts.out_bits == 8 else np.uint32)
    st = _Stats()
    o = opts.c()
    L = lib()
    if nbr.dtype == np.uint64:
        rc = L.sparx_pkt_run(off.ctypes.data, off.shape[0], nbr.ctypes.data, nbr.shape[0],
                             out.ctypes.data, ctypes.byref(o), ctypes.byref(st))
    elif nbr.dtype == np.uint32:
        rc = L.sparx_pkt_run_u32(off.ctypes.data, off.shape[0], nbr.ctypes.data, nbr.shape[0],
                                 out.ctypes.data, ctypes.byref(o), ctypes.byref(st))
    else:
        raise TypeError("neighbours must be u64 or u32")
    _check(rc)
    return out, PktStats.from_c(st)


def run_triangles(offsets: np.ndarray, neighbours: np.ndarray, opts: PktOptions | None = None):
    """Triangle support per CSR slot (u32), as ``Triangles::new`` computes it."""
    opts = opts or PktOptions()
    off = np.ascontiguousarray(offsets, dtype=np.uint64)
    nbr = np.ascontiguousarray(neighbours, dtype=np.uint64)
    out = np.empty(nbr.shape[0], dtype=np.uint32)
    st = _Stats()
    o = opts.c()
    _check(lib().sparx_triangles_run(off.ctypes.data, off.shape[0], nbr.ctypes.data, nbr.shape[0],
                                     out.ctypes.data, ctypes.byref(o), ctypes.byref(st)))
    return out, PktStats.from_c(st)


def run_clustering(offsets: np.ndarray, neighbours: np.ndarray, opts: PktOptions | None = None):
    """Local clustering coefficient per vertex (f64), transitivity, average and stats, as
    ``ClusteringCoefficient::new`` computes them (clustering_coefficient.rs:41-52,93-190)."""
    opts = opts or PktOptions()
    off = np.ascontiguousarray(offsets, dtype=np.uint64)
    nbr = np.ascontiguousarray(neighbours, dtype=np.uint64)
    local = np.empty(max(off.shape[0] - 1, 0), dtype=np.float64)
    trans, avg = ctypes.c_double(), ctypes.c_double()
    st = _Stats()
    o = opts.c()
    _check(lib().sparx_clustering_run(off.ctypes.data, off.shape[0], nbr.ctypes.data, nbr.shape[0],
                                      local.ctypes.data, ctypes.byref(trans), ctypes.byref(avg),
                                      ctypes.byref(o), ctypes.byref(st)))
    return local, trans.value, avg.value, PktStats.from_c(st)


def run_kcore(offsets: np.ndarray, neighbours: np.ndarray, opts: PktOptions | None = None):
    """Core number per vertex (u8 or u32 per ``opts.out_bits``) and stats, as
    ``AlgoLiuEtAl::new`` computes them (k_core/liu_et_al.rs:45-62,190-420)."""
    opts = opts or PktOptions()
    off = np.ascontiguousarray(offsets, dtype=np.uint64)
    nbr = np.ascontiguousarray(neighbours, dtype=np.uint64)
    out = np.empty(max(off.shape[0] - 1, 0), dtype=np.uint8 if opts.out_bits == 8 else np.uint32)
    st = _Stats()
    o = opts.c()
    _check(lib().sparx_kcore_run(off.ctypes.data, off.shape[0], nbr.ctypes.data, nbr.shape[0],
                                 out.ctypes.data, ctypes.byref(o), ctypes.byref(st)))
    return out, PktStats.from_c(st)


def _cache_file(g: GraphMemoryMap, kind: str) -> str:
    os.makedirs(CACHE_DIR, exist_ok=True)
    return os.path.join(CACHE_DIR, f"{kind}_{g.graph_id()}.mmap")


class AlgoPKT:
    """PKT k-truss decomposition of a ``GraphMemoryMap`` (pkt.rs:29-35)."""

    def __init__(self, g: GraphMemoryMap, k_trusses: np.ndarray, threads: int,
                 stats: PktStats | None = None):
        self.g = g
        self._k_trusses = k_trusses
        self.threads = threads
        self.stats = stats

    @classmethod
    def new(cls, g: GraphMemoryMap, opts: PktOptions | None = None) -> "AlgoPKT":
        return cls.new_with_conf(g, g.thread_num(), opts)

    @classmethod
    def new_with_conf(cls, g: GraphMemoryMap, threads: int,
                      opts: PktOptions | None = None) -> "AlgoPKT":
        opts = opts or PktOptions()
        off, nbr = _arrays(g)
        truss, stats = run_pkt(off, nbr, opts)
        if opts.out_bits == 8:
            path = _cache_file(g, "ktrusspkt")
            mm = np.memmap(path, dtype=np.uint8, mode="w+", shape=(max(1, truss.shape[0]),))
            mm[: truss.shape[0]] = truss
            mm.flush()
        return cls(g, truss, max(1, int(threads)), stats)

    _cache_kind = "ktrusspkt"

    @classmethod
    def get_or_compute(cls, g: GraphMemoryMap, opts: PktOptions | None = None) -> "AlgoPKT":
        path = _cache_file(g, cls._cache_kind)
        if os.path.exists(path):
            mm = np.memmap(path, dtype=np.uint8, mode="r")
            if mm.shape[0] >= g.width():
                return cls(g, np.asarray(mm[: g.width()]), g.thread_num())
        return cls.new(g, opts)

    def trussness(self, e_idx: int) -> int:
        assert e_idx < self.g.width()
        return int(self._k_trusses[e_idx])

    def k_trusses(self) -> np.ndarray:
        return self._k_trusses

    def drop_cache(self) -> None:
        path = _cache_file(self.g, self._cache_kind)
        os.remove(path)

    def get_throughput_factor(self) -> int:
        """pkt.rs:176-178: the bench divides by the CSR width."""
        return self.g.width()


class AlgoBurkhardtEtAl(AlgoPKT):
    """k-truss decomposition with the API of ``AlgoBurkhardtEtAl`` (burkhardt_et_al.rs:28-98), the
    reference's default ``GraphMemoryMap::k_truss`` (graph/impl_algos.rs:29-36).

    The truss decomposition is unique, so the result is the one the PKT engine computes; with
    wide (default) support it equals the reference Burkhardt peel's.  In ``SUPPORT_U8`` mode the
    engine follows the reference PKT's wrapped-count semantics, which differ from its Burkhardt
    peel's (a count that wraps to zero removes the edge there)."""

    _cache_kind = "ktrussbea"

    @classmethod
    def new_with_conf(cls, g: GraphMemoryMap, threads: int,
                      opts: PktOptions | None = None) -> "AlgoBurkhardtEtAl":
        opts = opts or PktOptions()
        off, nbr = _arrays(g)
        truss, stats = run_pkt(off, nbr, opts)
        if opts.out_bits == 8:
            path = _cache_file(g, cls._cache_kind)
            mm = np.memmap(path, dtype=np.uint8, mode="w+", shape=(max(1, truss.shape[0]),))
            mm[: truss.shape[0]] = truss
            mm.flush()
        return cls(g, truss, max(1, int(threads)), stats)


class AlgoLiuEtAl:
    """k-core decomposition of a ``GraphMemoryMap`` with the API of ``AlgoLiuEtAl``
    (k_core/liu_et_al.rs:24-188): one core number per vertex, u8 in the reference's layout."""

    _cache_kind = "kcorelea"

    def __init__(self, g: GraphMemoryMap, k_cores: np.ndarray, threads: int,
                 stats: PktStats | None = None):
        self.g = g
        self._k_cores = k_cores
        self.threads = threads
        self.stats = stats

    @classmethod
    def new(cls, g: GraphMemoryMap, opts: PktOptions | None = None) -> "AlgoLiuEtAl":
        return cls.new_with_conf(g, g.thread_num(), opts)

    @classmethod
    def new_with_conf(cls, g: GraphMemoryMap, threads: int,
                      opts: PktOptions | None = None) -> "AlgoLiuEtAl":
        opts = opts or PktOptions()
        off, nbr = _arrays(g)
        cores, stats = run_kcore(off, nbr, opts)
        if opts.out_bits == 8:
            path = _cache_file(g, cls._cache_kind)
            mm = np.memmap(path, dtype=np.uint8, mode="w+", shape=(max(1, cores.shape[0]),))
            mm[: cores.shape[0]] = cores
            mm.flush()
        return cls(g, cores, max(1, int(threads)), stats)

    @classmethod
    def get_or_compute(cls, g: GraphMemoryMap, opts: PktOptions | None = None) -> "AlgoLiuEtAl":
        path = _cache_file(g, cls._cache_kind)
        if os.path.exists(path):
            mm = np.memmap(path, dtype=np.uint8, mode="r")
            if mm.shape[0] >= g.size():
                return cls(g, np.asarray(mm[: g.size()]), g.thread_num())
        return cls.new(g, opts)

    def coreness(self, node: int) -> int:
        assert node < self.g.size()
        return int(self._k_cores[node])

    def k_cores(self) -> np.ndarray:
        return self._k_cores

    def drop_cache(self) -> None:
        os.remove(_cache_file(self.g, self._cache_kind))

    def get_throughput_factor(self) -> int:
        """liu_et_al.rs:186-188: the bench divides by the CSR width."""
        return self.g.width()


class ClusteringCoefficient:
    """Local clustering coefficients, transitivity and their average for a ``GraphMemoryMap``
    (clustering_coefficient.rs:17-79), computed on the GPU from the triangle supports."""

    def __init__(self, g: GraphMemoryMap, local: np.ndarray, transitivity: float, average: float,
                 stats: PktStats):
        self.g = g
        self._local = local
        self._transitivity = transitivity
        self._average = average
        self.stats = stats

    @classmethod
    def new(cls, g: GraphMemoryMap, opts: PktOptions | None = None) -> "ClusteringCoefficient":
        off, nbr = _arrays(g)
        local, trans, avg, stats = run_clustering(off, nbr, opts)
        return cls(g, local, trans, avg, stats)

    def get_average_clustering_coefficient(self) -> float:
        return self._average

    def get_node_clusteringcoefficient(self, node_id: int) -> float:
        assert node_id < self.g.size(), "id < |V| --- not met"
        return float(self._local[node_id])

    def get_graph_transitivity(self) -> float:
        return self._transitivity

    def local_coefficients(self) -> np.ndarray:
        return self._local


class Triangles:
    """Per-slot triangle support of a ``GraphMemoryMap`` (triangles.rs:16-69)."""

    def __init__(self, g: GraphMemoryMap, support: np.ndarray, stats: PktStats):
        self.g = g
        self._support = support
        self.stats = stats

    @classmethod
    def new(cls, g: GraphMemoryMap, opts: PktOptions | None = None) -> "Triangles":
        off, nbr = _arrays(g)
        sup, stats = run_triangles(off, nbr, opts)
        return cls(g, sup, stats)

    def triangles(self, e_idx: int) -> int:
        assert e_idx < self.g.width()
        return int(self._support[e_idx])

    def all_triangles(self) -> np.ndarray:
        return self._support


def run_pkt_device(d_offsets: int, n_plus_1: int, d_neighbours: int, width: int, d_out: int,
                   opts: PktOptions | None = None, stream: int = 0) -> PktStats:
    """Device-resident run: raw device pointers (u64 offsets, u32 ids, output per
    ``opts.out_bits``) on ``stream`` (a cudaStream_t as int, 0 = library stream)."""
    opts = opts or PktOptions()
    st = _Stats()
    o = opts.c()
    _check(lib().sparx_pkt_run_device(d_offsets, n_plus_1, d_neighbours, width, d_out,
                                      ctypes.byref(o), ctypes.byref(st), stream or None))
    return PktStats.from_c(st)


def run_batch(graphs, opts: PktOptions | None = None, hbm_budget_bytes: int = 0):
    """Decompose many independent graphs with ``sparx_pkt_run_batch``.

    ``graphs``: sequence of (offsets u64[n+1], neighbours u64|u32[width]).
    Returns a list of (truss, PktStats, status) in input order; a failing graph
    gets ``truss=None`` and its status (the others still complete)."""
    opts = opts or PktOptions()
    views = (_GraphView * max(1, len(graphs)))()
    keep, outs = [], []
    for i, (off, nbr) in enumerate(graphs):
        off = np.ascontiguousarray(off, dtype=np.uint64)
        nbr = np.ascontiguousarray(nbr)
        if nbr.dtype not in (np.uint64, np.uint32):
            nbr = nbr.astype(np.uint64)
        out = np.empty(nbr.shape[0], dtype=np.uint8 if opts.out_bits == 8 else np.uint32)
        keep += [off, nbr]
        outs.append(out)
        v = views[i]
        v.offsets = off.ctypes.data
        v.n_plus_1 = off.shape[0]
        v.neighbours = nbr.ctypes.data
        v.width = nbr.shape[0]
        v.neighbour_bits = 64 if nbr.dtype == np.uint64 else 32
        v.truss_out = out.ctypes.data
    n = len(graphs)
    status = (ctypes.c_int * max(1, n))()
    stats = (_Stats * max(1, n))()
    o = opts.c()
    lib().sparx_pkt_run_batch(views, n, hbm_budget_bytes, ctypes.byref(o), status, stats)
    return [(outs[i] if status[i] == OK else None, PktStats.from_c(stats[i]), int(status[i])) for i in range(n)]


def run_pkt_device_noalloc(d_offsets: int, n_plus_1: int, d_neighbours: int, width: int, d_out: int,
                           device: int = -1, stream: int = 0) -> None:
    """Allocation-free variant (``sparx_pkt_run_device_noalloc``): u32 truss per
    slot into ``d_out``; scratch is the library's fixed per-device array, so the
    graph must fit it and calls must not overlap on the GPU."""
    _check(lib().sparx_pkt_run_device_noalloc(d_offsets, n_plus_1, d_neighbours, width, d_out, device,
                                              stream or None))


# ---- tuning ----------------------------------------------------------------------------------

@dataclasses.dataclass(frozen=True)
class PktTuning:
    """The engine's performance knobs (``sparx_tuning``); none changes a result."""
    merge_ratio: int = 8
    hub_min_degree: int = 1024
    sample_min: int = 64
    support_kernel: int = 1
    compact_pct: int = 85
    hash_min_degree: int = 128
    sup_hash_min: int = 0
    relabel: int = 0

    def c(self) -> _Tuning:
        t = _Tuning()
        t.struct_size = ctypes.sizeof(_Tuning)
        for f in dataclasses.fields(self):
            setattr(t, f.name, getattr(self, f.name))
        return t

    @classmethod
    def from_c(cls, t: _Tuning) -> "PktTuning":
        return cls(**{f.name: getattr(t, f.name) for f in dataclasses.fields(cls)})


def _key(key):
    return (ctypes.c_uint32 * 3)(*key)


def tuning_signature(offsets) -> tuple:
    """Degree signature (log2 slots, log2 bucket of the max degree, eighths of slots in rows of
    degree >= 256) under which tuned knobs are cached."""
    off = np.ascontiguousarray(offsets, dtype=np.uint64)
    k = (ctypes.c_uint32 * 3)()
    _check(lib().sparx_tuning_signature(off.ctypes.data, off.shape[0], k))
    return tuple(k)


def tuning_lookup(key) -> tuple[PktTuning, bool]:
    t, found = _Tuning(), ctypes.c_int()
    _check(lib().sparx_tuning_lookup(_key(key), ctypes.byref(t), ctypes.byref(found)))
    return PktTuning.from_c(t), bool(found.value)


def tuning_store(key, tuning: PktTuning) -> None:
    t = tuning.c()
    _check(lib().sparx_tuning_store(_key(key), ctypes.byref(t)))


def tuning_clear() -> None:
    _check(lib().sparx_tuning_clear())


def tuning_last() -> tuple[PktTuning, tuple]:
    """Knobs and key the last launch on this thread used."""
    t, k = _Tuning(), (ctypes.c_uint32 * 3)()
    _check(lib().sparx_tuning_last(ctypes.byref(t), k))
    return PktTuning.from_c(t), tuple(k)


def tuning_save(path: str) -> None:
    _check(lib().sparx_tuning_save(path.encode()))


def tuning_load(path: str) -> None:
    _check(lib().sparx_tuning_load(path.encode()))


def autotune(offsets, neighbours, opts: PktOptions | None = None, repeats: int = 3) -> tuple[PktTuning, tuple]:
    """Measure candidate knobs on one sample graph and cache the best under its key."""
    opts = opts or PktOptions(out_bits=32)
    off = np.ascontiguousarray(offsets, dtype=np.uint64)
    nbr = np.ascontiguousarray(neighbours, dtype=np.uint64)
    t, k = _Tuning(), (ctypes.c_uint32 * 3)()
    o = opts.c()
    _check(lib().sparx_autotune(off.ctypes.data, off.shape[0], nbr.ctypes.data, nbr.shape[0], ctypes.byref(o),
                                repeats, ctypes.byref(t), k))
    return PktTuning.from_c(t), tuple(k)


def autotune_batch(graphs, opts: PktOptions | None = None, repeats: int = 3,
                   hbm_budget_bytes: int = 0) -> tuple[PktTuning, tuple]:
    """Autotune on a batch sample (timed on its first union, whose key gets the winner)."""
    opts = opts or PktOptions(out_bits=32)
    views = (_GraphView * len(graphs))()
    keep = []
    for i, (off, nbr) in enumerate(graphs):
        off = np.ascontiguousarray(off, dtype=np.uint64)
        nbr = np.ascontiguousarray(nbr)
        if nbr.dtype not in (np.uint64, np.uint32):
            nbr = nbr.astype(np.uint64)
        out = np.empty(nbr.shape[0], dtype=np.uint8 if opts.out_bits == 8 else np.uint32)
        keep += [off, nbr, out]
        v = views[i]
        v.offsets, v.n_plus_1 = off.ctypes.data, off.shape[0]
        v.neighbours, v.width = nbr.ctypes.data, nbr.shape[0]
        v.neighbour_bits = 64 if nbr.dtype == np.uint64 else 32
        v.truss_out = out.ctypes.data
    t, k = _Tuning(), (ctypes.c_uint32 * 3)()
    o = opts.c()
    _check(lib().sparx_autotune_batch(views, len(graphs), hbm_budget_bytes, ctypes.byref(o), repeats,
                                      ctypes.byref(t), k))
    return PktTuning.from_c(t), tuple(k)


# ---- input ------------------------------------------------------------------------------------

def mtx_to_csr(data: bytes, device: int = -1):
    """MatrixMarket text -> (offsets u64[n+1], neighbours u64[width]) on the GPU, with the
    semantics of ``GraphCache::from_mtx_file`` (parser_mtx/mod.rs:34-162, producers.rs:139-240,
    impl_sort.rs:10-51): entries mirrored unless the header says ``general``, duplicates kept,
    rows sorted.  Raises PktError(E_PARSE) on malformed text."""
    L = lib()
    o = PktOptions(device=device).c()
    n, w = ctypes.c_uint64(), ctypes.c_uint64()
    _check(L.sparx_mtx_to_csr(data, len(data), None, 0, None, 0, ctypes.byref(n), ctypes.byref(w), ctypes.byref(o)))
    off = np.empty(n.value + 1, dtype=np.uint64)
    nbr = np.empty(max(w.value, 1), dtype=np.uint64)
    _check(L.sparx_mtx_to_csr(data, len(data), off.ctypes.data, off.shape[0], nbr.ctypes.data, nbr.shape[0],
                              ctypes.byref(n), ctypes.byref(w), ctypes.byref(o)))
    return off, nbr[: w.value]
