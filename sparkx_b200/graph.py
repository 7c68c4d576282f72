"""Host-side CSR graph in the reference's on-disk layout.

Mirrors the parts of ``GraphMemoryMap`` (``src/graph/mod.rs:365-378``) that the
PKT path reads: ``offsets_ptr``/``neighbours_ptr`` (``:482-489``) over a
memory-mapped offsets file (u64[n+1]) and neighbours file (u64[width]),
``size()``/``width()`` (``:648-658``) and ``thread_num()`` (``:493-495``).
The files are raw little-endian u64 arrays exactly as the reference's cache
writes them (``graph/cache/parser_mtx/mod.rs:96-155``), so a cache entry built
by the reference can be opened here unchanged.
"""
from __future__ import annotations

import hashlib
import os

import numpy as np


class GraphMemoryMap:
    """Memory-mapped symmetric CSR (offsets u64[n+1], neighbour ids u64 or u32)."""

    def __init__(self, offsets: np.ndarray, neighbours: np.ndarray, thread_count: int = 1,
                 graph_id: str | None = None, path_hint: str | None = None):
        if offsets.ndim != 1 or neighbours.ndim != 1:
            raise ValueError("offsets and neighbours must be 1-D")
        if offsets.dtype != np.uint64:
            raise ValueError("offsets must be u64 (the reference's usize layout)")
        if neighbours.dtype not in (np.uint64, np.uint32):
            raise ValueError("neighbours must be u64 (reference layout) or u32")
        if offsets.shape[0] < 1:
            raise ValueError("offsets needs n + 1 >= 1 entries")
        self._offsets = offsets
        self._neighbours = neighbours
        self._threads = max(1, min(int(thread_count), 255))
        self._id = graph_id
        self._path_hint = path_hint

    # -- construction -----------------------------------------------------
    @classmethod
    def from_arrays(cls, offsets, neighbours, thread_count: int = 1, graph_id: str | None = None):
        off = np.ascontiguousarray(offsets, dtype=np.uint64)
        nb = np.ascontiguousarray(neighbours)
        if nb.dtype not in (np.uint64, np.uint32):
            nb = nb.astype(np.uint64)
        return cls(off, nb, thread_count, graph_id)

    @classmethod
    def from_csr(cls, csr, thread_count: int = 1):
        return cls.from_arrays(csr.offsets, csr.neighbours, thread_count, csr.name or None)

    @classmethod
    def from_mtx_file(cls, path: str, thread_count: int = 1, device: int = -1):
        """Build the CSR from a MatrixMarket file on the GPU, as ``GraphCache::from_mtx_file``
        builds its cache (``graph/cache/parser_mtx/mod.rs:34-162``): see ``mtx_to_csr``."""
        from .pkt import mtx_to_csr
        with open(path, "rb") as f:
            data = f.read()
        off, nbr = mtx_to_csr(data, device=device)
        return cls(off, nbr, thread_count, os.path.basename(path), path)

    @classmethod
    def open(cls, offsets_path: str, neighbours_path: str, thread_count: int = 1):
        """Map an existing cache entry (raw u64 offsets file + raw u64 neighbours file)."""
        off = np.memmap(offsets_path, dtype=np.uint64, mode="r")
        nb = np.memmap(neighbours_path, dtype=np.uint64, mode="r")
        gid = os.path.basename(neighbours_path)
        return cls(off, nb, thread_count, gid, neighbours_path)

    def write_cache(self, offsets_path: str, neighbours_path: str) -> None:
        """Write the raw u64 files the reference memory-maps."""
        self._offsets.astype(np.uint64).tofile(offsets_path)
        self._neighbours.astype(np.uint64).tofile(neighbours_path)

    # -- accessors mirroring graph/mod.rs ---------------------------------
    def offsets(self) -> np.ndarray:
        return self._offsets

    def neighbours(self) -> np.ndarray:
        return self._neighbours

    def offsets_size(self) -> int:
        return int(self._offsets.shape[0])

    def size(self) -> int:
        return max(0, int(self._offsets.shape[0]) - 1)

    def width(self) -> int:
        return int(self._neighbours.shape[0])

    def thread_num(self) -> int:
        return self._threads

    def node_degree(self, u: int) -> int:
        if not 0 <= u < self.size():
            raise IndexError(u)
        return int(self._offsets[u + 1] - self._offsets[u])

    def index_node(self, u: int) -> range:
        if not 0 <= u < self.size():
            raise IndexError(u)
        return range(int(self._offsets[u]), int(self._offsets[u + 1]))

    def neighbour_ids(self, u: int) -> np.ndarray:
        r = self.index_node(u)
        return self._neighbours[r.start:r.stop]

    # algorithm facade (graph/impl_algos.rs:25-40): k_truss is Burkhardt et al.'s by default
    def k_truss(self):
        from .pkt import AlgoBurkhardtEtAl
        return AlgoBurkhardtEtAl.new(self)

    def k_truss_bea(self):
        from .pkt import AlgoBurkhardtEtAl
        return AlgoBurkhardtEtAl.new(self)

    def k_core_lea(self):
        from .pkt import AlgoLiuEtAl
        return AlgoLiuEtAl.new(self)

    def k_truss_pkt(self):
        from .pkt import AlgoPKT
        return AlgoPKT.new(self)

    def graph_id(self) -> str:
        """Stable id: the cache key the result file is named after."""
        if self._id is None:
            h = hashlib.sha256()
            h.update(np.ascontiguousarray(self._offsets).view(np.uint8))
            h.update(np.ascontiguousarray(self._neighbours.astype(np.uint64, copy=False)).view(np.uint8))
            self._id = h.hexdigest()[:24]
        return self._id
