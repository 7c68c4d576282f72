"""Continuous-batching PKT service (``sparx_server_*``).

Requests are decompositions of independent graphs submitted at any time.  The
engine runs them on execution lanes (4; SPARX_SERVE_LANES overrides), each on
its own stream: an idle lane packs the queued requests that fit its share of
the HBM budget into one concatenated CSR with room to spare and runs it;
requests that arrive while it runs join it at the next wave boundary, and every
member's result is returned as soon as its own peel ends.  Each request's
result is the same as a solo decomposition of its graph.
"""
from __future__ import annotations

import ctypes
import dataclasses

import numpy as np

from . import pkt as P


def _lib():
    L = P.lib()
    if not getattr(L, "_sparx_server_typed", False):
        vp, u64, i32 = ctypes.c_void_p, ctypes.c_uint64, ctypes.c_int
        L.sparx_server_create.restype = i32
        L.sparx_server_create.argtypes = [ctypes.POINTER(vp), u64, ctypes.POINTER(P._Opts)]
        L.sparx_server_submit.restype = i32
        L.sparx_server_submit.argtypes = [vp, ctypes.POINTER(P._GraphView), ctypes.POINTER(u64)]
        L.sparx_server_poll.restype = i32
        L.sparx_server_poll.argtypes = [vp, u64, ctypes.POINTER(i32), ctypes.POINTER(i32),
                                        ctypes.POINTER(P._Stats)]
        L.sparx_server_wait.restype = i32
        L.sparx_server_wait.argtypes = [vp, u64, u64, ctypes.POINTER(i32), ctypes.POINTER(P._Stats)]
        L.sparx_server_cancel.restype = i32
        L.sparx_server_cancel.argtypes = [vp, u64]
        L.sparx_server_destroy.restype = i32
        L.sparx_server_destroy.argtypes = [vp]
        L.sparx_server_info.restype = i32
        L.sparx_server_info.argtypes = [vp, ctypes.POINTER(u64), ctypes.POINTER(u64)]
        L._sparx_server_typed = True
    return L


@dataclasses.dataclass
class Result:
    ticket: int
    status: int
    truss: np.ndarray | None
    stats: P.PktStats
    latency_ms: float


class PktServer:
    """``with PktServer(budget) as srv: t = srv.submit(off, nbr); r = srv.wait(t)``"""

    def __init__(self, hbm_budget_bytes: int = 0, opts: P.PktOptions | None = None):
        self.opts = opts or P.PktOptions(out_bits=32)
        self._h = ctypes.c_void_p()
        o = self.opts.c()
        rc = _lib().sparx_server_create(ctypes.byref(self._h), hbm_budget_bytes, ctypes.byref(o))
        P._check(rc)
        self._pending: dict[int, tuple] = {}

    def submit(self, offsets: np.ndarray, neighbours: np.ndarray) -> int:
        off = np.ascontiguousarray(offsets, dtype=np.uint64)
        nbr = np.ascontiguousarray(neighbours)
        if nbr.dtype not in (np.uint64, np.uint32):
            nbr = nbr.astype(np.uint64)
        out = np.empty(nbr.shape[0], dtype=np.uint8 if self.opts.out_bits == 8 else np.uint32)
        v = P._GraphView()
        v.offsets = off.ctypes.data
        v.n_plus_1 = off.shape[0]
        v.neighbours = nbr.ctypes.data
        v.width = nbr.shape[0]
        v.neighbour_bits = 64 if nbr.dtype == np.uint64 else 32
        v.truss_out = out.ctypes.data
        t = ctypes.c_uint64()
        P._check(_lib().sparx_server_submit(self._h, ctypes.byref(v), ctypes.byref(t)))
        self._pending[t.value] = (off, nbr, out)  # the engine reads/writes these until done
        return t.value

    def _result(self, ticket: int, status: int, st: P._Stats) -> Result:
        arrays = self._pending.pop(ticket, None)
        stats = P.PktStats.from_c(st)
        truss = arrays[2] if (arrays is not None and status == P.OK) else None
        return Result(ticket, status, truss, stats, stats.ms_total)

    def poll(self, ticket: int) -> Result | None:
        done, status, st = ctypes.c_int(), ctypes.c_int(), P._Stats()
        P._check(_lib().sparx_server_poll(self._h, ticket, ctypes.byref(done), ctypes.byref(status),
                                          ctypes.byref(st)))
        return self._result(ticket, status.value, st) if done.value else None

    def wait(self, ticket: int, timeout_ms: int = 0) -> Result:
        status, st = ctypes.c_int(), P._Stats()
        P._check(_lib().sparx_server_wait(self._h, ticket, timeout_ms, ctypes.byref(status), ctypes.byref(st)))
        return self._result(ticket, status.value, st)

    def info(self) -> dict:
        """Served unions started, and requests that joined a union already running."""
        u, j = ctypes.c_uint64(), ctypes.c_uint64()
        P._check(_lib().sparx_server_info(self._h, ctypes.byref(u), ctypes.byref(j)))
        return {"unions": u.value, "joined": j.value}

    def cancel(self, ticket: int) -> bool:
        rc = _lib().sparx_server_cancel(self._h, ticket)
        return rc == P.OK

    def close(self) -> None:
        if self._h:
            _lib().sparx_server_destroy(self._h)
            self._h = ctypes.c_void_p()
            self._pending.clear()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
