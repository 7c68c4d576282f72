"""Locates and loads the in-tree native libraries.

The CUDA library is required: there is no CPU fallback for the k-truss path,
so a missing or unloadable ``libsparx_pkt.so`` raises instead of degrading.
"""
from __future__ import annotations

import ctypes
import os
import threading

_HERE = os.path.dirname(os.path.abspath(__file__))
_LOCK = threading.Lock()
_LOADED: dict[str, ctypes.CDLL] = {}


class NativeLibraryMissing(RuntimeError):
    pass


def library_path(name: str) -> str:
    """In-tree library; SPARX_LIB_DIR points at another build of the same sources."""
    return os.path.join(os.environ.get("SPARX_LIB_DIR", _HERE), name)


def load_library(name: str) -> ctypes.CDLL:
    with _LOCK:
        lib = _LOADED.get(name)
        if lib is not None:
            return lib
        path = library_path(name)
        if not os.path.exists(path):
            raise NativeLibraryMissing(
                f"{name} is not built ({path}); run __graft_entry__.build() or "
                f"python -m sparkx_b200.build")
        lib = ctypes.CDLL(path, mode=ctypes.RTLD_GLOBAL)
        _LOADED[name] = lib
        return lib
