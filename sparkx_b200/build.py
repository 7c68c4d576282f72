"""Builds the in-tree native libraries.

* ``libsparx_pkt.so``      CUDA engine for sm_100a (nvcc -gencode arch=compute_100a,code=sm_100a)
* ``libsparx_graphgen.so`` host C++ workload generators (OpenMP)

Run ``python -m sparkx_b200.build``; outputs land next to this file so they
travel with the source tree.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC,-fopenmp", "-shared",
]


def _nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale(target: str, sources: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def _sources(exts) -> list[str]:
    out = []
    for root in (CSRC, INCLUDE):
        for f in os.listdir(root):
            if f.endswith(exts):
                out.append(os.path.join(root, f))
    return out


def build_engine(force: bool = False, verbose: bool = False) -> str:
    target = os.path.join(HERE, "libsparx_pkt.so")
    deps = _sources((".cu", ".cuh", ".h"))
    if force or _stale(target, deps):
        extra = os.environ.get("SPARX_NVCC_FLAGS", "").split()
        cmd = [_nvcc(), *NVCC_FLAGS, *extra, "-o", target, os.path.join(CSRC, "sparx_pkt.cu"), "-lgomp"]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        subprocess.run(cmd, check=True)
    return target


def build_graphgen(force: bool = False) -> str:
    target = os.path.join(HERE, "libsparx_graphgen.so")
    src = os.path.join(CSRC, "graphgen.cpp")
    if force or _stale(target, [src]):
        cxx = shutil.which("g++") or "g++"
        subprocess.run([cxx, "-O2", "-std=c++17", "-fPIC", "-fopenmp", "-shared", "-Wall",
                        "-o", target, src], check=True)
    return target


def build_all(force: bool = False, verbose: bool = False) -> None:
    build_graphgen(force)
    build_engine(force, verbose)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv, verbose="-v" in sys.argv)
