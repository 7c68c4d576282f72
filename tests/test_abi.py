"""The C ABI library builds, loads and exports every entry point that
include/sparx_pkt.h declares (no GPU needed: nothing here launches work)."""
import os
import re

import pytest

from sparkx_b200 import build, pkt

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared(header):
    text = open(os.path.join(ROOT, "include", header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(sparx_[a-z0-9_]+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib():
    build.build_engine()
    return pkt.lib()


def test_every_declared_symbol_is_exported(lib):
    names = declared("sparx_pkt.h")
    assert "sparx_pkt_run" in names and "sparx_pkt_run_device" in names
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_status_codes_and_defaults(lib):
    import ctypes
    text = open(os.path.join(ROOT, "include", "sparx_pkt.h")).read()
    codes = dict((k, int(v)) for k, v in re.findall(r"#define SPARX_(E_[A-Z_0-9]+|OK)\s+(\d+)", text))
    for k, v in codes.items():
        assert getattr(pkt, k) == v, k
        assert lib.sparx_strerror(v)
    o = pkt._Opts()
    assert lib.sparx_pkt_default_opts(ctypes.byref(o)) == 0
    assert o.struct_size == ctypes.sizeof(pkt._Opts) and o.out_bits == 8 and o.device == -1
    assert ctypes.sizeof(pkt._Stats) == 8 * 6 + 4 * 4 + 8 * 7 + 8 * 5 + 8 + 8 * 3


def test_sm100a_build_flags():
    assert "arch=compute_100a,code=sm_100a" in build.NVCC_FLAGS
