"""CPU-side checks of the C ABI library: it loads without a GPU, exports every
symbol include/zyklop_b200.h declares, and reports errors as status codes."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "zyklop_b200.h")


def declared_symbols():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(zk_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    assert "zk_msm_g1" in syms and "zk_ntt" in syms and len(syms) >= 10


def test_library_exports_every_declared_symbol():
    from zyklop_b200 import _lib
    L = _lib.lib()
    missing = [s for s in declared_symbols() if not hasattr(L, s)]
    assert not missing, missing
    # every declared symbol has a ctypes signature in the binding
    assert not [s for s in declared_symbols() if s not in _lib.SIGNATURES]


def test_version_and_error_without_gpu():
    from zyklop_b200 import _lib
    L = _lib.lib()
    assert b"sm_100a" in L.zk_version()
    # a bad argument is rejected with a status code, not a crash
    rc = L.zk_msm_set_config(None, 3, 0, 32, 16, 16)
    assert rc != 0
    assert L.zk_last_error()
