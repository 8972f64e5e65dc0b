"""The C-ABI library loads and exports every entry point declared in include/lpcuda.h
(no GPU needed: nothing is called)."""
import ctypes
import os
import re

import pytest

from lightpropagation_b200 import _native

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared(header):
    src = open(os.path.join(ROOT, "include", header)).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(lp_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_declared_symbols():
    if not os.path.isfile(_native.LIB_PATH):
        pytest.fail("liblpcuda.so not built (run lightpropagation_b200.build.build())")
    lib = ctypes.CDLL(_native.LIB_PATH)
    names = declared("lpcuda.h")
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # the Python bindings cover every declared entry point
    assert set(names) <= set(_native.EXPORTED), set(names) - set(_native.EXPORTED)


def test_errors_without_context_are_reported():
    L = _native.lib()
    rc = L.lp_set_media(None, 1, None)
    assert rc == 1
    assert b"ctx is NULL" in L.lp_last_error(None)
