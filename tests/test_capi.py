"""The C-ABI library: loads, exports every symbol include/trspmm.h declares,
and reports argument errors through status codes (no GPU needed)."""
import ctypes
import os
import re

import numpy as np
import pytest

import trspmm
from trspmm import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "trspmm.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(tr_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    L = ctypes.CDLL(_lib.LIB_PATH)
    names = declared_symbols()
    assert len(names) >= 15
    for n in names:
        assert hasattr(L, n), n
    assert set(names) == set(_lib.EXPORTED)


def test_library_loads_without_gpu():
    L = trspmm.lib()
    assert L.tr_version() >= 1


def test_status_codes_without_gpu():
    L = trspmm.lib()
    prm = _lib.RouteParams(32, 32, 3, 8, 0, 16, 0.0, 0.5, 12, 2, 0, 0, 0)   # window = 0
    indptr = np.zeros(2, np.int32)
    h = ctypes.c_void_p()
    rc = L.tr_route_build(indptr.ctypes.data, None, None, 1, ctypes.byref(prm), ctypes.byref(h))
    assert rc == _lib.TR_ERR_ARG
    assert b"window" in L.tr_last_error()
    rc = L.tr_spmm_routed(None, None, 8, None, 0, 7, None)
    assert rc == _lib.TR_ERR_ARG
    rc = L.tr_spmm_csr(None, None, None, -1, 0, 0, None, 8, None, 0, None)
    assert rc == _lib.TR_ERR_ARG


def test_python_error_is_runtime_error():
    with pytest.raises(RuntimeError):
        trspmm.route(np.array([0, 1], np.int32), np.array([0], np.int32), np.ones(1, np.float32),
                     window=64)
