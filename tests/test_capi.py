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


def test_new_entry_points_check_their_arguments_without_gpu():
    L = trspmm.lib()
    # FP32-feature route: null plan, negative K, bad output dtype
    assert L.tr_spmm_routed_f32(None, None, 8, None, 0, 7, None) == _lib.TR_ERR_ARG
    assert b"null plan" in L.tr_last_error()
    assert L.tr_adjoint_sddmm_f32(None, None, None, 0, 0, None, None, 8, None, 0, None,
                                  None) == _lib.TR_ERR_ARG
    assert L.tr_sddmm_csr_f32(None, None, -1, 0, 0, None, None, 8, None, None) == _lib.TR_ERR_ARG
    assert b"negative size" in L.tr_last_error()
    assert L.tr_sddmm_csr_f32(None, None, 4, 4, 10, None, None, 8, None, None) == _lib.TR_ERR_ARG
    assert b"null device pointer" in L.tr_last_error()
    # TCA order: null arguments, malformed row pointers
    st = _lib.TcaStats()
    assert L.tr_tca_order(None, None, 3, None, None, ctypes.byref(st)) == _lib.TR_ERR_ARG
    ptr = np.array([1, 2], np.int32)
    idx = np.array([0, 0], np.int32)
    order = np.empty(1, np.int32)
    assert L.tr_tca_order(ptr.ctypes.data, idx.ctypes.data, 1, None, order.ctypes.data,
                          None) == _lib.TR_ERR_ARG
    assert b"indptr must start at 0" in L.tr_last_error()
    # LSH banding: thresholds outside (0, 1), permutation counts outside [1, 1024]
    b, r = ctypes.c_int32(), ctypes.c_int32()
    for t, n in ((0.0, 128), (1.0, 128), (0.5, 0), (0.5, 2048)):
        assert L.tr_lsh_params(t, n, ctypes.byref(b), ctypes.byref(r)) == _lib.TR_ERR_ARG
    assert L.tr_lsh_params(0.2, 128, ctypes.byref(b), ctypes.byref(r)) == _lib.TR_OK
    assert (b.value, r.value) == (28, 2)


def test_empty_tca_order_and_null_stats():
    L = trspmm.lib()
    ptr = np.zeros(1, np.int32)
    assert L.tr_tca_order(ptr.ctypes.data, None, 0, None, None, None) == _lib.TR_OK
