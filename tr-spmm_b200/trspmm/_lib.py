"""ctypes binding of libtrspmm.so (the C ABI in include/trspmm.h).

The library is built in-tree (``make -C tr-spmm_b200/csrc``) and loaded from
this directory; there is no fallback: a missing or stale library raises.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libtrspmm.so")

TR_OK, TR_ERR_ARG, TR_ERR_CUDA, TR_ERR_TIMEOUT, TR_ERR_NOMEM, TR_ERR_UNSUPPORTED = range(6)
TR_OUT_F32, TR_OUT_F16 = 0, 1
TR_ROUTE_TC, TR_ROUTE_SPTC, TR_ROUTE_CUDA, TR_ROUTE_ALL = 1, 2, 4, 7
TR_ROUTE_PER_WINDOW, TR_ROUTE_PIPELINED, TR_ROUTE_RESIDUAL_PASS = 8, 16, 32
TR_ROUTE_COMPAT, TR_ROUTE_EXACT = 0, 1

# Every symbol declared in include/trspmm.h.
EXPORTED = [
    "tr_last_error", "tr_version", "tr_device_info",
    "tr_route_build", "tr_route_device", "tr_route_table_device", "tr_route_tc_device", "tr_route_tc_device_noalloc", "tr_route_table",
    "tr_route_seconds", "tr_route_free", "tr_match_2to4", "tr_match_2to4_online",
    "tr_plan_from_tables", "tr_plan_from_csr", "tr_plan_build", "tr_plan_build_host",
    "tr_host_plan_array", "tr_host_plan_upload", "tr_host_plan_free", "tr_host_plan_save",
    "tr_host_plan_load", "tr_plan_info_get",
    "tr_plan_free", "tr_spmm_csr", "tr_spmm_routed", "tr_plan_set_values", "tr_sddmm_csr",
    "tr_adjoint_sddmm",
    "tr_forward_fp16_tcu_cuda_sptc_mma_parallel_online", "tr_forward_fp16_sptc_online",
    "tr_forward_fp16_sptc_mma_online", "tr_forward_fp16_sptc_mma_packed_online",
    "tr_tca_order", "tr_lsh_params", "tr_label_order", "tr_spmm_routed_f32", "tr_sddmm_csr_f32",
    "tr_adjoint_sddmm_f32", "tr_plan_entry_order", "tr_plan_renumber_edges", "tr_plan_set_k_tile",
    "tr_plan_set_deterministic",
]


TR_MATCH_SLIDING, TR_MATCH_HASH, TR_MATCH_BUCKET, TR_MATCH_ONLINE = 0, 1, 2, 3


class MatchStats(ctypes.Structure):
    """tr_match_stats (include/trspmm.h)."""
    _fields_ = [("total_rows", ctypes.c_int32), ("total_cols", ctypes.c_int32),
                ("total_nnz", ctypes.c_int64), ("sparsity", ctypes.c_double),
                ("num_row_panels", ctypes.c_int32), ("reserved", ctypes.c_int32),
                ("num_groups", ctypes.c_int64), ("num_tc_blocks", ctypes.c_int64),
                ("num_16x16_blocks", ctypes.c_int64), ("block_padding_groups", ctypes.c_int64),
                ("fine_fallback", ctypes.c_int64), ("coarse_fallback", ctypes.c_int64),
                ("fake_zeros", ctypes.c_int64), ("dense_to_tc_cols", ctypes.c_int64),
                ("dense_to_sptc_cols", ctypes.c_int64)]


class TrError(RuntimeError):
    """A non-zero status from libtrspmm (raised as RuntimeError, like TORCH_CHECK)."""

    def __init__(self, code, msg):
        super().__init__(msg)
        self.code = code


class RouteParams(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int32) for n in ("partsize_t", "partsize_c", "shortsize", "density",
                                                 "window", "wide")] + [
        ("tc_min_util", ctypes.c_float), ("sptc_min_util", ctypes.c_float),
        ("sptc_threshold", ctypes.c_int32), ("unit_min_nnz", ctypes.c_int32),
        ("skip_tc", ctypes.c_int32), ("mode", ctypes.c_int32), ("threads", ctypes.c_int32),
        ("skip_sptc", ctypes.c_int32)]


class PlanInfo(ctypes.Structure):
    _fields_ = [("n_rows", ctypes.c_int32), ("n_cols", ctypes.c_int32),
                ("n_windows", ctypes.c_int32), ("nnz", ctypes.c_int64),
                ("tc_tiles", ctypes.c_int64), ("sptc_tiles", ctypes.c_int64),
                ("residual_nnz", ctypes.c_int64), ("device_bytes", ctypes.c_int64),
                ("promoted_tiles", ctypes.c_int64), ("row_scaled", ctypes.c_int32),
                ("reordered", ctypes.c_int32), ("engine", ctypes.c_int32),
                ("n_blocks", ctypes.c_int32), ("chunks", ctypes.c_int64),
                ("n_edges", ctypes.c_int64), ("slots", ctypes.c_int64)]


class PlanOpts(ctypes.Structure):
    _fields_ = [("row_scale", ctypes.c_int32), ("promote_min", ctypes.c_int32),
                ("transpose", ctypes.c_int32), ("reorder", ctypes.c_int32),
                ("demote_below", ctypes.c_int32), ("row_order", ctypes.c_void_p),
                ("engine", ctypes.c_int32)]


TR_REORDER_NONE, TR_REORDER_LABEL, TR_REORDER_TCA, TR_REORDER_GIVEN = 0, 1, 2, 3
TR_ENGINE_WINDOW, TR_ENGINE_BLOCK = 0, 1


class TcaParams(ctypes.Structure):
    """tr_tca_params (include/trspmm.h)."""
    _fields_ = [("thres", ctypes.c_int32), ("cluster_thres", ctypes.c_int32),
                ("lsh_threshold", ctypes.c_double), ("seed", ctypes.c_uint64),
                ("max_pairs", ctypes.c_int64), ("device", ctypes.c_int32)]


class TcaStats(ctypes.Structure):
    """tr_tca_stats (include/trspmm.h)."""
    _fields_ = [("bands", ctypes.c_int32), ("rows_per_band", ctypes.c_int32),
                ("pairs1", ctypes.c_int64), ("clusters1", ctypes.c_int64),
                ("pairs2", ctypes.c_int64), ("clusters2", ctypes.c_int64),
                ("seconds", ctypes.c_double * 4)]


_TABLE_FIELDS = ["t_row_offset", "t_block_offset", "t_column", "t_value", "t_window_row",
                 "t_binary", "c_row_offset", "c_row", "c_column", "c_value", "cs_row_offset",
                 "cs_row", "cs_column", "cs_value", "s_tile_column", "s_packed_a",
                 "s_packed_meta", "s_window_tile_offset"]


class Tables(ctypes.Structure):
    _fields_ = [f for name in _TABLE_FIELDS
                for f in ((name, ctypes.c_void_p), ("n_" + name, ctypes.c_int64))]


_lib = None


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"libtrspmm.so not built ({LIB_PATH}); run make -C tr-spmm_b200/csrc")
    L = ctypes.CDLL(LIB_PATH)
    P, I32, I64, F = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_float
    L.tr_last_error.restype = ctypes.c_char_p
    L.tr_version.restype = ctypes.c_int
    L.tr_device_info.argtypes = [P, P, P]
    L.tr_route_build.argtypes = [P, P, P, I32, ctypes.POINTER(RouteParams), P]
    L.tr_route_table.argtypes = [P, ctypes.c_int, ctypes.POINTER(P), ctypes.POINTER(I64)]
    L.tr_route_tc_device.argtypes = [P, P, P, I32, ctypes.POINTER(RouteParams), P]
    L.tr_route_device.argtypes = [P, P, P, I32, ctypes.POINTER(RouteParams), P]
    L.tr_route_table_device.argtypes = [P, ctypes.c_int, ctypes.POINTER(P), ctypes.POINTER(I64)]
    L.tr_route_tc_device_noalloc.argtypes = [P, P, P, I32, ctypes.POINTER(RouteParams), P, P, P, P,
                                             I64, I64, P, P, P]
    L.tr_match_2to4.argtypes = [P, P, I32, ctypes.c_int, I32, I32, I32, ctypes.POINTER(MatchStats)]
    L.tr_match_2to4_online.argtypes = [P, P, I32, I32, I32, I32, ctypes.POINTER(MatchStats)]
    L.tr_tca_order.argtypes = [P, P, I32, ctypes.POINTER(TcaParams), P, ctypes.POINTER(TcaStats)]
    L.tr_label_order.argtypes = [P, P, I32, I32, I32, P]
    L.tr_lsh_params.argtypes = [ctypes.c_double, I32, ctypes.POINTER(I32), ctypes.POINTER(I32)]
    L.tr_route_seconds.restype = ctypes.c_double
    L.tr_route_seconds.argtypes = [P]
    L.tr_route_free.argtypes = [P]
    L.tr_plan_from_tables.argtypes = [ctypes.POINTER(Tables), I32, I32, I32, P]
    L.tr_plan_from_csr.argtypes = [P, P, P, I32, I32, ctypes.POINTER(RouteParams), P]
    L.tr_plan_build.argtypes = [P, P, P, I32, I32, ctypes.POINTER(RouteParams),
                                ctypes.POINTER(PlanOpts), P]
    L.tr_plan_build_host.argtypes = [P, P, P, I32, I32, ctypes.POINTER(RouteParams),
                                     ctypes.POINTER(PlanOpts), P]
    L.tr_host_plan_array.argtypes = [P, ctypes.c_int, ctypes.POINTER(P), ctypes.POINTER(I64)]
    L.tr_host_plan_upload.argtypes = [P, P]
    L.tr_host_plan_free.argtypes = [P]
    L.tr_host_plan_save.argtypes = [P, ctypes.c_char_p]
    L.tr_host_plan_load.argtypes = [ctypes.c_char_p, ctypes.POINTER(P)]
    L.tr_plan_set_values.argtypes = [P, P, I64, P]
    L.tr_plan_entry_order.argtypes = [P, P, P]
    L.tr_plan_set_k_tile.argtypes = [P, I32]
    L.tr_plan_set_deterministic.argtypes = [P, I32]
    L.tr_plan_renumber_edges.argtypes = [P, P, I64, P]
    L.tr_sddmm_csr.argtypes = [P, P, I32, I32, I64, P, P, I32, P, P]
    L.tr_adjoint_sddmm.argtypes = [P, P, P, I32, I64, P, P, I32, P, ctypes.c_int, P, P]
    L.tr_plan_info_get.argtypes = [P, ctypes.POINTER(PlanInfo)]
    L.tr_plan_free.argtypes = [P]
    L.tr_spmm_csr.argtypes = [P, P, P, I32, I32, I64, P, I32, P, ctypes.c_int, P]
    L.tr_spmm_routed.argtypes = [P, P, I32, P, ctypes.c_int, ctypes.c_int, P]
    L.tr_spmm_routed_f32.argtypes = [P, P, I32, P, ctypes.c_int, ctypes.c_int, P]
    L.tr_sddmm_csr_f32.argtypes = [P, P, I32, I32, I64, P, P, I32, P, P]
    L.tr_adjoint_sddmm_f32.argtypes = [P, P, P, I32, I64, P, P, I32, P, ctypes.c_int, P, P]
    pairs29 = [P, I64] * 27 + [P, I64]
    L.tr_forward_fp16_tcu_cuda_sptc_mma_parallel_online.argtypes = (
        [P, I64] * 27 + [I32] * 9 + [P, P])
    L.tr_forward_fp16_sptc_online.argtypes = [P, I64] * 5 + [I32] * 5 + [P, P]
    L.tr_forward_fp16_sptc_mma_online.argtypes = [P, I64] * 5 + [I32] * 5 + [P, P]
    L.tr_forward_fp16_sptc_mma_packed_online.argtypes = [P, I64] * 5 + [I32] * 5 + [P, P]
    del pairs29
    for name in EXPORTED:
        if name not in ("tr_last_error", "tr_route_seconds"):
            getattr(L, name).restype = ctypes.c_int
    L.tr_plan_free.restype = None
    L.tr_host_plan_free.restype = None
    L.tr_route_free.restype = None
    _lib = L
    return L


def check(rc):
    if rc != TR_OK:
        msg = lib().tr_last_error().decode(errors="replace")
        raise TrError(rc, msg or f"libtrspmm error {rc}")
    return rc
