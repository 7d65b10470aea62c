"""trspmm — B200-native three-way routed FP16 SpMM (host side).

The compute lives in libtrspmm.so (CUDA for sm_100a, C ABI in
include/trspmm.h); this package binds it with ctypes and mirrors the
reference's Python-facing operators.  There is no CPU fallback: every entry
point that computes raises if the library or a CUDA device is missing.
"""
from ._lib import (TR_ENGINE_BLOCK, TR_ENGINE_WINDOW, TR_OUT_F16, TR_OUT_F32, TR_ROUTE_ALL,
                   TR_ROUTE_CUDA, TR_ROUTE_PER_WINDOW,
                   TR_ROUTE_PIPELINED, TR_ROUTE_RESIDUAL_PASS, TR_ROUTE_SPTC,
                   TR_ROUTE_TC, EXPORTED, LIB_PATH, TrError, lib)
from .core import (TABLE_NAMES, Plan, host_plan, match_2to4, route, route_device, route_tc_device, sddmm_csr,
                   spmm_csr, tables_struct)

__all__ = ["TR_ENGINE_BLOCK", "TR_ENGINE_WINDOW", "TR_OUT_F16", "TR_OUT_F32", "TR_ROUTE_ALL", "TR_ROUTE_CUDA", "TR_ROUTE_PER_WINDOW",
           "TR_ROUTE_PIPELINED", "TR_ROUTE_RESIDUAL_PASS", "TR_ROUTE_SPTC",
           "TR_ROUTE_TC", "EXPORTED", "LIB_PATH", "TrError", "lib", "TABLE_NAMES", "Plan",
           "route", "route_device", "route_tc_device", "spmm_csr", "sddmm_csr", "host_plan", "tables_struct",
           "match_2to4"]
