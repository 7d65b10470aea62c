"""ORACLE — test infrastructure only.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg may
import this package, and only as the checker.  The shipped library never
imports it.

Contents
  route()            CPU restatement of the reference router
                     (TR-source/Block/block_online.cpp:545-871), via liboracle.so.
  ref_route()        the reference router itself, compiled from its source into
                     oracle/_ref (present only where it was built).
  ref_match()        the reference's matching-stats functions (matching_utils,
                     _hash, _bucket), compiled the same way.
  ref_sptc_online()  the reference's scalar 2:4 SpMM operator
                     (TR-source/SpMM/mGCN_online.cpp:202-400) compiled for
                     sm_100a into oracle/_ref; check_sptc_tables() its
                     host-side bounds checks.
  ref_parallel_cuda_route()  the reference's parallel operator on tables of
                     CUDA-route parts only (its TC and 2:4 kernels are not
                     launched then); check_cuda_route_tables() its checks.
  decode_tables()    rebuilds the matrix the 29 route tables encode (TC bitmap
                     sub-blocks, SPTC groups, CUDA parts), i.e. the operand the
                     reference's routed forward multiplies.
  decode_plan()      rebuilds the matrix a device plan multiplies from the
                     native builder's host arrays (tiles, residual, row
                     scales, output rows); plan_value_of_entries() reads back
                     each CSR entry's value through the entry -> slot map.
  spmm_f64() / spmm_f16_f32() / sddmm_f64()   CSR arithmetic in C (OpenMP).
  tca.tca_order()    Python restatement of the TCA row reorder
                     (spmm/tr_csr_fp16/tr_tca_reorder.py:44-357).
"""
from . import tca
from .core import (TABLE_NAMES, route, ref_route, ref_available, ref_match, ref_match_available,
                   ref_spmm_available, ref_sptc_online, check_sptc_tables,
                   ref_parallel_cuda_route, check_cuda_route_tables,
                   decode_tables,
                   decode_sptc_tiles, decode_plan, plan_value_of_entries, spmm_f64,
                   spmm_f16_f32, sddmm_f64, sddmm_f16_f32, max_threads, lib_path)

__all__ = ["tca", "TABLE_NAMES", "route", "ref_route", "ref_available", "ref_match",
           "ref_match_available", "decode_tables",
           "decode_sptc_tiles", "decode_plan", "plan_value_of_entries", "spmm_f64", "spmm_f16_f32", "sddmm_f64", "sddmm_f16_f32", "max_threads",
           "lib_path"]
