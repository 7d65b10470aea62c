"""Drop-in for the reference's ``Libra6SpMMOnline`` extension module.

The four operators keep the reference signatures
(TR-source/SpMM/mGCN_online.cpp:1142-1152): CPU tensors in, a freshly
allocated FP32 CPU output plus averaged millisecond timings out.  Inside,
each call builds a device plan from the route tables and runs the routed
product (libtrspmm.so: the CUDA-core residual pass, then the tensor-core
tiles added into C) ``epoches`` times after 10 warm-ups, as the reference's
launcher does (mGCNkernel_online.cu:1604-1674).  The result is
C = A_tables . B in FP32 accumulation for every route; there is no CPU
fallback.

Per-route times of ``forward_fp16_tcu_cuda_sptc_mma_parallel_online`` come
from the one-CTA-per-window kernel restricted to one route at a time (TC,
CUDA, SPTC); the CUDA time is reported for both the long and the short CUDA
parts, which this library processes together.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from trspmm._lib import check, lib


def _cpu(x, name, dtype):
    if x.is_cuda:
        raise RuntimeError(f"{name} must be a CPU tensor")
    if x.dtype != dtype:
        raise RuntimeError(f"{name} has an unexpected dtype")
    return x.contiguous()


def _arg(t):
    return [ctypes.c_void_p(t.data_ptr() if t.numel() else 0), ctypes.c_int64(t.numel())]


def _run(fn, tensors, ints, mOri, dimN):
    out = torch.zeros((mOri, dimN), dtype=torch.float32)
    ms = (ctypes.c_float * 5)()
    args = []
    for t in tensors:
        args += _arg(t)
    args += [ctypes.c_int32(int(v)) for v in ints]
    args += [ctypes.c_void_p(out.data_ptr()), ms]
    check(fn(*args))
    return out, [torch.tensor(float(ms[i]), dtype=torch.float32) for i in range(5)]


def forward_fp16_tcu_cuda_sptc_mma_parallel_online(
        t_row_offset, t_blockNew_offset, t_column, t_value, t_window_row, t_atomic, t_binary,
        c_row_offsets, c_row, c_atomic, c_column, c_value,
        c_row_offsets_short, c_row_short, c_atomic_short, c_column_short, c_value_short,
        s_column, s_value, s_pos, s_offsets, s_tile_window, s_tile_column, s_packed_a,
        s_packed_meta, s_window_tile_offset, rhs_matrix,
        parts_t, parts_c, partsize_c, parts_c_short, window, dimN, mOri, kOri, epoches):
    """Routed TC + SPTC + CUDA forward (mGCN_online.cpp:760-1138).  Returns
    [out f32 [mOri, dimN], ms, tc_ms, cuda_long_ms, cuda_short_ms, sptc_ms]."""
    i32, f16, f32 = torch.int32, torch.float16, torch.float32
    spec = [(t_row_offset, "t_row_offset", i32), (t_blockNew_offset, "t_blockNew_offset", i32),
            (t_column, "t_column", i32), (t_value, "t_value", f16),
            (t_window_row, "t_window_row", i32), (t_atomic, "t_atomic", i32),
            (t_binary, "t_binary", torch.int64),
            (c_row_offsets, "c_row_offsets", i32), (c_row, "c_row", i32),
            (c_atomic, "c_atomic", i32), (c_column, "c_column", i32), (c_value, "c_value", f16),
            (c_row_offsets_short, "c_row_offsets_short", i32), (c_row_short, "c_row_short", i32),
            (c_atomic_short, "c_atomic_short", i32), (c_column_short, "c_column_short", i32),
            (c_value_short, "c_value_short", f16),
            (s_column, "s_column", i32), (s_value, "s_value", f32), (s_pos, "s_pos", torch.int8),
            (s_offsets, "s_offsets", i32), (s_tile_window, "s_tile_window", i32),
            (s_tile_column, "s_tile_column", i32), (s_packed_a, "s_packed_a", i32),
            (s_packed_meta, "s_packed_meta", i32),
            (s_window_tile_offset, "s_window_tile_offset", i32), (rhs_matrix, "rhs_matrix", f16)]
    ts = [_cpu(t, n, d) for t, n, d in spec]
    if not (0 < window <= 16):
        raise RuntimeError("parallel mma path requires 0 < window <= 16")
    if s_column.dim() != 2 or s_column.shape[1] != 4:
        raise RuntimeError("s_column must have shape [groups, 4]")
    if s_value.dim() != 3 or s_value.shape[1] != window or s_value.shape[2] != 2:
        raise RuntimeError("s_value must have shape [groups, window, 2]")
    if s_pos.dim() != 3 or s_pos.shape[1] != window or s_pos.shape[2] != 2:
        raise RuntimeError("s_pos must have shape [groups, window, 2]")
    if s_tile_column.dim() != 2 or s_tile_column.shape[1] != 16:
        raise RuntimeError("s_tile_column must have shape [tiles, 16]")
    if s_packed_a.dim() != 4 or tuple(s_packed_a.shape[1:]) != (8, 4, 2):
        raise RuntimeError("s_packed_a must have shape [tiles, 8, 4, 2]")
    if s_packed_meta.dim() != 2 or s_packed_meta.shape[1] != 8:
        raise RuntimeError("s_packed_meta must have shape [tiles, 8]")
    if s_value.shape[0] != s_column.shape[0]:
        raise RuntimeError("s_value group count mismatch")
    if s_pos.shape[0] != s_column.shape[0]:
        raise RuntimeError("s_pos group count mismatch")
    out, ms = _run(lib().tr_forward_fp16_tcu_cuda_sptc_mma_parallel_online, ts,
                   [parts_t, parts_c, partsize_c, parts_c_short, window, dimN, mOri, kOri,
                    epoches], mOri, dimN)
    return [out] + ms


def forward_fp16_sptc_online(s_column, s_value, s_pos, s_window, rhs_matrix, window, dimN, mOri,
                             kOri, epoches):
    """SPTC route alone from the group tables (mGCN_online.cpp:202-400). Returns [out, ms]."""
    ts = [_cpu(s_column, "s_column", torch.int32), _cpu(s_value, "s_value", torch.float32),
          _cpu(s_pos, "s_pos", torch.int8), _cpu(s_window, "s_window", torch.int32),
          _cpu(rhs_matrix, "rhs_matrix", torch.float16)]
    if s_column.dim() != 2 or s_column.shape[1] != 4:
        raise RuntimeError("s_column must have shape [groups, 4]")
    if s_value.dim() != 3 or s_value.shape[1] != window or s_value.shape[2] != 2:
        raise RuntimeError("s_value must have shape [groups, window, 2]")
    if s_pos.dim() != 3 or s_pos.shape[1] != window or s_pos.shape[2] != 2:
        raise RuntimeError("s_pos must have shape [groups, window, 2]")
    if s_window.dim() != 1:
        raise RuntimeError("s_window must be 1-D")
    out, ms = _run(lib().tr_forward_fp16_sptc_online, ts, [window, dimN, mOri, kOri, epoches],
                   mOri, dimN)
    return [out, ms[0]]


def forward_fp16_sptc_mma_online(s_column, s_value, s_pos, s_offsets, rhs_matrix, window, dimN,
                                 mOri, kOri, epoches):
    """SPTC route from group tables with per-window offsets (mGCN_online.cpp:404-652)."""
    ts = [_cpu(s_column, "s_column", torch.int32), _cpu(s_value, "s_value", torch.float32),
          _cpu(s_pos, "s_pos", torch.int8), _cpu(s_offsets, "s_offsets", torch.int32),
          _cpu(rhs_matrix, "rhs_matrix", torch.float16)]
    if s_column.dim() != 2 or s_column.shape[1] != 4:
        raise RuntimeError("s_column must have shape [groups, 4]")
    out, ms = _run(lib().tr_forward_fp16_sptc_mma_online, ts, [window, dimN, mOri, kOri, epoches],
                   mOri, dimN)
    return [out, ms[0]]


def forward_fp16_sptc_mma_packed_online(s_tile_column, s_packed_a, s_packed_meta,
                                        s_window_tile_offset, rhs_matrix, window, dimN, mOri, kOri,
                                        epoches):
    """SPTC route from the packed tiles (mGCN_online.cpp:654-757). Returns [out, ms]."""
    ts = [_cpu(s_tile_column, "s_tile_column", torch.int32),
          _cpu(s_packed_a, "s_packed_a", torch.int32),
          _cpu(s_packed_meta, "s_packed_meta", torch.int32),
          _cpu(s_window_tile_offset, "s_window_tile_offset", torch.int32),
          _cpu(rhs_matrix, "rhs_matrix", torch.float16)]
    if not (0 < window <= 16):
        raise RuntimeError("packed mma path requires 0 < window <= 16")
    if s_tile_column.dim() != 2 or s_tile_column.shape[1] != 16:
        raise RuntimeError("s_tile_column must have shape [tiles, 16]")
    if s_packed_a.dim() != 4 or tuple(s_packed_a.shape[1:]) != (8, 4, 2):
        raise RuntimeError("s_packed_a must have shape [tiles, 8, 4, 2]")
    if s_packed_meta.dim() != 2 or s_packed_meta.shape[1] != 8:
        raise RuntimeError("s_packed_meta must have shape [tiles, 8]")
    if s_window_tile_offset.dim() != 1 or s_window_tile_offset.shape[0] < 2:
        raise RuntimeError("s_window_tile_offset must be 1-D with at least 2 elements")
    if rhs_matrix.numel() != kOri * dimN:
        raise RuntimeError("rhs_matrix must have kOri * dimN elements")
    out, ms = _run(lib().tr_forward_fp16_sptc_mma_packed_online, ts,
                   [window, dimN, mOri, kOri, epoches], mOri, dimN)
    return [out, ms[0]]
