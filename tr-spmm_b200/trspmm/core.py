"""Host-side API over libtrspmm: routing, device plans, forward SpMM.

  route(...)              the three-stage router -> the reference's 30 tables
  Plan.from_tables(...)   device plan from route tables (reference layout)
  Plan.from_csr(...)      route with this library's router and build the plan
  Plan.build(...)         native builder: row scaling, promotion of shared
                          residual columns to tensor-core tiles, adjoint
                          (transposed) plans, row clustering
  Plan.spmm(B)            routed forward C = A_plan . B on the GPU
  Plan.set_values(w)      re-value a plan from FP32 per-entry values (device)
  spmm_csr(...)           the plain single-route CSR kernel
  sddmm_csr(...)          out[e] = <X[row e], Y[col e]> on a CSR pattern
"""
from __future__ import annotations

import collections
import ctypes
import hashlib
import os

import numpy as np

from . import _lib
from ._lib import (TR_MATCH_BUCKET, TR_MATCH_HASH, TR_MATCH_ONLINE, TR_MATCH_SLIDING, TR_OUT_F16,
                   TR_OUT_F32,
                   TR_ENGINE_BLOCK, TR_ENGINE_WINDOW,
                   TR_REORDER_GIVEN, TR_REORDER_LABEL, TR_REORDER_NONE, TR_REORDER_TCA,
                   TR_ROUTE_ALL, TR_ROUTE_COMPAT, TR_ROUTE_EXACT, MatchStats, PlanInfo, PlanOpts,
                   RouteParams, Tables, TcaParams, TcaStats, check, lib)

TABLE_NAMES = [
    "t_row_offset", "t_block_offset", "t_column", "t_value", "t_window_row", "t_atomic",
    "t_binary",
    "c_row_offset", "c_row", "c_atomic", "c_column", "c_value",
    "c_row_offset_short", "c_row_short", "c_atomic_short", "c_column_short", "c_value_short",
    "s_column", "s_mask", "s_value", "s_pos", "s_window", "s_offsets",
    "s_tile_window", "s_tile_group", "s_tile_column", "s_packed_a", "s_packed_meta",
    "s_window_tile_offset", "duration",
]
_DTYPES = [np.int32, np.int32, np.int32, np.float32, np.int32, np.int32, np.int64,
           np.int32, np.int32, np.int32, np.int32, np.float32,
           np.int32, np.int32, np.int32, np.int32, np.float32,
           np.int32, np.uint8, np.float32, np.int8, np.int32, np.int32,
           np.int32, np.int32, np.int32, np.int32, np.int32, np.int32]


def _vp(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None and a.size else ctypes.c_void_p(0)


REORDER_MODES = {False: TR_REORDER_NONE, None: TR_REORDER_NONE, "none": TR_REORDER_NONE,
                 True: TR_REORDER_LABEL, "label": TR_REORDER_LABEL, "tca": TR_REORDER_TCA}


ENGINES = {"window": TR_ENGINE_WINDOW, "block": TR_ENGINE_BLOCK}

_LABEL_ORDERS = collections.OrderedDict()      # structure digest -> order
_LABEL_ORDERS_KEPT = 8


def label_order(indptr, indices, n_rows, n_cols, transpose=False):
    """The row order that reorder=True ("label") gives a plan of A, or of A^T
    when transpose (tr_label_order): plan row i = row order[i].

    Memoised on the matrix's structure (a BLAKE2b digest of n_rows, n_cols,
    indptr and indices; the last few matrices kept): an autotuner builds
    several plans of one matrix, and label propagation costs seconds on large
    graphs.  The order is deterministic, and Plan.build / host_plan with
    reorder=True pass it on as the caller's permutation, which builds the
    same plan as the builder's own label mode."""
    rp = np.ascontiguousarray(indptr, dtype=np.int32)
    ci = np.ascontiguousarray(indices, dtype=np.int32)
    h = hashlib.blake2b(digest_size=16)
    h.update(np.array([n_rows, n_cols, int(bool(transpose))], dtype=np.int64).tobytes())
    h.update(memoryview(rp).cast("B"))
    h.update(memoryview(ci).cast("B"))
    key = h.digest()
    if key in _LABEL_ORDERS:
        _LABEL_ORDERS.move_to_end(key)
        return _LABEL_ORDERS[key]
    order = np.empty(int(n_cols if transpose else n_rows), dtype=np.int32)
    if order.size:
        check(lib().tr_label_order(_vp(rp), _vp(ci), int(n_rows), int(n_cols),
                                   int(bool(transpose)), _vp(order)))
    order.flags.writeable = False
    _LABEL_ORDERS[key] = order
    while len(_LABEL_ORDERS) > _LABEL_ORDERS_KEPT:
        _LABEL_ORDERS.popitem(last=False)
    return order


def _resolve_reorder(reorder, indptr, indices, n_rows, n_cols, transpose):
    """reorder=True / "label" as the memoised label order; anything else as given."""
    if isinstance(reorder, (bool, str)) and REORDER_MODES.get(reorder) == TR_REORDER_LABEL:
        return label_order(indptr, indices, n_rows, n_cols, transpose)
    return reorder


def plan_opts(row_scale=False, promote_min=0, transpose=False, reorder=False, demote_below=0,
              engine="window"):
    """(tr_plan_opts, keep-alive array).  ``reorder``: False / "none", True /
    "label" (label propagation), "tca" (TCA clustering, tr_tca_order's
    defaults) or an int array, the caller's row permutation (plan row i is row
    reorder[i] of the matrix the plan is built for: A, or A^T when
    transpose).  ``engine``: "window" (the three routes over 16-row windows)
    or "block" (every entry on the tensor cores over 128-row blocks)."""
    if engine not in ENGINES:
        raise ValueError(f"unknown plan engine {engine!r}")
    order = None
    if isinstance(reorder, (str, bool)) or reorder is None:
        if reorder not in REORDER_MODES:
            raise ValueError(f"unknown reorder mode {reorder!r}")
        mode = REORDER_MODES[reorder]
    else:
        order = np.ascontiguousarray(reorder, dtype=np.int32)
        mode = TR_REORDER_GIVEN
    opts = PlanOpts(int(bool(row_scale)), int(promote_min), int(bool(transpose)), int(mode),
                    int(demote_below), _vp(order) if order is not None else ctypes.c_void_p(0),
                    ENGINES[engine])
    return opts, order


def _params(partsize_t=32, partsize_c=32, shortsize=3, density=8, window=16, wide=16,
            tc_min_util=0.0, sptc_min_util=0.5, sptc_threshold=12, unit_min_nnz=None,
            skip_tc=None, mode="compat", threads=0, skip_sptc=False):
    if unit_min_nnz is None:
        unit_min_nnz = int(os.environ.get("LIBRA_SPTC_UNIT_MIN_NNZ", "2"))
    if skip_tc is None:
        skip_tc = os.environ.get("LIBRA_SKIP_TC", "0") in ("1", "true", "TRUE")
    m = {"compat": TR_ROUTE_COMPAT, "exact": TR_ROUTE_EXACT}[mode]
    return RouteParams(int(partsize_t), int(partsize_c), int(shortsize), int(density), int(window),
                       int(wide), float(tc_min_util), float(sptc_min_util), int(sptc_threshold),
                       int(unit_min_nnz), int(bool(skip_tc)), m, int(threads),
                       int(bool(skip_sptc)))


def route(indptr, indices, values, partsize_t=32, partsize_c=32, shortsize=3, density=8,
          window=16, wide=16, tc_min_util=0.0, sptc_min_util=0.5, sptc_threshold=12,
          mode="compat", unit_min_nnz=None, skip_tc=None, threads=0, skip_sptc=False):
    """Route a CSR matrix; returns the 30 tables of block_sptc_2to4_online
    (TR-source/Block/block_online.cpp:844-870) as numpy arrays, the last being
    the routing time in seconds (float32).  skip_sptc: no 2:4 groups (every
    column outside the dense-TC funnel goes to the CUDA parts)."""
    L = lib()
    rp = np.ascontiguousarray(indptr, dtype=np.int32)
    ci = np.ascontiguousarray(indices, dtype=np.int32)
    vv = np.ascontiguousarray(values, dtype=np.float32)
    prm = _params(partsize_t, partsize_c, shortsize, density, window, wide, tc_min_util,
                  sptc_min_util, sptc_threshold, unit_min_nnz, skip_tc, mode, threads,
                  skip_sptc)
    h = ctypes.c_void_p()
    check(L.tr_route_build(_vp(rp), _vp(ci), _vp(vv), rp.shape[0] - 1, ctypes.byref(prm),
                           ctypes.byref(h)))
    return _read_route(h, window)


class _DeviceArray:
    """A device table seen through __cuda_array_interface__ (no copy)."""

    def __init__(self, ptr, n, dtype):
        self.__cuda_array_interface__ = {"shape": (int(n),), "typestr": np.dtype(dtype).str,
                                         "data": (int(ptr or 0), False), "version": 3}


def route_device(indptr, indices, values, partsize_t=32, partsize_c=32, shortsize=3, density=8,
                 window=16, wide=16, tc_min_util=0.0, sptc_min_util=0.5, sptc_threshold=12,
                 mode="compat", unit_min_nnz=None, skip_tc=None, skip_sptc=False, out="numpy"):
    """route() on the GPU (tr_route_device): every router stage as device
    kernels over a CSR on the device (int32 indptr / indices and float32
    values as CUDA tensors, or numpy arrays, uploaded first; rows sorted by
    column).  Returns the same 30 tables as route(), equal item for item:
    numpy arrays (out="numpy"), or CUDA tensors that never leave the device
    (out="torch"; the last item is still the routing time in seconds)."""
    import torch
    dev = torch.device("cuda", torch.cuda.current_device())
    t = [x if hasattr(x, "is_cuda") else torch.from_numpy(np.ascontiguousarray(x, dtype=d))
         for x, d in ((indptr, np.int32), (indices, np.int32), (values, np.float32))]
    t = [x.to(dev) for x in t]
    for x, dt in zip(t, (torch.int32, torch.int32, torch.float32)):
        if not (x.dtype == dt and x.is_contiguous()):
            raise RuntimeError("indptr/indices (int32) and values (float32) must be contiguous")
    prm = _params(partsize_t, partsize_c, shortsize, density, window, wide, tc_min_util,
                  sptc_min_util, sptc_threshold, unit_min_nnz, skip_tc, mode, 0, skip_sptc)
    h = ctypes.c_void_p()
    check(lib().tr_route_device(ctypes.c_void_p(t[0].data_ptr()), ctypes.c_void_p(t[1].data_ptr()),
                                ctypes.c_void_p(t[2].data_ptr()), t[0].numel() - 1,
                                ctypes.byref(prm), ctypes.byref(h)))
    if out == "numpy":
        return _read_route(h, window)
    L = lib()
    try:
        tabs = []
        for i, dt in enumerate(_DTYPES):
            data = ctypes.c_void_p()
            n = ctypes.c_int64()
            check(L.tr_route_table_device(h, i, ctypes.byref(data), ctypes.byref(n)))
            view = torch.as_tensor(_DeviceArray(data.value, n.value, dt), device=dev)
            tabs.append(view.clone())
        torch.cuda.synchronize(dev)
        seconds = L.tr_route_seconds(h)
    finally:
        L.tr_route_free(h)
    g = tabs[21].shape[0]
    nt = tabs[23].shape[0]
    tabs[17] = tabs[17].reshape(g, 4)
    tabs[18] = tabs[18].reshape(g, window)
    tabs[19] = tabs[19].reshape(g, window, 2)
    tabs[20] = tabs[20].reshape(g, window, 2)
    tabs[25] = tabs[25].reshape(nt, 16)
    tabs[26] = tabs[26].reshape(nt, 8, 4, 2)
    tabs[27] = tabs[27].reshape(nt, 8)
    tabs.append(np.float32(seconds))
    return tabs


def _read_route(h, window):
    """The 30 tables of a tr_route handle (which it frees)."""
    L = lib()
    try:
        out = []
        for i, dt in enumerate(_DTYPES):
            data = ctypes.c_void_p()
            n = ctypes.c_int64()
            check(L.tr_route_table(h, i, ctypes.byref(data), ctypes.byref(n)))
            if n.value == 0:
                out.append(np.zeros(0, dtype=dt))
            else:
                nbytes = n.value * np.dtype(dt).itemsize
                buf = (ctypes.c_char * nbytes).from_address(data.value)
                out.append(np.frombuffer(buf, dtype=dt, count=n.value).copy())
        seconds = L.tr_route_seconds(h)
    finally:
        L.tr_route_free(h)
    g = out[21].shape[0]
    t = out[23].shape[0]
    out[17] = out[17].reshape(g, 4)
    out[18] = out[18].reshape(g, window)
    out[19] = out[19].reshape(g, window, 2)
    out[20] = out[20].reshape(g, window, 2)
    out[25] = out[25].reshape(t, 16)
    out[26] = out[26].reshape(t, 8, 4, 2)
    out[27] = out[27].reshape(t, 8)
    out.append(np.float32(seconds))
    return out


TC_TABLE_IDX = {"t_row_offset": 0, "t_block_offset": 1, "t_column": 2, "t_value": 3,
                "t_window_row": 4, "t_binary": 6}


def route_tc_device(indptr, indices, values, n_rows, partsize_t=32, density=8, tc_min_util=0.0,
                    skip_tc=False):
    """The dense-TC funnel of the router on the GPU (tr_route_tc_device):
    CUDA int32 indptr/indices and float32 values of a CSR whose rows are
    sorted by column; returns the TC tables (numpy) keyed by name, equal to
    route(..., mode="exact")'s t_row_offset, t_block_offset, t_column,
    t_value, t_window_row and t_binary."""
    import torch
    for t, dt in ((indptr, torch.int32), (indices, torch.int32), (values, torch.float32)):
        if not (t.is_cuda and t.dtype == dt and t.is_contiguous()):
            raise RuntimeError("indptr/indices (int32) and values (float32) must be contiguous CUDA tensors")
    L = lib()
    prm = _params(partsize_t=partsize_t, density=density, tc_min_util=tc_min_util,
                  skip_tc=skip_tc, mode="exact")
    h = ctypes.c_void_p()
    check(L.tr_route_tc_device(ctypes.c_void_p(indptr.data_ptr()),
                               ctypes.c_void_p(indices.data_ptr()),
                               ctypes.c_void_p(values.data_ptr()), int(n_rows), ctypes.byref(prm),
                               ctypes.byref(h)))
    try:
        out = {}
        for name, i in TC_TABLE_IDX.items():
            dt = _DTYPES[i]
            data = ctypes.c_void_p()
            n = ctypes.c_int64()
            check(L.tr_route_table(h, i, ctypes.byref(data), ctypes.byref(n)))
            if n.value == 0:
                out[name] = np.zeros(0, dtype=dt)
            else:
                buf = (ctypes.c_char * (n.value * np.dtype(dt).itemsize)).from_address(data.value)
                out[name] = np.frombuffer(buf, dtype=dt, count=n.value).copy()
        out["seconds"] = L.tr_route_seconds(h)
    finally:
        L.tr_route_free(h)
    return out


def _half_bits(x):
    a = np.ascontiguousarray(x)
    if a.dtype != np.float16:
        a = a.astype(np.float32).astype(np.float16)
    return a.view(np.uint16)


def _np(x, dtype):
    if hasattr(x, "detach"):
        x = x.detach().cpu().numpy()
    return np.ascontiguousarray(x, dtype=dtype)


def tables_struct(tabs):
    """ctypes Tables struct over a 30-table list (values rounded to FP16);
    returns (struct, keepalive list)."""
    T = dict(zip(TABLE_NAMES, tabs))
    keep = {
        "t_row_offset": _np(T["t_row_offset"], np.int32),
        "t_block_offset": _np(T["t_block_offset"], np.int32),
        "t_column": _np(T["t_column"], np.int32),
        "t_value": _half_bits(_np(T["t_value"], None)),
        "t_window_row": _np(T["t_window_row"], np.int32),
        "t_binary": _np(T["t_binary"], np.int64),
        "c_row_offset": _np(T["c_row_offset"], np.int32),
        "c_row": _np(T["c_row"], np.int32),
        "c_column": _np(T["c_column"], np.int32),
        "c_value": _half_bits(_np(T["c_value"], None)),
        "cs_row_offset": _np(T["c_row_offset_short"], np.int32),
        "cs_row": _np(T["c_row_short"], np.int32),
        "cs_column": _np(T["c_column_short"], np.int32),
        "cs_value": _half_bits(_np(T["c_value_short"], None)),
        "s_tile_column": _np(T["s_tile_column"], np.int32).ravel(),
        "s_packed_a": _np(T["s_packed_a"], np.int32).ravel(),
        "s_packed_meta": _np(T["s_packed_meta"], np.int32).ravel(),
        "s_window_tile_offset": _np(T["s_window_tile_offset"], np.int32),
    }
    st = Tables()
    for name, arr in keep.items():
        setattr(st, name, arr.ctypes.data if arr.size else None)
        setattr(st, "n_" + name, int(arr.size))
    return st, keep


class Plan:
    """Routed operand resident in HBM (see csrc/plan.h for its layout)."""

    def __init__(self, handle):
        self._h = handle
        info = PlanInfo()
        check(lib().tr_plan_info_get(self._h, ctypes.byref(info)))
        self.info = {f: getattr(info, f) for f, _ in PlanInfo._fields_}
        self.n_rows = info.n_rows
        self.n_cols = info.n_cols
        self.k_tile = 0
        self.deterministic = False

    @classmethod
    def from_tables(cls, tabs, n_rows, n_cols, window=16):
        st, keep = tables_struct(tabs)
        h = ctypes.c_void_p()
        check(lib().tr_plan_from_tables(ctypes.byref(st), int(n_rows), int(n_cols), int(window),
                                        ctypes.byref(h)))
        del keep
        return cls(h)

    @classmethod
    def from_csr(cls, indptr, indices, values, n_rows, n_cols, mode="exact", **route_kw):
        rp = np.ascontiguousarray(indptr, dtype=np.int32)
        ci = np.ascontiguousarray(indices, dtype=np.int32)
        vv = np.ascontiguousarray(values, dtype=np.float32)
        prm = _params(mode=mode, **route_kw)
        h = ctypes.c_void_p()
        check(lib().tr_plan_from_csr(_vp(rp), _vp(ci), _vp(vv), int(n_rows), int(n_cols),
                                     ctypes.byref(prm), ctypes.byref(h)))
        return cls(h)

    @classmethod
    def build(cls, indptr, indices, values, n_rows, n_cols, row_scale=False, promote_min=0,
              transpose=False, reorder=False, demote_below=0, mode="exact", engine="window",
              k_tile=0, **route_kw):
        """Native builder (tr_plan_build): route A (or A^T when transpose) and
        lay it out; the plan keeps, for every CSR entry of A, where its value
        lives (set_values).  For a transposed plan n_rows/n_cols are A's.
        ``engine="block"`` lays the matrix out for the block engine;
        ``k_tile`` its features per tensor-core launch (set_k_tile)."""
        rp = np.ascontiguousarray(indptr, dtype=np.int32)
        ci = np.ascontiguousarray(indices, dtype=np.int32)
        vv = None if values is None else np.ascontiguousarray(values, dtype=np.float32)
        prm = _params(mode=mode, **route_kw)
        reorder = _resolve_reorder(reorder, rp, ci, n_rows, n_cols, transpose)
        opts, keep = plan_opts(row_scale, promote_min, transpose, reorder, demote_below, engine)
        h = ctypes.c_void_p()
        check(lib().tr_plan_build(_vp(rp), _vp(ci), _vp(vv), int(n_rows), int(n_cols),
                                  ctypes.byref(prm), ctypes.byref(opts), ctypes.byref(h)))
        plan = cls(h)
        if k_tile:
            plan.set_k_tile(k_tile)
        return plan

    def set_k_tile(self, k_tile):
        """Features per tensor-core launch of a block-engine plan
        (tr_plan_set_k_tile: 0 = 256, else 64, 128, 192 or 256)."""
        check(lib().tr_plan_set_k_tile(self._h, int(k_tile)))
        self.k_tile = int(k_tile)

    def set_deterministic(self, on=True):
        """Bitwise-repeatable backward (tr_plan_set_deterministic): the fused
        adjoint + SDDMM of a window plan combines rows cut by its segments in
        a fixed order; block plans are always repeatable."""
        check(lib().tr_plan_set_deterministic(self._h, int(bool(on))))
        self.deterministic = bool(on)

    def set_values(self, values, stream=None):
        """Re-value the plan from a CUDA float32 tensor of A's CSR entries."""
        import torch
        if not (values.is_cuda and values.dtype == torch.float32 and values.is_contiguous()
                and values.dim() == 1):
            raise RuntimeError("values must be a contiguous 1-D float32 CUDA tensor")
        s = stream if stream is not None else torch.cuda.current_stream(values.device).cuda_stream
        check(lib().tr_plan_set_values(self._h, ctypes.c_void_p(values.data_ptr()),
                                       int(values.numel()), ctypes.c_void_p(s)))

    def entry_order(self, device=None, stream=None):
        """The plan's entry order (tr_plan_entry_order): int32 CUDA tensor
        ``order`` with order[q] = the edge at plan position q (-1 where no
        edge sits).  Block-engine plans and window plans without tiles."""
        import torch
        dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        order = torch.empty(int(self.info["n_edges"]), dtype=torch.int32, device=dev)
        s = stream if stream is not None else torch.cuda.current_stream(dev).cuda_stream
        check(lib().tr_plan_entry_order(self._h, ctypes.c_void_p(order.data_ptr()), ctypes.c_void_p(s)))
        return order

    def renumber_edges(self, new_id, stream=None):
        """Give the plan's edges new numbers (tr_plan_renumber_edges): the edge
        now numbered e becomes new_id[e] (int32 CUDA permutation).  Afterwards
        set_values takes, and adjoint_sddmm returns, per-entry arrays in the
        new numbering."""
        import torch
        if not (new_id.is_cuda and new_id.dtype == torch.int32 and new_id.is_contiguous()
                and new_id.dim() == 1):
            raise RuntimeError("new_id must be a contiguous 1-D int32 CUDA tensor")
        s = stream if stream is not None else torch.cuda.current_stream(new_id.device).cuda_stream
        check(lib().tr_plan_renumber_edges(self._h, ctypes.c_void_p(new_id.data_ptr()),
                                           int(new_id.numel()), ctypes.c_void_p(s)))

    def spmm(self, b, out=None, out_dtype=None, route_mask=TR_ROUTE_ALL, stream=None):
        """C = A_plan . B for a CUDA tensor B [n_cols, K]: FP16 B on the routed
        kernels (tensor-core tiles + CUDA-core residual), FP32 B on the
        FP32-feature route (tr_spmm_routed_f32, CUDA cores in FP32)."""
        import torch
        _check_b(b, self.n_cols, fp32_ok=True)
        k = b.shape[1]
        if out is None:
            out = torch.empty((self.n_rows, k), dtype=out_dtype or torch.float32, device=b.device)
        _check_out(out, self.n_rows, k)
        s = stream if stream is not None else torch.cuda.current_stream(b.device).cuda_stream
        fn = lib().tr_spmm_routed_f32 if b.dtype == torch.float32 else lib().tr_spmm_routed
        check(fn(self._h, ctypes.c_void_p(b.data_ptr()), int(k), ctypes.c_void_p(out.data_ptr()),
                 _odt(out), int(route_mask), ctypes.c_void_p(s)))
        return out

    def adjoint_sddmm(self, a_indptr, a_indices, dc, b, db=None, dval=None, db_dtype=None,
                      stream=None):
        """For an adjoint plan (built with transpose=True): dB = A^T . dC and
        dval = SDDMM(dC, B) on A's pattern, fused into one pass where the plan
        allows (tr_adjoint_sddmm).  dc [A rows, K], b [A cols, K] CUDA, both
        FP16 or both FP32 (tr_adjoint_sddmm_f32)."""
        import torch
        _check_b(dc, self.n_cols, fp32_ok=True)
        if not (b.is_cuda and b.dtype == dc.dtype and b.is_contiguous() and b.dim() == 2
                and b.shape == (self.n_rows, dc.shape[1])):
            raise RuntimeError("b must be a contiguous CUDA tensor [A cols, K] of dc's dtype")
        k = dc.shape[1]
        nnz = a_indices.numel()
        if db is None:
            db = torch.empty((self.n_rows, k), dtype=db_dtype or torch.float32, device=dc.device)
        _check_out(db, self.n_rows, k)
        if dval is None:
            dval = torch.empty(nnz, dtype=torch.float32, device=dc.device)
        if not (dval.is_cuda and dval.dtype == torch.float32 and dval.numel() == nnz):
            raise RuntimeError("dval must be a float32 CUDA tensor with one item per entry")
        s = stream if stream is not None else torch.cuda.current_stream(dc.device).cuda_stream
        fn = lib().tr_adjoint_sddmm_f32 if dc.dtype == torch.float32 else lib().tr_adjoint_sddmm
        check(fn(self._h, ctypes.c_void_p(a_indptr.data_ptr()),
                 ctypes.c_void_p(a_indices.data_ptr()), int(self.n_cols),
                 int(nnz), ctypes.c_void_p(dc.data_ptr()),
                 ctypes.c_void_p(b.data_ptr()), int(k),
                 ctypes.c_void_p(db.data_ptr()), _odt(db),
                 ctypes.c_void_p(dval.data_ptr()), ctypes.c_void_p(s)))
        return db, dval

    def close(self):
        if self._h:
            lib().tr_plan_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _odt(out):
    import torch
    if out.dtype == torch.float32:
        return TR_OUT_F32
    if out.dtype == torch.float16:
        return TR_OUT_F16
    raise TypeError("output must be float32 or float16")


def _check_b(b, n_cols, fp32_ok=False):
    import torch
    kinds = (torch.float16, torch.float32) if fp32_ok else (torch.float16,)
    if not (b.is_cuda and b.dtype in kinds and b.dim() == 2 and b.is_contiguous()):
        raise RuntimeError("B must be a contiguous 2-D " +
                           ("float16 or float32" if fp32_ok else "float16") + " CUDA tensor")
    if b.shape[0] != n_cols:
        raise RuntimeError(f"B has {b.shape[0]} rows, the matrix has {n_cols} columns")


def _check_out(out, m, k):
    if not (out.is_cuda and out.is_contiguous() and tuple(out.shape) == (m, k)):
        raise RuntimeError(f"out must be a contiguous CUDA tensor of shape ({m}, {k})")


def spmm_csr(indptr, indices, values, b, n_rows, out=None, out_dtype=None, stream=None):
    """Plain CSR SpMM (single CUDA-core route) on CUDA tensors: int32
    indptr/indices, FP16 values, FP16 B [n_cols, K]."""
    import torch
    _check_b(b, b.shape[0])
    k = b.shape[1]
    if out is None:
        out = torch.empty((n_rows, k), dtype=out_dtype or torch.float32, device=b.device)
    _check_out(out, n_rows, k)
    for t, dt in ((indptr, torch.int32), (indices, torch.int32), (values, torch.float16)):
        if not (t.is_cuda and t.dtype == dt and t.is_contiguous()):
            raise RuntimeError("indptr/indices must be int32 and values float16 contiguous CUDA tensors")
    s = stream if stream is not None else torch.cuda.current_stream(b.device).cuda_stream
    check(lib().tr_spmm_csr(ctypes.c_void_p(indptr.data_ptr()), ctypes.c_void_p(indices.data_ptr()),
                            ctypes.c_void_p(values.data_ptr()), int(n_rows), int(b.shape[0]),
                            int(indices.numel()), ctypes.c_void_p(b.data_ptr()), int(k),
                            ctypes.c_void_p(out.data_ptr()), _odt(out), ctypes.c_void_p(s)))
    return out


HOST_PLAN_ARRAYS = [("win_tile", np.int32), ("win_split", np.int32), ("win_prom", np.int32),
                    ("tile_col", np.int32), ("tile_a", np.uint16), ("res_ptr", np.int32),
                    ("res_col", np.int32), ("res_val", np.uint16), ("win_order", np.int32),
                    ("row_scale", np.float32), ("row_out", np.int32), ("val_slot", np.int32),
                    ("edge_row", np.int32), ("res_edge", np.int32), ("blk_chunk", np.int32),
                    ("chunk_col", np.int32), ("chunk_ent", np.int32), ("ent_pos", np.uint16),
                    ("ent_val", np.uint16), ("ent_src", np.int32), ("blk_order", np.int32)]


def host_plan(indptr, indices, values, n_rows, n_cols, row_scale=False, promote_min=0,
              transpose=False, reorder=False, demote_below=0, mode="exact", engine="window",
              k_tile=0, **route_kw):
    """The native builder's plan as host arrays (tr_plan_build_host), without
    a device: a dict name -> numpy array (layout in csrc/plan.h).  ``k_tile``
    is a launch setting and does not change the arrays."""
    rp = np.ascontiguousarray(indptr, dtype=np.int32)
    ci = np.ascontiguousarray(indices, dtype=np.int32)
    vv = None if values is None else np.ascontiguousarray(values, dtype=np.float32)
    prm = _params(mode=mode, **route_kw)
    reorder = _resolve_reorder(reorder, rp, ci, n_rows, n_cols, transpose)
    opts, keep = plan_opts(row_scale, promote_min, transpose, reorder, demote_below, engine)
    L = lib()
    h = ctypes.c_void_p()
    check(L.tr_plan_build_host(_vp(rp), _vp(ci), _vp(vv), int(n_rows), int(n_cols),
                               ctypes.byref(prm), ctypes.byref(opts), ctypes.byref(h)))
    try:
        out = host_plan_arrays(h)
    finally:
        L.tr_host_plan_free(h)
    out["n_rows"], out["n_cols"] = (n_cols, n_rows) if transpose else (n_rows, n_cols)
    return out


def host_plan_arrays(h):
    """Copies of a host plan handle's arrays (tr_host_plan_array), by name."""
    L = lib()
    out = {}
    for i, (name, dt) in enumerate(HOST_PLAN_ARRAYS):
        data = ctypes.c_void_p()
        n = ctypes.c_int64()
        check(L.tr_host_plan_array(h, i, ctypes.byref(data), ctypes.byref(n)))
        if n.value == 0:
            out[name] = np.zeros(0, dtype=dt)
        else:
            nbytes = n.value * np.dtype(dt).itemsize
            buf = (ctypes.c_char * nbytes).from_address(data.value)
            out[name] = np.frombuffer(buf, dtype=dt, count=n.value).copy()
    return out


def sddmm_csr(indptr, indices, x, y, out=None, stream=None):
    """out[e] = <x[row(e)], y[indices[e]]> (x [m, K], y [n, K], both FP16 or
    both FP32; FP32 out) for every entry of the CSR pattern (int32 CUDA
    indptr/indices)."""
    import torch
    m = indptr.numel() - 1
    for t in (x, y):
        if not (t.is_cuda and t.dtype in (torch.float16, torch.float32) and t.dim() == 2
                and t.is_contiguous()):
            raise RuntimeError("x and y must be contiguous 2-D float16 or float32 CUDA tensors")
    if x.dtype != y.dtype:
        raise RuntimeError("x and y must have the same dtype")
    if x.shape[0] != m or x.shape[1] != y.shape[1]:
        raise RuntimeError("x must be [rows, K] and y [cols, K] with the same K")
    for t in (indptr, indices):
        if not (t.is_cuda and t.dtype == torch.int32 and t.is_contiguous()):
            raise RuntimeError("indptr/indices must be contiguous int32 CUDA tensors")
    nnz = indices.numel()
    if out is None:
        out = torch.empty(nnz, dtype=torch.float32, device=x.device)
    if not (out.is_cuda and out.dtype == torch.float32 and out.numel() == nnz and out.is_contiguous()):
        raise RuntimeError("out must be a contiguous float32 CUDA tensor with one item per entry")
    s = stream if stream is not None else torch.cuda.current_stream(x.device).cuda_stream
    fn = lib().tr_sddmm_csr_f32 if x.dtype == torch.float32 else lib().tr_sddmm_csr
    check(fn(ctypes.c_void_p(indptr.data_ptr()), ctypes.c_void_p(indices.data_ptr()),
             int(m), int(y.shape[0]), int(nnz), ctypes.c_void_p(x.data_ptr()),
             ctypes.c_void_p(y.data_ptr()), int(x.shape[1]),
             ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(s)))
    return out


def tca_order(indptr, indices, n_rows=None, thres=16, cluster_thres=128, lsh_threshold=0.2,
              seed=1, max_pairs=1 << 25, device=False):
    """TCA row order of a host CSR (tr_tca_order): (order int32 [n_rows],
    new position -> old row; stats dict).  ``device=True`` computes the
    MinHash signatures and the Jaccard similarities on the current GPU."""
    order, stats, _ = tca_order_timed(indptr, indices, n_rows, thres=thres,
                                      cluster_thres=cluster_thres, lsh_threshold=lsh_threshold,
                                      seed=seed, max_pairs=max_pairs, device=device)
    return order, stats


def tca_order_timed(indptr, indices, n_rows=None, thres=16, cluster_thres=128,
                    lsh_threshold=0.2, seed=1, max_pairs=1 << 25, device=False):
    """tca_order plus the wall time of its stages: (order, stats, seconds)
    with seconds = {"signatures", "candidates", "jaccard", "cluster"}."""
    rp = np.ascontiguousarray(indptr, dtype=np.int32)
    ci = np.ascontiguousarray(indices, dtype=np.int32)
    n = int(rp.shape[0] - 1) if n_rows is None else int(n_rows)
    if rp.shape[0] < n + 1:
        raise ValueError("indptr shorter than n_rows + 1")
    prm = TcaParams(int(thres), int(cluster_thres), float(lsh_threshold), int(seed),
                    int(max_pairs), int(bool(device)))
    order = np.empty(max(n, 0), dtype=np.int32)
    st = TcaStats()
    check(lib().tr_tca_order(_vp(rp), _vp(ci), n, ctypes.byref(prm), _vp(order), ctypes.byref(st)))
    stats = {name: getattr(st, name) for name, _ in TcaStats._fields_ if name != "seconds"}
    secs = dict(zip(("signatures", "candidates", "jaccard", "cluster"), list(st.seconds)))
    return order, stats, secs


def lsh_params(threshold=0.2, num_perm=128):
    """(bands, rows per band) of the LSH banding tr_tca_order uses."""
    b, r = ctypes.c_int32(), ctypes.c_int32()
    check(lib().tr_lsh_params(float(threshold), int(num_perm), ctypes.byref(b), ctypes.byref(r)))
    return b.value, r.value


MATCH_VARIANTS = {"sliding": TR_MATCH_SLIDING, "hash": TR_MATCH_HASH, "bucket": TR_MATCH_BUCKET,
                  "online": TR_MATCH_ONLINE}


def match_2to4(indptr, indices, variant="sliding", window_size=16, dense_threshold=8, t_max=8):
    """2:4 matching statistics of a host CSR (tr_match_2to4): how the columns
    of each window pair into 1:2 pairs and 2:4 groups, and, for the sliding
    variant, which leftover columns form dense 16x8 blocks.  Returns a dict
    with every counter of tr_match_stats (num_groups counts 2:4 groups)."""
    rp = np.ascontiguousarray(indptr, dtype=np.int32)
    ci = np.ascontiguousarray(indices, dtype=np.int32)
    st = MatchStats()
    check(lib().tr_match_2to4(_vp(rp), _vp(ci), int(rp.shape[0] - 1), int(MATCH_VARIANTS[variant]),
                              int(window_size), int(dense_threshold), int(t_max),
                              ctypes.byref(st)))
    return {name: getattr(st, name) for name, _ in MatchStats._fields_ if name != "reserved"}


def match_2to4_online(indptr, indices, window_size=16, dense_threshold=8, t_max=8):
    """The online variant's statistics computed on the GPU
    (tr_match_2to4_online); equal to match_2to4(..., "online")."""
    rp = np.ascontiguousarray(indptr, dtype=np.int32)
    ci = np.ascontiguousarray(indices, dtype=np.int32)
    st = MatchStats()
    check(lib().tr_match_2to4_online(_vp(rp), _vp(ci), int(rp.shape[0] - 1), int(window_size),
                                     int(dense_threshold), int(t_max), ctypes.byref(st)))
    return {name: getattr(st, name) for name, _ in MatchStats._fields_ if name != "reserved"}
