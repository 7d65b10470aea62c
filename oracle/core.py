"""ORACLE — test infrastructure only (see oracle/__init__.py)."""
from __future__ import annotations

import ctypes
import glob
import os
import sys
import time

import numpy as np
import scipy.sparse as sp

HERE = os.path.dirname(os.path.abspath(__file__))
lib_path = os.path.join(HERE, "liboracle.so")

# Return order of block_sptc_2to4_online (TR-source/Block/block_online.cpp:844-870).
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

_lib = None


def _load():
    global _lib
    if _lib is None:
        if not os.path.exists(lib_path):
            raise RuntimeError(f"oracle library missing: {lib_path} (run make -C oracle)")
        L = ctypes.CDLL(lib_path)
        P = ctypes.c_void_p
        L.oracle_route.restype = P
        L.oracle_route.argtypes = [P, P, P, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                   ctypes.c_int, ctypes.c_int, ctypes.c_float, ctypes.c_int,
                                   ctypes.c_int]
        L.oracle_route_table.restype = ctypes.c_int
        L.oracle_route_table.argtypes = [P, ctypes.c_int, ctypes.POINTER(P),
                                         ctypes.POINTER(ctypes.c_long)]
        L.oracle_route_free.argtypes = [P]
        L.oracle_spmm_f64.argtypes = [P, P, P, ctypes.c_int, P, ctypes.c_int, P]
        L.oracle_spmm_f16_f32.argtypes = [P, P, P, ctypes.c_int, P, ctypes.c_int, P, ctypes.c_int]
        L.oracle_sddmm_f64.argtypes = [P, P, ctypes.c_int, P, P, ctypes.c_int, P]
        L.oracle_sddmm_f16_f32.argtypes = [P, P, ctypes.c_int, P, P, ctypes.c_int, P, ctypes.c_int]
        L.oracle_max_threads.restype = ctypes.c_int
        _lib = L
    return _lib


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _shape(tabs, window):
    """Apply the reference's tensor shapes (block_online.cpp:786-792, 863-865)."""
    g = tabs[21].shape[0]
    t = tabs[23].shape[0]
    tabs[17] = tabs[17].reshape(g, 4)
    tabs[18] = tabs[18].reshape(g, window)
    tabs[19] = tabs[19].reshape(g, window, 2)
    tabs[20] = tabs[20].reshape(g, window, 2)
    tabs[25] = tabs[25].reshape(t, 16)
    tabs[26] = tabs[26].reshape(t, 8, 4, 2)
    tabs[27] = tabs[27].reshape(t, 8)
    return tabs


def route(indptr, indices, values, partsize_t=32, partsize_c=32, shortsize=3, density=8,
          window=16, wide=16, tc_min_util=0.0, sptc_min_util=0.5, sptc_threshold=12,
          unit_min_nnz=None, skip_tc=None):
    """Restated router; returns the reference's 30-item list as numpy arrays.

    ``unit_min_nnz`` / ``skip_tc`` default to the reference's environment
    switches LIBRA_SPTC_UNIT_MIN_NNZ (2) and LIBRA_SKIP_TC (off)
    (block_online.cpp:564-567).  ``wide``, ``sptc_min_util`` and
    ``sptc_threshold`` are accepted and unused, as in the reference."""
    L = _load()
    if unit_min_nnz is None:
        unit_min_nnz = int(os.environ.get("LIBRA_SPTC_UNIT_MIN_NNZ", "2"))
    if skip_tc is None:
        skip_tc = os.environ.get("LIBRA_SKIP_TC", "0") in ("1", "true", "TRUE")
    rp = np.ascontiguousarray(indptr, dtype=np.int32)
    ci = np.ascontiguousarray(indices, dtype=np.int32)
    vv = np.ascontiguousarray(values, dtype=np.float32)
    t0 = time.perf_counter()
    h = L.oracle_route(_ptr(rp), _ptr(ci), _ptr(vv), rp.shape[0] - 1, partsize_t, partsize_c,
                       shortsize, density, window, float(tc_min_util), int(unit_min_nnz),
                       int(bool(skip_tc)))
    if not h:
        raise ValueError("oracle_route rejected its arguments")
    dur = time.perf_counter() - t0
    out = []
    try:
        for i, dt in enumerate(_DTYPES):
            data = ctypes.c_void_p()
            n = ctypes.c_long()
            L.oracle_route_table(h, i, ctypes.byref(data), ctypes.byref(n))
            cnt = n.value // np.dtype(dt).itemsize
            if cnt == 0:
                out.append(np.zeros(0, dtype=dt))
            else:
                buf = (ctypes.c_char * n.value).from_address(data.value)
                out.append(np.frombuffer(buf, dtype=dt, count=cnt).copy())
    finally:
        L.oracle_route_free(h)
    out = _shape(out, window)
    out.append(np.float32(dur))
    return out


def _ref_dir():
    return os.path.join(HERE, "_ref")


def ref_available():
    return bool(glob.glob(os.path.join(_ref_dir(), "Libra5BlockOnline*.so")))


_REF_MODULES = {}


def _load_ref(module):
    """A module of oracle/_ref loaded from its file, neither put on sys.path
    nor entered in sys.modules: the library's drop-in modules have the same
    names and must keep resolving to the library's own files."""
    if module not in _REF_MODULES:
        import importlib.util
        paths = (glob.glob(os.path.join(_ref_dir(), module + ".*.so")) +
                 glob.glob(os.path.join(_ref_dir(), module + ".so")))
        if not paths:
            raise ImportError(f"{module} not built under oracle/_ref")
        spec = importlib.util.spec_from_file_location(module, paths[0])
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        _REF_MODULES[module] = mod
    return _REF_MODULES[module]


def ref_route(indptr, indices, values, *args, quiet=True):
    """The reference router compiled from its own source (oracle/_ref).

    Same arguments as block_sptc_2to4_online; returns numpy arrays.  The
    reference prints per-window diagnostics on stdout; ``quiet`` drops them."""
    import torch
    Libra5BlockOnline = _load_ref("Libra5BlockOnline")     # built by oracle/Makefile
    rp = torch.from_numpy(np.ascontiguousarray(indptr, dtype=np.int32))
    ci = torch.from_numpy(np.ascontiguousarray(indices, dtype=np.int32))
    vv = torch.from_numpy(np.ascontiguousarray(values, dtype=np.float32))
    if quiet:
        sys.stdout.flush()
        fd = os.dup(1)
        devnull = os.open(os.devnull, os.O_WRONLY)
        os.dup2(devnull, 1)
    try:
        out = Libra5BlockOnline.block_sptc_2to4_online(rp, ci, vv, *args)
    finally:
        if quiet:
            sys.stdout.flush()
            os.dup2(fd, 1)
            os.close(fd)
            os.close(devnull)
    return [t.numpy() for t in out]


def ref_spmm_available():
    return bool(glob.glob(os.path.join(_ref_dir(), "Libra6SpMMOnline*.so")))


def check_sptc_tables(s_column, s_value, s_pos, s_window, window, dim_n, m_ori, k_ori):
    """Host checks that keep the reference's scalar 2:4 kernel
    (TR-source/SpMM/mGCNkernel_online.cu:250-337) inside its buffers: the
    operator itself checks shapes and dtypes (mGCN_online.cpp:202-300) but
    indexes a group's four columns with s_pos unchecked.  Raises ValueError."""
    groups = int(s_window.shape[0])
    if s_column.shape != (groups, 4) or s_value.shape != (groups, window, 2) or \
            s_pos.shape != (groups, window, 2):
        raise ValueError("SPTC table shapes disagree with s_window / window")
    if s_pos.size and (int(s_pos.min()) < -1 or int(s_pos.max()) > 3):
        raise ValueError("s_pos entries must lie in -1..3")
    if min(window, dim_n, m_ori, k_ori) <= 0:
        raise ValueError("window, dimN, mOri and kOri must be positive")
    if groups * window * 2 >= 2**31 or m_ori * dim_n >= 2**31 or k_ori * dim_n >= 2**31:
        raise ValueError("the reference kernel indexes with 32-bit ints")


def ref_sptc_online(s_column, s_value, s_pos, s_window, rhs, window, dim_n, m_ori, k_ori):
    """The reference's own scalar 2:4 SpMM operator, forward_fp16_sptc_online
    (TR-source/SpMM/mGCN_online.cpp:202-400), compiled from its sources for
    sm_100a into oracle/_ref (oracle/Makefile, ``ref-spmm``).  CPU tables and
    FP16 features in, FP32 [mOri, dimN] out; runs on the current GPU."""
    import torch
    check_sptc_tables(s_column, s_value, s_pos, s_window, window, dim_n, m_ori, k_ori)
    mod = _load_ref("Libra6SpMMOnline")
    t = [torch.from_numpy(np.ascontiguousarray(a)) for a in (s_column, s_value, s_pos, s_window)]
    b = torch.from_numpy(np.ascontiguousarray(rhs, dtype=np.float16))
    if b.numel() != k_ori * dim_n:
        raise ValueError("rhs must hold kOri * dimN values")
    out, _ms = mod.forward_fp16_sptc_online(*t, b, window, dim_n, m_ori, k_ori, 1)
    return out.numpy()


_PARALLEL_TABLES = ("t_row_offset", "t_block_offset", "t_column", "t_value", "t_window_row",
                    "t_atomic", "t_binary", "c_row_offset", "c_row", "c_atomic", "c_column",
                    "c_value", "c_row_offset_short", "c_row_short", "c_atomic_short",
                    "c_column_short", "c_value_short", "s_column", "s_value", "s_pos",
                    "s_offsets", "s_tile_window", "s_tile_column", "s_packed_a",
                    "s_packed_meta", "s_window_tile_offset")
_HALF_TABLES = ("t_value", "c_value", "c_value_short")


def check_cuda_route_tables(T, dim_n, m_ori, k_ori, partsize_c):
    """Host checks under which the reference's parallel operator
    (TR-source/SpMM/mGCN_online.cpp:760-1138) runs only its CUDA-route
    kernels (mGCNkernel.cu:976-1042 long, :1119-1171 short) and stays inside
    its buffers: no tensor-core parts (its TC kernel is then not launched,
    mGCNkernel_online.cu:1398) and no 2:4 tiles (its 2:4 kernel is not
    launched, :1509); exactly 128 features (each warp lane reads and writes
    four FP16 features, spmm_utils/compute.h:27-87, so a row must hold 128);
    long parts of at most 32 entries (one 32-thread block stages a part in
    shared memory sized by partsize_c); rows >= 0; columns in [0, kOri).
    Raises ValueError."""
    if dim_n != 128:
        raise ValueError("the reference's CUDA route reads exactly 128 features per row")
    if T["t_atomic"].size or T["s_column"].size or T["s_tile_column"].size:
        raise ValueError("tables must hold CUDA-route parts only")
    if not 0 < partsize_c <= 32:
        raise ValueError("partsize_c must lie in 1..32")
    if m_ori * dim_n >= 2**31 or k_ori * dim_n >= 2**31:
        raise ValueError("the reference kernels index with 32-bit ints")
    for sfx, cap in (("", partsize_c), ("_short", None)):
        ro, row = T["c_row_offset" + sfx], T["c_row" + sfx]
        col, val, at = T["c_column" + sfx], T["c_value" + sfx], T["c_atomic" + sfx]
        if len(ro) != len(row) + 1 or len(at) != len(row) or ro[0] != 0 or \
                ro[-1] != len(col) or len(val) != len(col) or (np.diff(ro) < 0).any():
            raise ValueError("inconsistent CUDA-route part tables" + sfx)
        if cap is not None and len(row) and np.diff(ro).max() > cap:
            raise ValueError("a long part holds more entries than partsize_c")
        if len(row) and row.min() < 0:
            raise ValueError("negative output row")
        if len(col) and (col.min() < 0 or col.max() >= k_ori):
            raise ValueError("column outside [0, kOri)")


def ref_parallel_cuda_route(T, rhs, window, dim_n, m_ori, k_ori, partsize_c):
    """The reference's parallel operator forward_fp16_tcu_cuda_sptc_mma_parallel_online
    (TR-source/SpMM/mGCN_online.cpp:760-1138) on tables that hold CUDA-route
    parts only (check_cuda_route_tables), compiled for sm_100a into
    oracle/_ref.  ``T`` maps table names to the router's numpy arrays.
    Returns the FP32 [mOri, dimN] output."""
    import torch
    check_cuda_route_tables(T, dim_n, m_ori, k_ori, partsize_c)
    mod = _load_ref("Libra6SpMMOnline")
    args = []
    for n in _PARALLEL_TABLES:
        a = np.ascontiguousarray(T[n])
        args.append(torch.from_numpy(a.astype(np.float16) if n in _HALF_TABLES else a))
    b = torch.from_numpy(np.ascontiguousarray(rhs, dtype=np.float16))
    if b.numel() != k_ori * dim_n:
        raise ValueError("rhs must hold kOri * dimN values")
    out = mod.forward_fp16_tcu_cuda_sptc_mma_parallel_online(
        *args, b, int(T["t_atomic"].shape[0]), int(T["c_atomic"].shape[0]), int(partsize_c),
        int(T["c_atomic_short"].shape[0]), window, dim_n, m_ori, k_ori, 1)
    return out[0].numpy()


def ref_match_available(module="matching_utils"):
    return bool(glob.glob(os.path.join(_ref_dir(), module + ".*.so")) +
                glob.glob(os.path.join(_ref_dir(), module + ".so")))


def ref_match(module, func, indptr, indices, values, quiet=True, **kw):
    """A matching-stats function of the reference compiled from its own
    source (oracle/_ref: matching_utils.match_2to4, matching_utils_hash.
    match_2to4_hash, matching_utils_bucket.match_2to4_bucket); returns its
    dict.  The reference prints a summary box on stdout; ``quiet`` drops it."""
    mod = _load_ref(module)
    rp = np.ascontiguousarray(indptr, dtype=np.int32)
    ci = np.ascontiguousarray(indices, dtype=np.int32)
    vv = np.ascontiguousarray(values, dtype=np.float32)
    if quiet:
        sys.stdout.flush()
        fd = os.dup(1)
        devnull = os.open(os.devnull, os.O_WRONLY)
        os.dup2(devnull, 1)
    try:
        return dict(getattr(mod, func)(rp, ci, vv, **kw))
    finally:
        if quiet:
            sys.stdout.flush()
            os.dup2(fd, 1)
            os.close(fd)
            os.close(devnull)


def _half(x):
    return np.asarray(x, dtype=np.float32).astype(np.float16)


def decode_sptc_tiles(tile_column, packed_a, packed_meta, window_tile_offset, window=16):
    """COO (rows, cols, fp16 values) of the packed mma.sp tiles (block_online.cpp:797-841):
    row group g, lane t -> half2 for rows g / g+8, chunk t, two positions from the meta
    nibbles.  Zero-valued padding slots are dropped."""
    rows, cols, vals = [], [], []
    pa = np.asarray(packed_a).reshape(-1, 8, 4, 2).view(np.uint32)
    pm = np.asarray(packed_meta).reshape(-1, 8).view(np.uint32)
    tc = np.asarray(tile_column).reshape(-1, 16)
    wto = np.asarray(window_tile_offset)
    tile_win = np.repeat(np.arange(len(wto) - 1), np.diff(wto))
    for t in range(tc.shape[0]):
        w = int(tile_win[t])
        for g in range(8):
            meta = int(pm[t, g])
            for ch in range(4):
                for half_sel, r in ((0, g), (1, g + 8)):
                    word = int(pa[t, g, ch, half_sel])
                    nib = (meta >> (16 * half_sel + 4 * ch)) & 0xF
                    for slot, pos in ((0, nib & 3), (1, (nib >> 2) & 3)):
                        bits = (word >> (16 * slot)) & 0xFFFF
                        v = np.array([bits], dtype=np.uint16).view(np.float16)[0]
                        if v == 0:
                            continue
                        c = int(tc[t, ch * 4 + pos])
                        rows.append(w * window + r)
                        cols.append(c)
                        vals.append(v)
    return (np.array(rows, dtype=np.int64), np.array(cols, dtype=np.int64),
            np.array(vals, dtype=np.float16))


def decode_tables(tabs, n_rows, n_cols, window=16, sptc_from="pos"):
    """Rebuild the routed operand from the reference's route tables.

    Returns a dict of scipy CSR matrices with FP16-rounded values stored as
    float64: 'tc', 'sptc', 'cuda' and 'all' (their sum).  ``sptc_from`` picks
    the SPTC source: 'pos' decodes s_value/s_pos (what the scalar kernel
    reads, mGCNkernel_online.cu:250-337); 'tiles' decodes the packed tiles
    (what the mma.sp kernel reads)."""
    T = dict(zip(TABLE_NAMES, tabs))
    # TC sub-blocks: bit = row*8 + k in binary_lo (rows 0-7) / binary_hi (rows 8-15);
    # values in bit order (block_online.cpp:462-488); part -> window via t_window_row.
    r_l, c_l, v_l = [], [], []
    t_row = T["t_row_offset"]
    t_blk = T["t_block_offset"]
    t_bin = T["t_binary"].view(np.uint64)
    for p in range(len(t_row) - 1):
        base_row = int(T["t_window_row"][p])
        for s in range(int(t_row[p]), int(t_row[p + 1])):
            lo, hi = int(t_bin[2 * s]), int(t_bin[2 * s + 1])
            off = int(t_blk[s])
            n = 0
            for half_idx, word in ((0, lo), (1, hi)):
                for bit in range(64):
                    if (word >> bit) & 1:
                        r = base_row + half_idx * 8 + bit // 8
                        c = int(T["t_column"][s * 8 + bit % 8])
                        r_l.append(r); c_l.append(c); v_l.append(T["t_value"][off + n])
                        n += 1
            assert n == int(t_blk[s + 1]) - off, "TC value count != bitmap popcount"
    tc = sp.csr_matrix((_half(v_l).astype(np.float64), (r_l, c_l)), shape=(n_rows, n_cols))

    if sptc_from == "pos":
        cols4 = T["s_column"].reshape(-1, 4)
        pos = T["s_pos"].reshape(cols4.shape[0], window, 2)
        sval = T["s_value"].reshape(cols4.shape[0], window, 2)
        g_idx, lr, slot = np.nonzero(pos >= 0)
        rr = T["s_window"][g_idx].astype(np.int64) * window + lr
        cc = cols4[g_idx, pos[g_idx, lr, slot]]
        vv = _half(sval[g_idx, lr, slot]).astype(np.float64)
        keep = rr < n_rows
        sptc = sp.csr_matrix((vv[keep], (rr[keep], cc[keep])), shape=(n_rows, n_cols))
    else:
        rr, cc, vv = decode_sptc_tiles(T["s_tile_column"], T["s_packed_a"], T["s_packed_meta"],
                                       T["s_window_tile_offset"], window)
        sptc = sp.csr_matrix((vv.astype(np.float64), (rr, cc)), shape=(n_rows, n_cols))

    rr, cc, vv = [], [], []
    for pre in ("", "_short"):
        off = T["c_row_offset" + pre]
        rows = T["c_row" + pre]
        cnt = np.diff(off)
        rr.append(np.repeat(rows, cnt))
        cc.append(T["c_column" + pre])
        vv.append(_half(T["c_value" + pre]).astype(np.float64))
    cuda = sp.csr_matrix((np.concatenate(vv), (np.concatenate(rr), np.concatenate(cc))),
                         shape=(n_rows, n_cols))
    total = (tc + sptc + cuda).tocsr()
    return {"tc": tc, "sptc": sptc, "cuda": cuda, "all": total}


def decode_plan(P):
    """Rebuild the matrix a device plan multiplies, from its host arrays (the
    dict of trspmm.host_plan; layout in tr-spmm_b200/csrc/plan.h): tile
    element (n, k) of tile t sits at (n//8)*128 + (k//8)*64 + (n%8)*8 + k%8
    and multiplies B[tile_col[t*16+k]] into plan row 16*w + n; residual
    entries are CSR over plan rows; every plan row r is scaled by
    row_scale[r] and lands in output row row_out[r].  Returns CSR float64
    matrices {'tc', 'sptc', 'prom' (tile parts), 'res', 'all'} in the output
    row space, values as the kernels see them (FP16 x FP32 scale)."""
    n_rows, n_cols = int(P["n_rows"]), int(P["n_cols"])
    if len(P.get("blk_order", ())):
        return decode_block_plan(P)
    wt, split, prom = P["win_tile"], P["win_split"], P["win_prom"]
    W = len(wt) - 1
    a = P["tile_a"].view(np.float16).astype(np.float64)
    cols = P["tile_col"]
    scale = P["row_scale"].astype(np.float64)
    out = P["row_out"]
    i = np.arange(256)
    n_of = (i // 128) * 8 + (i % 64) // 8
    k_of = ((i % 128) // 64) * 8 + (i % 8)
    parts = {"tc": [], "sptc": [], "prom": []}
    for w in range(W):
        for t in range(int(wt[w]), int(wt[w + 1])):
            key = "tc" if t < split[w] else ("sptc" if t < prom[w] else "prom")
            vals = a[t * 256:(t + 1) * 256]
            nz = np.nonzero(vals)[0]
            if nz.size == 0:
                continue
            c = cols[t * 16 + k_of[nz]]
            assert (c >= 0).all(), "non-zero tile element in an empty column slot"
            prow = w * 16 + n_of[nz]
            parts[key].append((prow, c, vals[nz]))

    def to_csr(lst):
        if not lst:
            return sp.csr_matrix((n_rows, n_cols))
        pr = np.concatenate([x[0] for x in lst])
        cc = np.concatenate([x[1] for x in lst])
        vv = np.concatenate([x[2] for x in lst]) * scale[pr]
        orow = out[pr]
        assert (orow >= 0).all(), "tile entry in a padding row"
        return sp.csr_matrix((vv, (orow, cc)), shape=(n_rows, n_cols))

    mats = {k: to_csr(v) for k, v in parts.items()}
    rp = P["res_ptr"]
    cnt = np.diff(rp)
    pr = np.repeat(np.arange(len(cnt)), cnt)
    rv = P["res_val"].view(np.float16).astype(np.float64) * scale[pr]
    assert (out[pr] >= 0).all(), "residual entry in a padding row"
    res = sp.csr_matrix((rv, (out[pr], P["res_col"])), shape=(n_rows, n_cols))
    total = (mats["tc"] + mats["sptc"] + mats["prom"] + res).tocsr()
    return {"tc": mats["tc"], "sptc": mats["sptc"], "prom": mats["prom"], "res": res,
            "all": total}


def decode_block_plan(P):
    """The matrix a block-layout plan multiplies (layout in
    tr-spmm_b200/csrc/plan.h): chunk c of block b multiplies B[chunk_col[16c
    + k]] into plan row 128b + m for every entry at byte offset
    (m//8)*256 + (k//8)*128 + (m%8)*16 + (k%8)*2 of its A tile; plan row r is
    scaled by row_scale[r] and lands in output row row_out[r].  Also checks
    that no two entries of a chunk share a tile position and that every
    entry's slot holds a column.  Returns {'block', 'all'} (CSR float64)."""
    n_rows, n_cols = int(P["n_rows"]), int(P["n_cols"])
    bc, cc, ce = P["blk_chunk"], P["chunk_col"], P["chunk_ent"]
    pos = P["ent_pos"].astype(np.int64)
    m = (pos >> 8) * 8 + ((pos >> 4) & 7)
    k = ((pos >> 7) & 1) * 8 + ((pos >> 1) & 7)
    assert ((pos & 1) == 0).all() and (pos < 4096).all(), "entry outside its A tile"
    n_chunks = len(ce) - 1
    chunk_of = np.repeat(np.arange(n_chunks), np.diff(ce))
    blk_of_chunk = np.repeat(np.arange(len(bc) - 1), np.diff(bc))
    blk = blk_of_chunk[chunk_of]
    cols = cc[chunk_of * 16 + k]
    assert (cols >= 0).all(), "entry in an empty column slot"
    key = chunk_of * 4096 + pos
    assert np.unique(key).size == key.size, "two entries at one tile position"
    prow = blk * 128 + m
    out = P["row_out"]
    assert (out[prow] >= 0).all(), "entry in a padding row"
    vv = P["ent_val"].view(np.float16).astype(np.float64) * P["row_scale"].astype(np.float64)[prow]
    mat = sp.csr_matrix((vv, (out[prow], cols)), shape=(n_rows, n_cols))
    return {"block": mat, "all": mat}


def plan_value_of_entries(P):
    """Value the plan holds for each CSR entry of A (via val_slot), FP16 x
    row scale, NaN where an entry has no slot."""
    if len(P.get("blk_order", ())):
        slot = P["val_slot"].astype(np.int64)
        v = np.full(slot.shape, np.nan)
        has = slot >= 0
        v[has] = P["ent_val"].view(np.float16).astype(np.float64)[slot[has]]
        v[has] *= P["row_scale"][P["edge_row"][has]]
        return v
    T = len(P["tile_col"]) // 16
    slot = P["val_slot"].astype(np.int64)
    a = P["tile_a"].view(np.float16).astype(np.float64)
    r = P["res_val"].view(np.float16).astype(np.float64)
    v = np.full(slot.shape, np.nan)
    t = (slot >= 0) & (slot < T * 256)
    v[t] = a[slot[t]]
    q = slot >= T * 256
    v[q] = r[slot[q] - T * 256]
    has = slot >= 0
    v[has] *= P["row_scale"][P["edge_row"][has]]
    return v


def max_threads():
    return _load().oracle_max_threads()


def spmm_f64(indptr, indices, values, b):
    """C = A·B in FP64 (C restatement, OpenMP)."""
    L = _load()
    rp = np.ascontiguousarray(indptr, dtype=np.int32)
    ci = np.ascontiguousarray(indices, dtype=np.int32)
    vv = np.ascontiguousarray(values, dtype=np.float64)
    bb = np.ascontiguousarray(b, dtype=np.float64)
    m, k = rp.shape[0] - 1, bb.shape[1]
    c = np.empty((m, k), dtype=np.float64)
    L.oracle_spmm_f64(_ptr(rp), _ptr(ci), _ptr(vv), m, _ptr(bb), k, _ptr(c))
    return c


def spmm_f16_f32(indptr, indices, values_f16, b_f16, threads=0, out=None):
    """C = A·B with FP16 operands, FP32 accumulation (C restatement, OpenMP)."""
    L = _load()
    rp = np.ascontiguousarray(indptr, dtype=np.int32)
    ci = np.ascontiguousarray(indices, dtype=np.int32)
    vv = np.ascontiguousarray(values_f16, dtype=np.float16)
    bb = np.ascontiguousarray(b_f16, dtype=np.float16)
    m, k = rp.shape[0] - 1, bb.shape[1]
    c = out if out is not None else np.empty((m, k), dtype=np.float32)
    L.oracle_spmm_f16_f32(_ptr(rp), _ptr(ci), _ptr(vv), m, _ptr(bb), k, _ptr(c), int(threads))
    return c


def sddmm_f16_f32(indptr, indices, dc_f16, b_f16, threads=0, out=None):
    """dval[e] = <dC[row(e)], B[col(e)]> with FP16 operands, FP32 sums (OpenMP)."""
    L = _load()
    rp = np.ascontiguousarray(indptr, dtype=np.int32)
    ci = np.ascontiguousarray(indices, dtype=np.int32)
    g = np.ascontiguousarray(dc_f16, dtype=np.float16)
    bb = np.ascontiguousarray(b_f16, dtype=np.float16)
    o = out if out is not None else np.empty(ci.shape[0], dtype=np.float32)
    L.oracle_sddmm_f16_f32(_ptr(rp), _ptr(ci), rp.shape[0] - 1, _ptr(g), _ptr(bb), g.shape[1],
                           _ptr(o), int(threads))
    return o


def sddmm_f64(indptr, indices, dc, b):
    """dval[e] = <dC[row(e)], B[col(e)]> in FP64."""
    L = _load()
    rp = np.ascontiguousarray(indptr, dtype=np.int32)
    ci = np.ascontiguousarray(indices, dtype=np.int32)
    g = np.ascontiguousarray(dc, dtype=np.float64)
    bb = np.ascontiguousarray(b, dtype=np.float64)
    out = np.empty(ci.shape[0], dtype=np.float64)
    L.oracle_sddmm_f64(_ptr(rp), _ptr(ci), rp.shape[0] - 1, _ptr(g), _ptr(bb), g.shape[1],
                       _ptr(out))
    return out
