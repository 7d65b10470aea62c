"""The reference's own SpMM operators against this library's drop-in, on the
same route tables and FP16 features, for the two routes whose reference
kernels read as correct and in bounds.

oracle/_ref/Libra6SpMMOnline is the reference's operator module compiled
from its own sources for sm_100a (oracle/Makefile, target ``ref-spmm``); the
tests skip where it was not built.

- forward_fp16_sptc_online (TR-source/SpMM/mGCN_online.cpp:202-400, kernel
  TR-source/SpMM/mGCNkernel_online.cu:250-337), the scalar 2:4 operator: its
  loads and stores are checked against mOri, dimN and kOri, and the one
  unchecked index, s_pos into a group's four columns, is checked on the host
  before the call (oracle.check_sptc_tables).
- forward_fp16_tcu_cuda_sptc_mma_parallel_online (mGCN_online.cpp:760-1138)
  on tables routed to CUDA parts only, at K = 128: its tensor-core and 2:4
  kernels are then not launched, and its CUDA-route kernels stay in bounds
  under the conditions oracle.check_cuda_route_tables checks first.

Tolerances (2:4 operator).  The pin is the 1e-2 relative error (max |C - C_ref| / max
|C_ref|) that the reference's own output is held to.  Tighter: the reference
multiplies the FP32 values of s_value, this library's operator their FP16
roundings (the plan it builds from the group tables has no row scale); the
two GPU outputs may differ by the FP64 difference between those two value
sets on the same tables (computed here on the CPU) plus FP32 accumulation
rounding on each side (2e-4).  The
reference's output also equals the FP64 product of its FP32-valued tables to
1e-4.
"""
import numpy as np
import pytest
import scipy.sparse as sp
import torch

import oracle
import trspmm
from helpers import rel_err, spmm_ref
from trspmm import graphs

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not oracle.ref_spmm_available(),
                                 reason="reference SpMM operator not built under oracle/_ref")]

TOL_PIN = 1e-2
TOL_ACC = 2e-4


def _sptc_f64(T, n_rows, n_cols, window=16, round_half=False):
    """The SPTC part of the tables with FP64 values: FP32 as stored, or rounded
    to FP16 first."""
    cols4 = T["s_column"].reshape(-1, 4)
    pos = T["s_pos"].reshape(cols4.shape[0], window, 2)
    val = T["s_value"].reshape(cols4.shape[0], window, 2)
    g, lr, slot = np.nonzero(pos >= 0)
    rr = T["s_window"][g].astype(np.int64) * window + lr
    cc = cols4[g, pos[g, lr, slot]]
    vv = val[g, lr, slot]
    if round_half:
        vv = vv.astype(np.float16)
    keep = (rr < n_rows) & (cc >= 0) & (cc < n_cols)
    return sp.csr_matrix((vv[keep].astype(np.float64), (rr[keep], cc[keep])), shape=(n_rows, n_cols))


GRAPHS = {
    "sbm": lambda: graphs.sbm_powerlaw(n=3000, avg_degree=16, communities=30, seed=8),
    "route_mix": lambda: graphs.route_mix(n=2048, target_nnz=100_000),
    "chung_lu": lambda: graphs.chung_lu(n=4096),
    "ragged": lambda: graphs.random_csr(1000, 777, 0.01, seed=3, empty_rows=0.3),
    "partial_window": lambda: graphs.random_csr(33, 50, 0.1, seed=2),
    "no_entries": lambda: graphs.random_csr(37, 20, 0.0, seed=1),
}


@pytest.mark.parametrize("k", [64, 128, 40])
@pytest.mark.parametrize("name", list(GRAPHS))
def test_sptc_operator_matches_reference(cuda, name, k):
    import Libra6SpMMOnline as L6
    g = GRAPHS[name]()
    tabs = trspmm.route(g.indptr, g.indices, g.values)
    T = dict(zip(trspmm.TABLE_NAMES, tabs))
    b = graphs.dense_features(g.n_cols, k, seed=4)
    ref = oracle.ref_sptc_online(T["s_column"], T["s_value"], T["s_pos"], T["s_window"], b, 16, k,
                                 g.n_rows, g.n_cols)
    Tt = {n: torch.from_numpy(np.ascontiguousarray(T[n]))
          for n in ("s_column", "s_value", "s_pos", "s_window")}
    out, _ = L6.forward_fp16_sptc_online(Tt["s_column"], Tt["s_value"], Tt["s_pos"],
                                         Tt["s_window"], torch.from_numpy(b), 16, k, g.n_rows,
                                         g.n_cols, 1)
    out = out.numpy()
    assert out.shape == ref.shape == (g.n_rows, k)
    c32 = spmm_ref(_sptc_f64(T, g.n_rows, g.n_cols), b)
    c16 = spmm_ref(_sptc_f64(T, g.n_rows, g.n_cols, round_half=True), b)
    if not np.abs(c32).max() > 0:
        assert not np.abs(ref).max() and not np.abs(out).max()
        return
    assert rel_err(ref, c32) <= 1e-4
    gap = rel_err(c16, c32)
    err = rel_err(out, ref)
    assert err <= TOL_PIN
    assert err <= gap + TOL_ACC, (err, gap)



CUDA_ROUTE_GRAPHS = {
    "sbm": GRAPHS["sbm"],
    "route_mix": GRAPHS["route_mix"],
    "chung_lu": GRAPHS["chung_lu"],
    "ragged": GRAPHS["ragged"],
    "partial_window": GRAPHS["partial_window"],
}


@pytest.mark.parametrize("name", list(CUDA_ROUTE_GRAPHS))
def test_cuda_route_matches_reference_at_k128(cuda, name):
    """The reference's parallel operator on tables routed to its CUDA route
    alone (long and short parts; its TC and 2:4 kernels are not launched),
    at the one feature width its CUDA-route kernels are written for, 128,
    against this library's drop-in on the same tables.  The reference
    accumulates each part in FP16, so only the 1e-2 pin applies between the
    two; this library's output also equals the FP64 product of the tables to
    1e-4."""
    import Libra6SpMMOnline as L6
    g = CUDA_ROUTE_GRAPHS[name]()
    k = 128
    tabs = trspmm.route(g.indptr, g.indices, g.values, skip_tc=True, skip_sptc=True)
    T = dict(zip(trspmm.TABLE_NAMES, tabs))
    b = graphs.dense_features(g.n_cols, k, seed=4)
    ref = oracle.ref_parallel_cuda_route(T, b, 16, k, g.n_rows, g.n_cols, 32)
    args = []
    for n in oracle.core._PARALLEL_TABLES:
        a = np.ascontiguousarray(T[n])
        args.append(torch.from_numpy(a.astype(np.float16) if n in oracle.core._HALF_TABLES else a))
    res = L6.forward_fp16_tcu_cuda_sptc_mma_parallel_online(
        *args, torch.from_numpy(b), int(T["t_atomic"].shape[0]), int(T["c_atomic"].shape[0]), 32,
        int(T["c_atomic_short"].shape[0]), 16, k, g.n_rows, g.n_cols, 1)
    out = res[0].numpy()
    assert out.shape == ref.shape == (g.n_rows, k)
    dec = oracle.decode_tables(tabs, g.n_rows, g.n_cols)
    c64 = spmm_ref(dec["all"], b)
    assert rel_err(out, c64) <= 1e-4
    err = rel_err(out, ref)
    assert err <= TOL_PIN, (err, rel_err(ref, c64))
