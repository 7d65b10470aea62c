"""GPU parity of the sm_100a kernels against the FP64 oracle.

Tolerances (stated per the path's FP16-in / FP32-accumulate contract):
  FP32 output: max |C - C64| / max |C64| <= 1e-4  (accumulation-order rounding)
  FP16 output: <= 2e-3                             (one FP16 rounding of C)
The FP64 reference uses the same FP16-rounded A values and B.
"""
import numpy as np
import pytest
import torch

import oracle
import trspmm
from helpers import half_csr, rel_err, spmm_ref
from trspmm import graphs

pytestmark = pytest.mark.gpu

TOL32 = 1e-4
TOL16 = 2e-3


def _dev(g, b, cuda):
    return (torch.from_numpy(g.indptr).to(cuda), torch.from_numpy(g.indices).to(cuda),
            torch.from_numpy(g.values.astype(np.float16)).to(cuda), torch.from_numpy(b).to(cuda))


GRAPHS = {
    "chung_lu": lambda: graphs.chung_lu(n=4096),
    "ragged": lambda: graphs.random_csr(1000, 777, 0.01, seed=3, empty_rows=0.3),
    "route_mix": lambda: graphs.route_mix(n=2048, target_nnz=100_000),
    "sbm": lambda: graphs.sbm_powerlaw(n=6000, avg_degree=30, communities=60),
    "single_row": lambda: graphs.random_csr(1, 300, 0.5, seed=5),
}


@pytest.mark.parametrize("name", list(GRAPHS))
@pytest.mark.parametrize("k", [8, 64, 128, 256, 24, 200, 12, 520])
@pytest.mark.parametrize("out_dtype", [torch.float32, torch.float16])
def test_csr_kernel(cuda, name, k, out_dtype):
    g = GRAPHS[name]()
    b = graphs.dense_features(g.n_cols, k, seed=k)
    ip, ix, iv, bd = _dev(g, b, cuda)
    out = trspmm.spmm_csr(ip, ix, iv, bd, g.n_rows, out_dtype=out_dtype)
    torch.cuda.synchronize()
    ref = spmm_ref(half_csr(g.indptr, g.indices, g.values, g.n_rows, g.n_cols), b)
    tol = TOL32 if out_dtype == torch.float32 else TOL16
    assert rel_err(out.float().cpu().numpy(), ref) <= tol


@pytest.mark.parametrize("name", ["chung_lu", "ragged", "route_mix", "sbm"])
@pytest.mark.parametrize("k", [64, 128, 256, 40])
def test_routed_compat_tables_per_route(cuda, name, k):
    """The plan built from the reference-layout tables computes exactly what
    the tables encode, route by route (TC, SPTC, CUDA) and in total."""
    g = GRAPHS[name]()
    tabs = trspmm.route(g.indptr, g.indices, g.values)
    dec = oracle.decode_tables(tabs, g.n_rows, g.n_cols)
    plan = trspmm.Plan.from_tables(tabs, g.n_rows, g.n_cols)
    b = graphs.dense_features(g.n_cols, k, seed=1)
    bd = torch.from_numpy(b).to(cuda)
    for mask, key in ((trspmm.TR_ROUTE_TC, "tc"), (trspmm.TR_ROUTE_SPTC, "sptc"),
                      (trspmm.TR_ROUTE_CUDA, "cuda"), (trspmm.TR_ROUTE_ALL, "all")):
        out = plan.spmm(bd, route_mask=mask)
        torch.cuda.synchronize()
        ref = spmm_ref(dec[key], b)
        if np.abs(ref).max() == 0:
            assert np.abs(out.cpu().numpy()).max() == 0, key
        else:
            assert rel_err(out.cpu().numpy(), ref) <= TOL32, key


@pytest.mark.parametrize("name", ["chung_lu", "route_mix", "sbm", "ragged"])
@pytest.mark.parametrize("out_dtype", [torch.float32, torch.float16])
def test_routed_exact_plan_equals_full_product(cuda, name, out_dtype):
    g = GRAPHS[name]()
    plan = trspmm.Plan.from_csr(g.indptr, g.indices, g.values, g.n_rows, g.n_cols)
    assert plan.info["nnz"] == g.nnz or plan.info["nnz"] <= g.nnz
    b = graphs.dense_features(g.n_cols, 128, seed=2)
    out = plan.spmm(torch.from_numpy(b).to(cuda), out_dtype=out_dtype)
    torch.cuda.synchronize()
    ref = spmm_ref(half_csr(g.indptr, g.indices, g.values, g.n_rows, g.n_cols), b)
    tol = TOL32 if out_dtype == torch.float32 else TOL16
    assert rel_err(out.float().cpu().numpy(), ref) <= tol


def test_routed_dense_tiles_tensor_core(cuda):
    """A matrix that routes almost entirely to dense TC tiles: checks the
    tcgen05 path (operand layouts, TMEM read-back) on its own."""
    g = graphs.route_mix(n=1024, target_nnz=60_000, frac_dense=0.95, frac_24=0.0)
    tabs = trspmm.route(g.indptr, g.indices, g.values, density=4)
    dec = oracle.decode_tables(tabs, g.n_rows, g.n_cols)
    assert dec["tc"].nnz > 0.5 * g.nnz
    plan = trspmm.Plan.from_tables(tabs, g.n_rows, g.n_cols)
    for k in (128, 64, 256, 136):
        b = graphs.dense_features(g.n_cols, k, seed=k)
        out = plan.spmm(torch.from_numpy(b).to(cuda), route_mask=trspmm.TR_ROUTE_TC)
        torch.cuda.synchronize()
        assert rel_err(out.cpu().numpy(), spmm_ref(dec["tc"], b)) <= TOL32, k


def test_dropin_parallel_forward(cuda):
    """Libra6SpMMOnline.forward_fp16_tcu_cuda_sptc_mma_parallel_online through
    the tr_csr_fp16 dataset object, against the FP64 product of its tables."""
    from tr_csr_fp16.mdataset2_online import GCN_dataset_tcu_sptc_cuda_online
    from tr_csr_fp16.test_tr_csr_online import kernel_tcu_sptc_cuda_online
    g = graphs.route_mix(n=1024, target_nnz=50_000)
    ds = GCN_dataset_tcu_sptc_cuda_online.from_csr(g.indptr, g.indices, g.n_cols, 128,
                                                   values=g.values)
    x, ms, _, kind = kernel_tcu_sptc_cuda_online(ds, 3)
    assert kind == "parallel_mma" and ms.item() > 0
    names = ["t_rowNew_offsetTensor", "t_blockTensor", "t_columnTensor", "t_valueTensor",
             "t_window_rowTensor", "t_atomicTensor", "t_binaryTensor", "c_row_offsetTensor",
             "c_rowTensor", "c_atomicTensor", "c_colTensor", "c_valueTensor",
             "c_row_offsetTensor_short", "c_rowTensor_short", "c_atomicTensor_short",
             "c_colTensor_short", "c_valueTensor_short", "s_columnTensor", "s_maskTensor",
             "s_valueTensor", "s_posTensor", "s_windowTensor", "s_offsetTensor",
             "s_tile_windowTensor", "s_tile_groupTensor", "s_tile_columnTensor",
             "s_packed_aTensor", "s_packed_metaTensor", "s_window_tile_offsetTensor"]
    tabs = [getattr(ds, n).float().numpy() if n in ("t_valueTensor", "c_valueTensor",
                                                      "c_valueTensor_short")
            else getattr(ds, n).numpy() for n in names]
    dec = oracle.decode_tables(tabs, ds.num_nodes, ds.num_nodes_dst)
    ref = spmm_ref(dec["all"], ds.x.numpy())[: ds.num_nodes_ori]
    assert x.dtype == torch.float32 and tuple(x.shape) == (ds.num_nodes_ori, 128)
    assert rel_err(x.numpy(), ref) <= TOL32


def test_dropin_sptc_only_entry_points(cuda):
    import Libra6SpMMOnline as L6
    g = graphs.sbm_powerlaw(n=3000, avg_degree=16, communities=30, seed=8)
    tabs = trspmm.route(g.indptr, g.indices, g.values)
    dec = oracle.decode_tables(tabs, g.n_rows, g.n_cols)
    b = torch.from_numpy(graphs.dense_features(g.n_cols, 64, seed=4))
    ref = spmm_ref(dec["sptc"], b.numpy())
    T = dict(zip(trspmm.TABLE_NAMES, [torch.from_numpy(np.ascontiguousarray(t)) if
                                      isinstance(t, np.ndarray) else t for t in tabs]))
    out, ms = L6.forward_fp16_sptc_online(T["s_column"], T["s_value"], T["s_pos"], T["s_window"],
                                          b, 16, 64, g.n_rows, g.n_cols, 2)
    assert rel_err(out.numpy(), ref) <= TOL32 and ms.item() > 0
    out, ms = L6.forward_fp16_sptc_mma_online(T["s_column"], T["s_value"], T["s_pos"],
                                              T["s_offsets"], b, 16, 64, g.n_rows, g.n_cols, 2)
    assert rel_err(out.numpy(), ref) <= TOL32
    out, ms = L6.forward_fp16_sptc_mma_packed_online(T["s_tile_column"], T["s_packed_a"],
                                                     T["s_packed_meta"], T["s_window_tile_offset"],
                                                     b, 16, 64, g.n_rows, g.n_cols, 2)
    assert rel_err(out.numpy(), ref) <= TOL32
    with pytest.raises(RuntimeError):
        L6.forward_fp16_sptc_mma_packed_online(T["s_tile_column"], T["s_packed_a"],
                                               T["s_packed_meta"], T["s_window_tile_offset"],
                                               b, 16, 64, g.n_rows, g.n_cols + 1, 2)


def test_edge_cases(cuda):
    # no entries at all, a partial last window, K = 8
    for g in (graphs.random_csr(37, 20, 0.0, seed=1), graphs.random_csr(33, 50, 0.1, seed=2)):
        b = graphs.dense_features(g.n_cols, 8)
        plan = trspmm.Plan.from_csr(g.indptr, g.indices, g.values, g.n_rows, g.n_cols)
        out = plan.spmm(torch.from_numpy(b).to(cuda))
        ip, ix, iv, bd = _dev(g, b, cuda)
        out2 = trspmm.spmm_csr(ip, ix, iv, bd, g.n_rows)
        torch.cuda.synchronize()
        ref = spmm_ref(half_csr(g.indptr, g.indices, g.values, g.n_rows, g.n_cols), b)
        assert np.allclose(out.cpu().numpy(), ref, atol=1e-5)
        assert np.allclose(out2.cpu().numpy(), ref, atol=1e-5)


def test_bad_device_arguments_raise(cuda):
    g = graphs.random_csr(40, 40, 0.1)
    plan = trspmm.Plan.from_csr(g.indptr, g.indices, g.values, g.n_rows, g.n_cols)
    with pytest.raises(RuntimeError):
        plan.spmm(torch.zeros((41, 8), dtype=torch.float16, device=cuda))
    for dt in (torch.float64, torch.bfloat16):       # FP32 B is the FP32-feature route
        with pytest.raises(RuntimeError):
            plan.spmm(torch.zeros((40, 8), dtype=dt, device=cuda))
    with pytest.raises(RuntimeError):
        plan.spmm(torch.zeros((41, 8), dtype=torch.float32, device=cuda))
    tabs = trspmm.route(g.indptr, g.indices, g.values)
    for idx in (10, 15, 25):          # CUDA long / short / SPTC tile columns out of range
        if tabs[idx].size == 0:
            continue
        bad = list(tabs)
        bad[idx] = np.where(tabs[idx] >= 0, tabs[idx] + 1000, tabs[idx]).astype(np.int32)
        with pytest.raises(RuntimeError, match="out of range"):
            trspmm.Plan.from_tables(bad, g.n_rows, g.n_cols)
    assert tabs[25].size > 0


def test_large_routed_workload_properties(cuda):
    """Full-size 200k-node workload: routed (exact) == plain CSR on the GPU,
    and the column-sum identity 1^T (A B) = (1^T A) B holds against FP64."""
    g, b = graphs.make_workload("large_routed")
    plan = trspmm.Plan.from_csr(g.indptr, g.indices, g.values, g.n_rows, g.n_cols)
    bd = torch.from_numpy(b).to(cuda)
    out = plan.spmm(bd)
    ip, ix, iv, _ = _dev(g, b, cuda)
    out2 = trspmm.spmm_csr(ip, ix, iv, bd, g.n_rows)
    torch.cuda.synchronize()
    assert rel_err(out.cpu().numpy(), out2.cpu().numpy()) <= 1e-5
    A = half_csr(g.indptr, g.indices, g.values, g.n_rows, g.n_cols)
    colsum = np.asarray(A.sum(axis=0)).ravel() @ b.astype(np.float64)
    got = out.double().sum(dim=0).cpu().numpy()
    assert rel_err(got, colsum) <= 1e-5
    # a sample of full rows against FP64
    rows = np.random.default_rng(0).choice(g.n_rows, 2000, replace=False)
    ref = A[rows] @ b.astype(np.float64)
    assert rel_err(out.cpu().numpy()[rows], ref) <= TOL32


def test_blocks_with_fewer_entries_than_warps(cuda):
    """Row blocks / windows holding 1-7 entries (fewer than the CTA's 8 warps),
    through the plain kernel and every route of the routed kernel."""
    rng = np.random.default_rng(11)
    n = 160
    rows = np.repeat(np.arange(0, n, 16), 3) + rng.integers(0, 16, size=3 * (n // 16))
    cols = rng.integers(0, 300, size=rows.shape[0])
    key = np.unique(rows.astype(np.int64) * 300 + cols)
    r, c = key // 300, (key % 300).astype(np.int32)
    indptr = np.zeros(n + 1, np.int64)
    indptr[1:] = np.cumsum(np.bincount(r, minlength=n))
    g = graphs.Graph(indptr.astype(np.int32), c, rng.uniform(-1, 1, c.shape[0]).astype(np.float32),
                     n, 300)
    A = half_csr(g.indptr, g.indices, g.values, n, 300)
    for k in (64, 128, 256):
        b = graphs.dense_features(300, k, seed=k)
        ip, ix, iv, bd = _dev(g, b, cuda)
        out = trspmm.spmm_csr(ip, ix, iv, bd, n)
        plan = trspmm.Plan.from_csr(g.indptr, g.indices, g.values, n, 300)
        outs = [plan.spmm(bd, route_mask=m) for m in (trspmm.TR_ROUTE_CUDA, trspmm.TR_ROUTE_ALL)]
        torch.cuda.synchronize()
        ref = spmm_ref(A, b)
        assert rel_err(out.cpu().numpy(), ref) <= TOL32
        assert rel_err(outs[1].cpu().numpy(), ref) <= TOL32
