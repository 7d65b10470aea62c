"""GPU parity of the block engine (engine="block": every entry on tcgen05 over
128-row blocks) against the FP64 product of the matrix the plan encodes.

Tolerances, as for the routed kernels (FP16 operands, FP32 accumulation):
  FP32 output: max |C - C64| / max |C64| <= 1e-4
  FP16 output: <= 2e-3
  FP32 features (CUDA-core block kernel, FP32 arithmetic): <= 1e-5
The plan's own values (FP16 x FP32 row scale) are decoded on the CPU by the
oracle (oracle.decode_plan), so the check covers the kernels alone; the
layout itself is checked against A in tests/test_block_plan.py.
"""
import numpy as np
import pytest
import torch

import oracle
import trspmm
from helpers import rel_err
from trspmm import graphs

pytestmark = pytest.mark.gpu

TOL32 = 1e-4
TOL16 = 2e-3

GRAPHS = {
    "chung_lu": lambda: graphs.chung_lu(n=4096),
    "ragged_dup": lambda: graphs.random_csr(1000, 777, 0.01, seed=3, dup=True, empty_rows=0.3),
    "route_mix": lambda: graphs.route_mix(n=2048, target_nnz=100_000),
    "sbm": lambda: graphs.sbm_powerlaw(n=6000, avg_degree=30, communities=60),
    "single_row": lambda: graphs.random_csr(1, 300, 0.5, seed=5),
    "hub_rows": lambda: graphs.random_csr(200, 5000, 0.6, seed=7),
}


def _plan_and_ref(g, **opts):
    P = trspmm.host_plan(g.indptr, g.indices, g.values, g.n_rows, g.n_cols, engine="block", **opts)
    dec = oracle.decode_plan(P)["all"]
    plan = trspmm.Plan.build(g.indptr, g.indices, g.values, g.n_rows, g.n_cols, engine="block",
                             **opts)
    return plan, dec


@pytest.mark.parametrize("name", list(GRAPHS))
@pytest.mark.parametrize("k", [64, 128, 192, 256])
@pytest.mark.parametrize("out_dtype", [torch.float32, torch.float16])
def test_block_mma_forward(cuda, name, k, out_dtype):
    g = GRAPHS[name]()
    plan, dec = _plan_and_ref(g, row_scale=True, reorder=name == "sbm")
    assert plan.info["engine"] == trspmm.TR_ENGINE_BLOCK
    b = graphs.dense_features(g.n_cols, k, seed=k)
    out = plan.spmm(torch.from_numpy(b).to(cuda), out_dtype=out_dtype)
    torch.cuda.synchronize()
    ref = dec @ b.astype(np.float64)
    tol = TOL32 if out_dtype == torch.float32 else TOL16
    assert rel_err(out.float().cpu().numpy(), ref) <= tol


@pytest.mark.parametrize("name", ["chung_lu", "ragged_dup", "sbm"])
@pytest.mark.parametrize("k", [8, 24, 100, 128, 320])
def test_block_cuda_core_kernel(cuda, name, k):
    """Shapes outside the tensor-core kernel (K not a multiple of 64, or
    above 256) run the CUDA-core block kernel; TR_ROUTE_PER_WINDOW forces it
    for any K."""
    g = GRAPHS[name]()
    plan, dec = _plan_and_ref(g, row_scale=True)
    b = graphs.dense_features(g.n_cols, k, seed=3)
    mask = trspmm.TR_ROUTE_ALL | trspmm.TR_ROUTE_PER_WINDOW
    out = plan.spmm(torch.from_numpy(b).to(cuda), route_mask=mask)
    torch.cuda.synchronize()
    assert rel_err(out.cpu().numpy(), dec @ b.astype(np.float64)) <= TOL32


@pytest.mark.parametrize("name", ["chung_lu", "sbm"])
@pytest.mark.parametrize("k", [64, 128])
def test_block_fp32_features(cuda, name, k):
    g = GRAPHS[name]()
    plan, dec = _plan_and_ref(g, row_scale=True)
    b = np.random.default_rng(5).standard_normal((g.n_cols, k)).astype(np.float32)
    out = plan.spmm(torch.from_numpy(b).to(cuda))
    torch.cuda.synchronize()
    assert rel_err(out.cpu().numpy(), dec @ b.astype(np.float64)) <= 1e-5


def test_block_bitwise_repeatable(cuda):
    """Each output row is summed by one thread in a fixed order: two runs
    give identical bits."""
    g = GRAPHS["sbm"]()
    plan, _ = _plan_and_ref(g, row_scale=True, reorder=True)
    b = torch.from_numpy(graphs.dense_features(g.n_cols, 128, seed=9)).to(cuda)
    c1 = plan.spmm(b)
    c2 = plan.spmm(b)
    torch.cuda.synchronize()
    assert torch.equal(c1, c2)


@pytest.mark.parametrize("name", ["chung_lu", "ragged_dup", "sbm"])
@pytest.mark.parametrize("k", [64, 128, 256])
def test_block_adjoint_and_sddmm(cuda, name, k):
    """Adjoint plan on the block engine: dB = A^T dC and dval = SDDMM(dC, B)."""
    g = GRAPHS[name]()
    P = trspmm.host_plan(g.indptr, g.indices, g.values, g.n_rows, g.n_cols, engine="block",
                         transpose=True, row_scale=True, reorder=True)
    dec = oracle.decode_plan(P)["all"]
    adj = trspmm.Plan.build(g.indptr, g.indices, g.values, g.n_rows, g.n_cols, engine="block",
                            transpose=True, row_scale=True, reorder=True)
    dc = graphs.dense_features(g.n_rows, k, seed=11)
    b = graphs.dense_features(g.n_cols, k, seed=12)
    ip = torch.from_numpy(g.indptr).to(cuda)
    ix = torch.from_numpy(g.indices).to(cuda)
    db, dval = adj.adjoint_sddmm(ip, ix, torch.from_numpy(dc).to(cuda), torch.from_numpy(b).to(cuda))
    torch.cuda.synchronize()
    assert rel_err(db.cpu().numpy(), dec @ dc.astype(np.float64)) <= TOL32
    rows = np.repeat(np.arange(g.n_rows), np.diff(g.indptr))
    ref = np.einsum("ij,ij->i", dc[rows].astype(np.float64), b[g.indices].astype(np.float64))
    assert rel_err(dval.cpu().numpy(), ref) <= 1e-5


def test_block_set_values(cuda):
    """Re-valuing a block plan on the device equals building it with the new
    values (row scales recomputed)."""
    g = GRAPHS["sbm"]()
    w = np.random.default_rng(2).random(g.nnz).astype(np.float32) * 1e-3
    plan = trspmm.Plan.build(g.indptr, g.indices, g.values, g.n_rows, g.n_cols, engine="block",
                             row_scale=True, reorder=True)
    plan.set_values(torch.from_numpy(w).to(cuda))
    P = trspmm.host_plan(g.indptr, g.indices, w, g.n_rows, g.n_cols, engine="block",
                         row_scale=True, reorder=True)
    dec = oracle.decode_plan(P)["all"]
    b = graphs.dense_features(g.n_cols, 128, seed=4)
    out = plan.spmm(torch.from_numpy(b).to(cuda))
    torch.cuda.synchronize()
    assert rel_err(out.cpu().numpy(), dec @ b.astype(np.float64)) <= TOL32


def test_block_empty_and_partial(cuda):
    """No entries at all, and a row count that is not a multiple of 128:
    every output row is written (zeros where a row has no entry)."""
    import scipy.sparse as sp
    for n_rows, density in ((300, 0.0), (130, 0.02)):
        g = graphs.random_csr(n_rows, 64, density, seed=1)
        plan = trspmm.Plan.build(g.indptr, g.indices, g.values, g.n_rows, g.n_cols, engine="block")
        b = graphs.dense_features(64, 64, seed=1)
        out = torch.full((n_rows, 64), float("nan"), device=cuda)
        plan.spmm(torch.from_numpy(b).to(cuda), out=out)
        torch.cuda.synchronize()
        A = sp.csr_matrix((g.values.astype(np.float16).astype(np.float64), g.indices, g.indptr),
                          shape=(n_rows, 64))
        got = out.cpu().numpy()
        assert np.isfinite(got).all()
        ref = A @ b.astype(np.float64)
        assert np.abs(got - ref).max() <= TOL32 * max(1.0, np.abs(ref).max())


@pytest.mark.parametrize("k, k_tile", [(128, 64), (256, 128), (256, 64), (320, 0), (384, 192),
                                       (512, 0), (320, 192)])
def test_block_feature_tiles(cuda, k, k_tile):
    """K in feature tiles of k_tile (0 = 256) on the tensor cores: every tile
    a launch over its feature slice, K above 256 included."""
    g = GRAPHS["sbm"]()
    plan, dec = _plan_and_ref(g, row_scale=True, reorder=True)
    plan.set_k_tile(k_tile)
    b = graphs.dense_features(g.n_cols, k, seed=k + 1)
    out = plan.spmm(torch.from_numpy(b).to(cuda))
    torch.cuda.synchronize()
    assert rel_err(out.cpu().numpy(), dec @ b.astype(np.float64)) <= TOL32
    whole = trspmm.Plan.build(g.indptr, g.indices, g.values, g.n_rows, g.n_cols, engine="block",
                              row_scale=True, reorder=True)
    if k <= 256:
        ref = whole.spmm(torch.from_numpy(b).to(cuda))
        torch.cuda.synchronize()
        # each output element is the same sequence of MMAs whatever the tile width
        assert rel_err(out.cpu().numpy(), ref.cpu().numpy().astype(np.float64)) <= 1e-6


def test_block_k_tile_refusals(cuda):
    g = GRAPHS["chung_lu"]()
    plan = trspmm.Plan.build(g.indptr, g.indices, g.values, g.n_rows, g.n_cols, engine="block")
    for bad in (32, 100, 320, -64):
        with pytest.raises(RuntimeError, match="k_tile"):
            plan.set_k_tile(bad)


@pytest.mark.parametrize("name", ["chung_lu", "ragged_dup", "sbm", "hub_rows", "single_row"])
@pytest.mark.parametrize("k", [64, 128])
@pytest.mark.parametrize("renumber", [False, True])
def test_block_tensor_core_backward(cuda, name, k, renumber):
    """K = 64 / 128 on a block adjoint plan run the tensor-core backward
    (dB by one MMA, dval by a second against the block's rows of B in tensor
    memory): dB and dval against FP64, bitwise repeatable, and with the
    edges numbered in the plan's entry order dval lands at the entry's
    position."""
    g = GRAPHS[name]()
    kw = dict(engine="block", transpose=True, row_scale=True, reorder=name == "sbm")
    P = trspmm.host_plan(g.indptr, g.indices, g.values, g.n_rows, g.n_cols, **kw)
    dec = oracle.decode_plan(P)["all"]
    adj = trspmm.Plan.build(g.indptr, g.indices, g.values, g.n_rows, g.n_cols, **kw)
    new_id = None
    if renumber:
        order = adj.entry_order(cuda)
        new_id = torch.empty_like(order)
        new_id[order.long()] = torch.arange(g.nnz, dtype=torch.int32, device=cuda)
        adj.renumber_edges(new_id)
    dc = graphs.dense_features(g.n_rows, k, seed=21)
    b = graphs.dense_features(g.n_cols, k, seed=22)
    ip = torch.from_numpy(g.indptr).to(cuda)
    ix = torch.from_numpy(g.indices).to(cuda)
    dct, bt = torch.from_numpy(dc).to(cuda), torch.from_numpy(b).to(cuda)
    db1, dv1 = adj.adjoint_sddmm(ip, ix, dct, bt)
    db2, dv2 = adj.adjoint_sddmm(ip, ix, dct, bt)
    torch.cuda.synchronize()
    assert torch.equal(db1, db2) and torch.equal(dv1, dv2)
    assert rel_err(db1.cpu().numpy(), dec @ dc.astype(np.float64)) <= TOL32
    dv = dv1 if new_id is None else dv1[new_id.long()]
    rows = np.repeat(np.arange(g.n_rows), np.diff(g.indptr))
    ref = np.einsum("ij,ij->i", dc[rows].astype(np.float64), b[g.indices].astype(np.float64))
    assert rel_err(dv.cpu().numpy(), ref) <= 1e-5
    db16, _ = adj.adjoint_sddmm(ip, ix, dct, bt, db_dtype=torch.float16)
    torch.cuda.synchronize()
    assert rel_err(db16.float().cpu().numpy(), dec @ dc.astype(np.float64)) <= TOL16


def test_block_backward_empty_blocks(cuda):
    """Rows of A^T without entries (columns of A nobody uses) get zero dB."""
    g = graphs.random_csr(300, 2000, 0.002, seed=4)
    adj = trspmm.Plan.build(g.indptr, g.indices, g.values, g.n_rows, g.n_cols, engine="block",
                            transpose=True)
    dc = torch.from_numpy(graphs.dense_features(g.n_rows, 64, seed=1)).to(cuda)
    b = torch.from_numpy(graphs.dense_features(g.n_cols, 64, seed=2)).to(cuda)
    db = torch.full((g.n_cols, 64), float("nan"), device=cuda)
    dv = torch.full((g.nnz,), float("nan"), device=cuda)
    adj.adjoint_sddmm(torch.from_numpy(g.indptr).to(cuda), torch.from_numpy(g.indices).to(cuda),
                      dc, b, db=db, dval=dv)
    torch.cuda.synchronize()
    assert torch.isfinite(db).all() and torch.isfinite(dv).all()
    used = np.zeros(g.n_cols, bool)
    used[g.indices] = True
    assert (db[torch.from_numpy(~used).to(cuda)] == 0).all()


def test_block_plan_slot_count(cuda):
    """plan.info["slots"]: the distinct (block, column) pairs the product
    gathers, as the host layout counts them."""
    g = GRAPHS["ragged_dup"]()
    P = trspmm.host_plan(g.indptr, g.indices, g.values, g.n_rows, g.n_cols, engine="block")
    plan = trspmm.Plan.build(g.indptr, g.indices, g.values, g.n_rows, g.n_cols, engine="block")
    assert plan.info["slots"] == int((P["chunk_col"] >= 0).sum())
    assert plan.info["chunks"] * 16 == P["chunk_col"].size
