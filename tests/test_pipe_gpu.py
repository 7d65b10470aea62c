"""The persistent pipelined routed kernel (full product, K % 64 == 0,
K <= 256) against the FP64 product and against the one-CTA-per-window fused
kernel on the same plan: windows with no tiles, with one tile, with more
tiles than a stage holds, with residual entries or none, every output row
written exactly once.  Other K take the per-window kernel through the same
call.  Tolerances as in test_spmm_gpu: 1e-4 (FP32 out), 2e-3 (FP16 out)."""
import numpy as np
import pytest
import scipy.sparse as sp
import torch

import trspmm
from helpers import rel_err
from trspmm import graphs

pytestmark = pytest.mark.gpu


def _heavy_row():
    # one row with 3000 entries (hundreds of tiles in one window), others sparse
    g = graphs.random_csr(200, 4000, 0.002, seed=9)
    rows = np.concatenate([np.repeat(np.arange(200), np.diff(g.indptr)), np.full(3000, 17)])
    cols = np.concatenate([g.indices, np.random.default_rng(1).choice(4000, 3000, replace=False)])
    A = sp.coo_matrix((np.ones(rows.size, np.float32), (rows, cols)), shape=(200, 4000)).tocsr()
    A.sum_duplicates()
    vals = np.random.default_rng(2).uniform(-1, 1, A.nnz).astype(np.float32)
    return graphs.Graph(A.indptr.astype(np.int32), A.indices.astype(np.int32), vals, 200, 4000)


GRAPHS = {
    "chung_lu": lambda: graphs.chung_lu(n=4096),
    "sbm": lambda: graphs.sbm_powerlaw(n=6000, avg_degree=30, communities=60, seed=4),
    "route_mix": lambda: graphs.route_mix(n=2048, target_nnz=100_000),
    "ragged": lambda: graphs.random_csr(1000, 777, 0.004, seed=3, empty_rows=0.6),
    "tiny": lambda: graphs.random_csr(3, 5, 0.5, seed=5),
    "heavy_row": _heavy_row,
    "batched": lambda: graphs.batched(num_graphs=40, seed=2),
}
PLANS = {
    "exact": dict(),
    "promote1": dict(promote_min=1),
    "reorder_scale": dict(reorder=True, row_scale=True, promote_min=2),
}


def _ref(g, opts):
    v = np.asarray(g.values, np.float32)
    rows = np.repeat(np.arange(g.n_rows), np.diff(g.indptr))
    s = np.ones(g.n_rows, np.float32)
    if opts.get("row_scale"):
        s = np.zeros(g.n_rows, np.float32)
        np.maximum.at(s, rows, np.abs(v))
        s[s == 0] = 1
    q = (v / s[rows]).astype(np.float16).astype(np.float64) * s[rows]
    return sp.csr_matrix((q, g.indices, g.indptr), shape=(g.n_rows, g.n_cols))


@pytest.mark.parametrize("plan_kind", list(PLANS))
@pytest.mark.parametrize("name", list(GRAPHS))
@pytest.mark.parametrize("k", [40, 64, 128, 192, 256])
@pytest.mark.parametrize("out_dtype", [torch.float32, torch.float16])
def test_pipe_kernel(cuda, name, plan_kind, k, out_dtype):
    g = GRAPHS[name]()
    opts = PLANS[plan_kind]
    plan = trspmm.Plan.build(g.indptr, g.indices, g.values, g.n_rows, g.n_cols, **opts)
    b = graphs.dense_features(g.n_cols, k, seed=k + 1)
    bd = torch.from_numpy(b).to(cuda)
    # poison the output: every element must be overwritten
    out = torch.full((g.n_rows, k), float("nan"), dtype=out_dtype, device=cuda)
    plan.spmm(bd, out=out, route_mask=trspmm.TR_ROUTE_ALL | trspmm.TR_ROUTE_PIPELINED)
    per_win = plan.spmm(bd, out_dtype=out_dtype,
                        route_mask=trspmm.TR_ROUTE_ALL | trspmm.TR_ROUTE_PER_WINDOW)
    default = plan.spmm(bd, out_dtype=out_dtype)
    torch.cuda.synchronize()
    o = out.float().cpu().numpy()
    assert np.isfinite(o).all(), "output element left unwritten"
    ref = _ref(g, opts) @ b.astype(np.float64)
    tol = 1e-4 if out_dtype == torch.float32 else 2e-3
    if np.abs(ref).max() == 0:
        assert np.abs(o).max() == 0
        return
    assert rel_err(o, ref) <= tol
    assert rel_err(o, per_win.float().cpu().numpy()) <= tol
    assert rel_err(default.float().cpu().numpy(), ref) <= tol


def test_pipe_kernel_repeated_calls_stable(cuda):
    """Back-to-back launches on one stream give identical results (no state
    is carried between launches)."""
    g = GRAPHS["sbm"]()
    plan = trspmm.Plan.build(g.indptr, g.indices, g.values, g.n_rows, g.n_cols, promote_min=1)
    bd = torch.from_numpy(graphs.dense_features(g.n_cols, 128, seed=3)).to(cuda)
    mask = trspmm.TR_ROUTE_ALL | trspmm.TR_ROUTE_PIPELINED
    first = plan.spmm(bd, route_mask=mask)
    for _ in range(5):
        again = plan.spmm(bd, route_mask=mask)
    torch.cuda.synchronize()
    assert torch.equal(first, again)
