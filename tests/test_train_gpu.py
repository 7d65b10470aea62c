"""GPU parity of the native plans and the differentiation path.

  * routed forward of plans with row scaling, promoted residual columns, row
    clustering and transposition vs the FP64 product;
  * on-device re-valuing (tr_plan_set_values) vs a freshly built plan;
  * SDDMM vs the oracle's FP64 SDDMM;
  * the autograd Function (forward, dB = A^T dC, dw = SDDMM) vs torch.sparse
    autograd in FP64, and the analytic gradients of a two-layer GCN vs FP64
    central finite differences on a 2,000-node subgraph.

Tolerances: FP32 outputs of the FP16 kernels 1e-4 (max |C - C64| / max |C64|);
gradients through FP16 operands 5e-3 (max relative error vs FP64).
"""
import numpy as np
import pytest
import scipy.sparse as sp
import torch

import oracle
import trspmm
from helpers import rel_err
from trspmm import graphs
from trspmm.autograd import RoutedAdjacency, routed_spmm

pytestmark = pytest.mark.gpu

TOL32 = 1e-4
TOL_GRAD = 5e-3

GRAPHS = {
    "chung_lu": lambda: graphs.chung_lu(n=4096),
    "sbm": lambda: graphs.sbm_powerlaw(n=6000, avg_degree=30, communities=60, seed=4),
    "route_mix": lambda: graphs.route_mix(n=2048, target_nnz=100_000),
    "ragged": lambda: graphs.random_csr(1000, 777, 0.01, seed=3, empty_rows=0.3),
}
OPTS = [
    dict(row_scale=True),
    dict(promote_min=2),
    dict(promote_min=1, row_scale=True),
    dict(reorder=True, promote_min=2),
    dict(transpose=True, row_scale=True, promote_min=2),
    dict(transpose=True, reorder=True, promote_min=1),
]


def _matrix(g, values=None, transpose=False, row_scale=False):
    v = np.asarray(g.values if values is None else values, np.float32)
    A = sp.csr_matrix((v, g.indices, g.indptr), shape=(g.n_rows, g.n_cols))
    if transpose:
        A = A.T.tocsr()
    rows = np.repeat(np.arange(A.shape[0]), np.diff(A.indptr))
    s = np.ones(A.shape[0], np.float32)
    if row_scale:
        s = np.zeros(A.shape[0], np.float32)
        np.maximum.at(s, rows, np.abs(A.data.astype(np.float32)))
        s[s == 0] = 1
    q = (A.data.astype(np.float32) / s[rows]).astype(np.float16).astype(np.float64) * s[rows]
    return sp.csr_matrix((q, A.indices, A.indptr), shape=A.shape)


@pytest.mark.parametrize("opt", range(len(OPTS)))
@pytest.mark.parametrize("name", list(GRAPHS))
@pytest.mark.parametrize("k", [64, 128, 256, 40])
def test_native_plan_forward(cuda, name, opt, k):
    g = GRAPHS[name]()
    o = OPTS[opt]
    plan = trspmm.Plan.build(g.indptr, g.indices, g.values, g.n_rows, g.n_cols, **o)
    A = _matrix(g, transpose=o.get("transpose", False), row_scale=o.get("row_scale", False))
    b = graphs.dense_features(A.shape[1], k, seed=k)
    out = plan.spmm(torch.from_numpy(b).to(cuda))
    torch.cuda.synchronize()
    assert rel_err(out.cpu().numpy(), A @ b.astype(np.float64)) <= TOL32


@pytest.mark.parametrize("name", ["chung_lu", "sbm", "ragged"])
@pytest.mark.parametrize("row_scale", [False, True])
@pytest.mark.parametrize("transpose", [False, True])
def test_set_values_matches_rebuilt_plan(cuda, name, row_scale, transpose):
    g = GRAPHS[name]()
    plan = trspmm.Plan.build(g.indptr, g.indices, g.values, g.n_rows, g.n_cols,
                             row_scale=row_scale, transpose=transpose, promote_min=2)
    rng = np.random.default_rng(5)
    for trial in range(2):                      # twice: the second starts from re-valued scales
        w = (rng.standard_normal(g.nnz) * 10.0 ** rng.integers(-4, 1, g.nnz)).astype(np.float32)
        plan.set_values(torch.from_numpy(w).to(cuda))
        A = _matrix(g, values=w, transpose=transpose, row_scale=row_scale)
        b = graphs.dense_features(A.shape[1], 128, seed=trial)
        out = plan.spmm(torch.from_numpy(b).to(cuda))
        torch.cuda.synchronize()
        assert rel_err(out.cpu().numpy(), A @ b.astype(np.float64)) <= TOL32


def test_set_values_rejects_wrong_length(cuda):
    g = GRAPHS["ragged"]()
    plan = trspmm.Plan.build(g.indptr, g.indices, g.values, g.n_rows, g.n_cols)
    with pytest.raises(trspmm.TrError, match="value count"):
        plan.set_values(torch.zeros(g.nnz + 1, device=cuda))


@pytest.mark.parametrize("name", list(GRAPHS))
@pytest.mark.parametrize("k", [64, 128, 256, 24, 20])
def test_sddmm(cuda, name, k):
    g = GRAPHS[name]()
    x = graphs.dense_features(g.n_rows, k, seed=1)
    y = graphs.dense_features(g.n_cols, k, seed=2)
    ip = torch.from_numpy(g.indptr).to(cuda)
    ix = torch.from_numpy(g.indices).to(cuda)
    out = trspmm.sddmm_csr(ip, ix, torch.from_numpy(x).to(cuda), torch.from_numpy(y).to(cuda))
    torch.cuda.synchronize()
    ref = oracle.sddmm_f64(g.indptr, g.indices, x.astype(np.float64), y.astype(np.float64))
    assert rel_err(out.cpu().numpy(), ref) <= 1e-5


FUSED_CASES = [
    ("chung_lu", 128, dict(row_scale=True)),                     # fused (all residual)
    ("sbm", 64, dict(row_scale=True, demote_below=1000)),        # fused
    ("ragged", 40, dict()),                                      # fused, K not a power of 2
    ("sbm", 128, dict(reorder=True, demote_below=1000, row_scale=True)),   # fused, reordered
    ("route_mix", 128, dict()),                                  # tiles: two launches
    ("chung_lu", 256, dict()),                                   # fused, 32-lane groups
    ("ragged", 200, dict(row_scale=True)),                       # fused, 25 of 32 lanes active
    ("sbm", 256, dict(reorder=True, demote_below=1000)),         # fused, 32-lane groups, reordered
    ("chung_lu", 264, dict()),                                   # K > 256: two launches
]


@pytest.mark.parametrize("case", range(len(FUSED_CASES)))
def test_adjoint_sddmm(cuda, case):
    name, k, opts = FUSED_CASES[case]
    g = GRAPHS[name]()
    if name == "sbm" and "demote_below" in opts:
        opts = dict(opts)          # the SBM's dense route stays on tiles; force all-residual
    plan = trspmm.Plan.build(g.indptr, g.indices, g.values, g.n_rows, g.n_cols, transpose=True,
                             **opts)
    dc = graphs.dense_features(g.n_rows, k, seed=11)
    b = graphs.dense_features(g.n_cols, k, seed=12)
    ip = torch.from_numpy(g.indptr).to(cuda)
    ix = torch.from_numpy(g.indices).to(cuda)
    db, dval = plan.adjoint_sddmm(ip, ix, torch.from_numpy(dc).to(cuda),
                                  torch.from_numpy(b).to(cuda))
    torch.cuda.synchronize()
    AT = _matrix(g, transpose=True, row_scale=opts.get("row_scale", False))
    assert rel_err(db.cpu().numpy(), AT @ dc.astype(np.float64)) <= TOL32
    ref = oracle.sddmm_f64(g.indptr, g.indices, dc.astype(np.float64), b.astype(np.float64))
    assert rel_err(dval.cpu().numpy(), ref) <= 1e-5


def _torch_sparse_grads(g, w, b, dc):
    """FP64 torch.sparse autograd reference: C = A(w) B, grads of <C, dc>."""
    wt = torch.tensor(w, dtype=torch.float64, requires_grad=True)
    bt = torch.tensor(b, dtype=torch.float64, requires_grad=True)
    A = torch.sparse_csr_tensor(torch.from_numpy(g.indptr.astype(np.int64)),
                                torch.from_numpy(g.indices.astype(np.int64)), wt,
                                size=(g.n_rows, g.n_cols))
    c = torch.sparse.mm(A, bt) if False else (A @ bt)
    (c * torch.tensor(dc, dtype=torch.float64)).sum().backward()
    return c.detach().numpy(), bt.grad.numpy(), wt.grad.numpy()


@pytest.mark.parametrize("name", ["chung_lu", "sbm", "ragged"])
@pytest.mark.parametrize("k", [64, 128])
def test_autograd_vs_torch_sparse(cuda, name, k):
    g = GRAPHS[name]()
    adj = RoutedAdjacency(g.indptr, g.indices, g.values, g.n_rows, g.n_cols, device=cuda)
    rng = np.random.default_rng(7)
    w = (np.asarray(g.values, np.float32) * rng.uniform(0.5, 1.5, g.nnz)).astype(np.float32)
    b = rng.standard_normal((g.n_cols, k)).astype(np.float32)
    dc = rng.standard_normal((g.n_rows, k)).astype(np.float32)
    wt = torch.tensor(w, device=cuda, requires_grad=True)
    bt = torch.tensor(b, device=cuda, requires_grad=True)
    c = routed_spmm(adj, bt, wt)
    c.backward(torch.tensor(dc, device=cuda))
    c64, db64, dw64 = _torch_sparse_grads(g, w, b, dc)
    assert rel_err(c.detach().cpu().numpy(), c64) <= TOL_GRAD
    assert rel_err(bt.grad.cpu().numpy(), db64) <= TOL_GRAD
    assert rel_err(wt.grad.cpu().numpy(), dw64) <= TOL_GRAD


def test_gcn_two_layer_finite_differences(cuda):
    """Two-layer GCN (features 256 -> 128 -> 64) on a 2,000-node SBM subgraph
    with learnable FP32 edge weights initialised to GCN normalisation: the
    routed autograd gradients against FP64 central differences of the same
    loss computed in FP64 on the host."""
    full = graphs.sbm_powerlaw(n=100_000, avg_degree=30, communities=1000, seed=21)
    g = graphs.subgraph(full, 2000, seed=3)
    rng = np.random.default_rng(0)
    x = rng.standard_normal((g.n_rows, 256)).astype(np.float32)
    w1 = (rng.standard_normal((256, 128)) / 16).astype(np.float32)
    w2 = (rng.standard_normal((128, 64)) / 11).astype(np.float32)
    tgt = rng.standard_normal((g.n_rows, 64)).astype(np.float32)
    ew = np.asarray(g.values, np.float32)

    adj = RoutedAdjacency(g.indptr, g.indices, ew, g.n_rows, g.n_cols, device=cuda)
    X = torch.tensor(x, device=cuda)
    W1 = torch.tensor(w1, device=cuda, requires_grad=True)
    W2 = torch.tensor(w2, device=cuda, requires_grad=True)
    EW = torch.tensor(ew, device=cuda, requires_grad=True)
    T = torch.tensor(tgt, device=cuda)
    h1 = torch.relu(routed_spmm(adj, X @ W1, EW))
    h2 = routed_spmm(adj, h1 @ W2, EW)
    loss = 0.5 * ((h2 - T) ** 2).sum()
    loss.backward()

    ip, ix = g.indptr, g.indices

    def loss64(w1_, w2_, ew_):
        A = sp.csr_matrix((ew_, ix, ip), shape=(g.n_rows, g.n_cols))
        h = np.maximum(A @ (x.astype(np.float64) @ w1_), 0)
        o = A @ (h @ w2_)
        return 0.5 * ((o - tgt) ** 2).sum()

    base = (w1.astype(np.float64), w2.astype(np.float64), ew.astype(np.float64))
    grads = (W1.grad.cpu().numpy(), W2.grad.cpu().numpy(), EW.grad.cpu().numpy())
    for which in range(3):
        g_an = grads[which].astype(np.float64).ravel()
        top = np.argsort(-np.abs(g_an))[:6]
        pick = np.unique(np.concatenate([top, rng.choice(g_an.size, 6, replace=False)]))
        scale = np.abs(g_an).max()
        for i in pick:
            eps = 1e-3 * max(abs(base[which].ravel()[i]), 1e-2)
            args_p = [a.copy() for a in base]
            args_m = [a.copy() for a in base]
            args_p[which].ravel()[i] += eps
            args_m[which].ravel()[i] -= eps
            fd = (loss64(*args_p) - loss64(*args_m)) / (2 * eps)
            assert abs(fd - g_an[i]) <= TOL_GRAD * scale, (which, int(i), fd, g_an[i], scale)
