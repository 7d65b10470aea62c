"""FP32-feature route (tr_spmm_routed_f32, tr_sddmm_csr_f32, autograd with
features="f32") against FP64 products.

The plan's values are what the kernels multiply (FP16 significand x FP32
row scale); the oracle decodes them from the host plan (oracle.decode_plan),
so the forward is compared with that exact matrix times FP32 B in FP64:
max |C - C64| / max |C64| <= 1e-5 with FP32 output (FP32 products and
sums), 2e-3 with FP16 output.  Gradients through autograd are compared with
torch.sparse FP64 autograd on the unrounded values: dB within 1e-3 (A's FP16
significand), dw within 1e-5 (FP32 SDDMM, no rounded operand).
"""
import numpy as np
import pytest
import torch

import oracle
import trspmm
from helpers import rel_err
from trspmm import graphs
from trspmm.autograd import RoutedAdjacency, routed_spmm

pytestmark = pytest.mark.gpu

TOL_F32 = 1e-5
TOL_F16 = 2e-3

GRAPHS = {
    "chung_lu": lambda: graphs.chung_lu(n=4096),
    "route_mix": lambda: graphs.route_mix(n=2048, target_nnz=100_000),
    "sbm": lambda: graphs.sbm_powerlaw(n=6000, avg_degree=30, communities=60, seed=4),
    "ragged": lambda: graphs.random_csr(1000, 777, 0.01, seed=3, empty_rows=0.3),
}
OPTS = [
    dict(),                                          # the reference's routing: TC + 2:4 tiles
    dict(row_scale=True, promote_min=2),             # + promoted residual columns
    dict(row_scale=True, demote_below=1000),         # residual-heavy
    dict(transpose=True, row_scale=True, promote_min=2),
    dict(reorder="tca", promote_min=2),
]
_built = {}


def _graph(name):
    if name not in _built:
        _built[name] = GRAPHS[name]()
    return _built[name]


def _decoded(g, opts):
    P = trspmm.host_plan(g.indptr, g.indices, g.values, g.n_rows, g.n_cols, **opts)
    return oracle.decode_plan(P)


@pytest.fixture(scope="module")
def dev():
    return torch.device("cuda:0")


@pytest.mark.parametrize("opt", range(len(OPTS)))
@pytest.mark.parametrize("name", list(GRAPHS))
@pytest.mark.parametrize("k", [64, 200])
def test_forward_matches_fp64(dev, name, opt, k):
    g = _graph(name)
    o = OPTS[opt]
    plan = trspmm.Plan.build(g.indptr, g.indices, g.values, g.n_rows, g.n_cols, **o)
    D = _decoded(g, o)["all"]
    b = np.random.default_rng(k).standard_normal((D.shape[1], k)).astype(np.float32)
    c = plan.spmm(torch.from_numpy(b).to(dev))
    torch.cuda.synchronize()
    assert rel_err(c.cpu().numpy(), D @ b.astype(np.float64)) <= TOL_F32


@pytest.mark.parametrize("k", [4, 8, 36, 128, 132, 256, 13, 1])
def test_feature_widths_and_fp16_output(dev, k):
    g = _graph("route_mix")
    o = dict(row_scale=True, promote_min=2)
    plan = trspmm.Plan.build(g.indptr, g.indices, g.values, g.n_rows, g.n_cols, **o)
    D = _decoded(g, o)["all"]
    b = np.random.default_rng(k).uniform(-1, 1, (g.n_cols, k)).astype(np.float32)
    ref = D @ b.astype(np.float64)
    bt = torch.from_numpy(b).to(dev)
    assert rel_err(plan.spmm(bt).cpu().numpy(), ref) <= TOL_F32
    c16 = plan.spmm(bt, out_dtype=torch.float16)
    torch.cuda.synchronize()
    assert rel_err(c16.float().cpu().numpy(), ref) <= TOL_F16


@pytest.mark.parametrize("mask,parts", [
    (trspmm.TR_ROUTE_TC, ("tc",)),
    (trspmm.TR_ROUTE_SPTC, ("sptc",)),
    (trspmm.TR_ROUTE_CUDA, ("res", "prom")),
    (trspmm.TR_ROUTE_TC | trspmm.TR_ROUTE_CUDA, ("tc", "res", "prom")),
])
def test_route_masks(dev, mask, parts):
    g = _graph("route_mix")
    o = dict(promote_min=2)
    plan = trspmm.Plan.build(g.indptr, g.indices, g.values, g.n_rows, g.n_cols, **o)
    D = _decoded(g, o)
    ref_m = sum(D[p] for p in parts)
    assert ref_m.nnz > 0
    b = np.random.default_rng(5).standard_normal((g.n_cols, 64)).astype(np.float32)
    c = plan.spmm(torch.from_numpy(b).to(dev), route_mask=mask)
    torch.cuda.synchronize()
    assert rel_err(c.cpu().numpy(), ref_m @ b.astype(np.float64)) <= TOL_F32


def test_misaligned_features_take_the_scalar_kernel(dev):
    g = _graph("ragged")
    plan = trspmm.Plan.build(g.indptr, g.indices, g.values, g.n_rows, g.n_cols, promote_min=2)
    D = _decoded(g, dict(promote_min=2))["all"]
    b = np.random.default_rng(1).standard_normal((g.n_cols, 64)).astype(np.float32)
    # a contiguous view starting 4 bytes into an allocation: not 16-byte aligned
    off = torch.empty(g.n_cols * 64 + 1, device=dev)[1:].view(g.n_cols, 64)
    off.copy_(torch.from_numpy(b).to(dev))
    assert off.data_ptr() % 16 != 0
    c = plan.spmm(off)
    torch.cuda.synchronize()
    assert rel_err(c.cpu().numpy(), D @ b.astype(np.float64)) <= TOL_F32


@pytest.mark.parametrize("k", [4, 64, 128, 256, 13])
def test_sddmm_f32(dev, k):
    g = _graph("sbm")
    rng = np.random.default_rng(k)
    x = rng.standard_normal((g.n_rows, k)).astype(np.float32)
    y = rng.standard_normal((g.n_cols, k)).astype(np.float32)
    ip = torch.from_numpy(g.indptr).to(dev)
    ix = torch.from_numpy(g.indices).to(dev)
    out = trspmm.sddmm_csr(ip, ix, torch.from_numpy(x).to(dev), torch.from_numpy(y).to(dev))
    torch.cuda.synchronize()
    ref = oracle.sddmm_f64(g.indptr, g.indices, x.astype(np.float64), y.astype(np.float64))
    assert rel_err(out.cpu().numpy(), ref) <= TOL_F32
    with pytest.raises(RuntimeError, match="same dtype"):
        trspmm.sddmm_csr(ip, ix, torch.from_numpy(x).to(dev), torch.from_numpy(y).to(dev).half())


@pytest.mark.parametrize("name", ["chung_lu", "sbm", "ragged"])
def test_autograd_f32_vs_torch_sparse(dev, name):
    g = _graph(name)
    k = 64
    rng = np.random.default_rng(7)
    w = (rng.uniform(0.1, 1.0, g.nnz)).astype(np.float32)
    b = rng.standard_normal((g.n_cols, k)).astype(np.float32)
    dc = rng.standard_normal((g.n_rows, k)).astype(np.float32)
    adj = RoutedAdjacency(g.indptr, g.indices, w, g.n_rows, g.n_cols, features="f32")
    wt = torch.tensor(w, device=dev, requires_grad=True)
    bt = torch.tensor(b, device=dev, requires_grad=True)
    c = routed_spmm(adj, bt, wt)
    (c * torch.tensor(dc, device=dev)).sum().backward()
    torch.cuda.synchronize()
    w64 = torch.tensor(w, dtype=torch.float64, requires_grad=True)
    b64 = torch.tensor(b, dtype=torch.float64, requires_grad=True)
    A = torch.sparse_csr_tensor(torch.from_numpy(g.indptr.astype(np.int64)),
                                torch.from_numpy(g.indices.astype(np.int64)), w64,
                                size=(g.n_rows, g.n_cols))
    c64 = A @ b64
    (c64 * torch.tensor(dc, dtype=torch.float64)).sum().backward()
    assert rel_err(c.detach().cpu().numpy(), c64.detach().numpy()) <= 1e-3
    assert rel_err(bt.grad.cpu().numpy(), b64.grad.numpy()) <= 1e-3
    assert rel_err(wt.grad.cpu().numpy(), w64.grad.numpy()) <= TOL_F32
    with pytest.raises(ValueError, match="features"):
        RoutedAdjacency(g.indptr, g.indices, w, g.n_rows, g.n_cols, features="tf32")


@pytest.mark.parametrize("name,k,opts", [
    ("chung_lu", 128, dict(row_scale=True, demote_below=1000)),     # fused, 32-lane groups
    ("sbm", 64, dict(row_scale=True, demote_below=1000)),           # fused, 16-lane groups
    ("ragged", 20, dict()),                                          # fused, 8-lane groups, 5 active
    ("sbm", 256, dict(demote_below=1000)),                           # K > 128: two launches
    ("route_mix", 64, dict()),                                       # tiles: two launches
])
def test_adjoint_sddmm_f32(dev, name, k, opts):
    g = _graph(name)
    plan = trspmm.Plan.build(g.indptr, g.indices, g.values, g.n_rows, g.n_cols, transpose=True,
                             **opts)
    rng = np.random.default_rng(k)
    dc = rng.standard_normal((g.n_rows, k)).astype(np.float32)
    b = rng.standard_normal((g.n_cols, k)).astype(np.float32)
    ip = torch.from_numpy(g.indptr).to(dev)
    ix = torch.from_numpy(g.indices).to(dev)
    db, dval = plan.adjoint_sddmm(ip, ix, torch.from_numpy(dc).to(dev), torch.from_numpy(b).to(dev))
    torch.cuda.synchronize()
    AT = _decoded(g, dict(transpose=True, **opts))["all"]
    assert rel_err(db.cpu().numpy(), AT @ dc.astype(np.float64)) <= TOL_F32
    ref = oracle.sddmm_f64(g.indptr, g.indices, dc.astype(np.float64), b.astype(np.float64))
    assert rel_err(dval.cpu().numpy(), ref) <= TOL_F32
