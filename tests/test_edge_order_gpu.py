"""Edge numbering of device plans (tr_plan_entry_order / tr_plan_renumber_edges)
and RoutedAdjacency(edge_order="adjoint").

A renumbered plan must compute exactly what it computed before, with every
per-entry array (set_values' input, adjoint_sddmm's dval) moved to the new
numbers: dval is compared bit for bit (each entry's dot product is the same
arithmetic wherever it is stored), dB and C within the FP32 tolerance of the
kernels (dB's segment-boundary rows are combined in a run-dependent order).
"""
import numpy as np
import pytest
import torch

import trspmm
from helpers import rel_err
from trspmm import graphs
from trspmm.autograd import RoutedAdjacency, routed_spmm

pytestmark = pytest.mark.gpu


def _graph():
    return graphs.sbm_powerlaw(n=3000, avg_degree=20, communities=30)


def _csr_t_order(g):
    """A's entries in A^T's CSR order (by column, then row)."""
    rows = np.repeat(np.arange(g.n_rows), np.diff(g.indptr))
    return np.lexsort((rows, g.indices)).astype(np.int32)


def _build(g, **kw):
    return trspmm.Plan.build(g.indptr, g.indices, g.values, g.n_rows, g.n_cols, **kw)


def test_entry_order_of_all_residual_adjoint_is_transpose_order(cuda):
    g = _graph()
    adj = _build(g, transpose=True, row_scale=True, demote_below=1000, promote_min=0)
    order = adj.entry_order(cuda).cpu().numpy()
    assert np.array_equal(order, _csr_t_order(g))


def test_entry_order_of_block_plan_is_a_permutation(cuda):
    g = _graph()
    fwd = _build(g, engine="block", row_scale=True, reorder=True)
    order = fwd.entry_order(cuda).cpu().numpy()
    assert np.array_equal(np.sort(order), np.arange(g.nnz))
    P = trspmm.host_plan(g.indptr, g.indices, g.values, g.n_rows, g.n_cols, engine="block",
                         row_scale=True, reorder=True)
    assert np.array_equal(order, P["ent_src"])


def test_entry_order_refuses_plans_with_tiles(cuda):
    g = graphs.route_mix(n=1024, target_nnz=40_000)
    p = _build(g, promote_min=2)
    assert p.info["tc_tiles"] + p.info["promoted_tiles"] > 0
    with pytest.raises(RuntimeError, match="tiles"):
        p.entry_order(cuda)


@pytest.mark.parametrize("k", [64, 128, 24])
@pytest.mark.parametrize("adj_engine", ["window", "block"])
def test_renumbered_adjoint_sddmm(cuda, k, adj_engine):
    """K = 64 / 128 on a window plan take the fused backward (dval at the
    plan position); K = 24 and the block engine take the adjoint kernel and
    the SDDMM over A's CSR, which writes through the plan's edge numbers."""
    g = _graph()
    kw = dict(transpose=True, row_scale=True, demote_below=1000, promote_min=0)
    if adj_engine == "block":
        kw = dict(transpose=True, row_scale=True, engine="block", reorder=True)
    base = _build(g, **kw)
    ren = _build(g, **kw)
    new_id = torch.from_numpy(np.random.default_rng(1).permutation(g.nnz).astype(np.int32)).to(cuda)
    ren.renumber_edges(new_id)
    ip = torch.from_numpy(g.indptr).to(cuda)
    ix = torch.from_numpy(g.indices).to(cuda)
    dc = torch.from_numpy(graphs.dense_features(g.n_rows, k, seed=3)).to(cuda)
    b = torch.from_numpy(graphs.dense_features(g.n_cols, k, seed=4)).to(cuda)
    db0, dv0 = base.adjoint_sddmm(ip, ix, dc, b)
    db1, dv1 = ren.adjoint_sddmm(ip, ix, dc, b)
    torch.cuda.synchronize()
    moved = torch.empty_like(dv0)
    moved[new_id.long()] = dv0
    assert torch.equal(moved, dv1)
    assert rel_err(db1.cpu().numpy(), db0.cpu().numpy().astype(np.float64)) <= 1e-6


@pytest.mark.parametrize("engine", ["window", "block"])
def test_renumbered_set_values(cuda, engine):
    g = _graph()
    kw = dict(row_scale=True, engine=engine, reorder=engine == "block")
    base = _build(g, **kw)
    ren = _build(g, **kw)
    new_id = torch.from_numpy(np.random.default_rng(2).permutation(g.nnz).astype(np.int32)).to(cuda)
    ren.renumber_edges(new_id)
    w = torch.from_numpy(np.random.default_rng(3).random(g.nnz).astype(np.float32)).to(cuda)
    w_new = torch.empty_like(w)
    w_new[new_id.long()] = w
    base.set_values(w)
    ren.set_values(w_new)
    b = torch.from_numpy(graphs.dense_features(g.n_cols, 128, seed=5)).to(cuda)
    c0 = base.spmm(b)
    c1 = ren.spmm(b)
    torch.cuda.synchronize()
    if engine == "block":
        assert torch.equal(c0, c1)        # one thread sums each output row
    else:
        assert rel_err(c1.cpu().numpy(), c0.cpu().numpy().astype(np.float64)) <= 1e-6


def test_renumbering_composes(cuda):
    g = _graph()
    kw = dict(transpose=True, row_scale=True, demote_below=1000, promote_min=0)
    once, twice = _build(g, **kw), _build(g, **kw)
    rng = np.random.default_rng(4)
    p1 = rng.permutation(g.nnz).astype(np.int32)
    p2 = rng.permutation(g.nnz).astype(np.int32)
    twice.renumber_edges(torch.from_numpy(p1).to(cuda))
    twice.renumber_edges(torch.from_numpy(p2).to(cuda))
    once.renumber_edges(torch.from_numpy(p2[p1]).to(cuda))
    ip = torch.from_numpy(g.indptr).to(cuda)
    ix = torch.from_numpy(g.indices).to(cuda)
    dc = torch.from_numpy(graphs.dense_features(g.n_rows, 64, seed=6)).to(cuda)
    b = torch.from_numpy(graphs.dense_features(g.n_cols, 64, seed=7)).to(cuda)
    _, d1 = once.adjoint_sddmm(ip, ix, dc, b)
    _, d2 = twice.adjoint_sddmm(ip, ix, dc, b)
    torch.cuda.synchronize()
    assert torch.equal(d1, d2)


def test_renumber_refuses_non_permutations(cuda):
    g = _graph()
    p = _build(g, transpose=True, demote_below=1000, promote_min=0)
    bad_range = torch.arange(g.nnz, dtype=torch.int32, device=cuda)
    bad_range[7] = g.nnz
    with pytest.raises(RuntimeError, match="permutation"):
        p.renumber_edges(bad_range)
    dup = torch.arange(g.nnz, dtype=torch.int32, device=cuda)
    dup[7] = 8
    with pytest.raises(RuntimeError, match="permutation"):
        p.renumber_edges(dup)
    with pytest.raises(RuntimeError):
        p.renumber_edges(torch.arange(g.nnz - 1, dtype=torch.int32, device=cuda))
    # the refused calls left the numbering alone
    order = p.entry_order(cuda).cpu().numpy()
    assert np.array_equal(order, _csr_t_order(g))


@pytest.mark.parametrize("features", ["f16", "f32"])
def test_routed_adjacency_adjoint_edge_order(cuda, features):
    """The same step with per-entry tensors in CSR order and in the adjoint
    plan's order: C and dB agree, dw is the same vector rearranged."""
    g = _graph()
    opts = dict(row_scale=True, promote_min=0, engine="block", reorder=True,
                adjoint_options={"demote_below": 1000}, features=features)
    a0 = RoutedAdjacency(g.indptr, g.indices, g.values, g.n_rows, g.n_cols, device=cuda, **opts)
    a1 = RoutedAdjacency(g.indptr, g.indices, g.values, g.n_rows, g.n_cols, device=cuda,
                         edge_order="adjoint", **opts)
    assert np.array_equal(a1.edge_id.cpu().numpy()[_csr_t_order(g)], np.arange(g.nnz))
    assert torch.equal(a1.to_csr_order(a1.values), a0.values)
    b = torch.from_numpy(graphs.dense_features(g.n_cols, 64, seed=8)).to(cuda).float()
    dc = torch.from_numpy(graphs.dense_features(g.n_rows, 64, seed=9)).to(cuda).float()
    outs = []
    for a in (a0, a1):
        w = a.values.clone().requires_grad_(True)
        bb = b.clone().requires_grad_(True)
        c = routed_spmm(a, bb, w)
        c.backward(dc)
        outs.append((c.detach(), bb.grad, w.grad))
    torch.cuda.synchronize()
    (c0, db0, dw0), (c1, db1, dw1) = outs
    assert torch.equal(c0, c1)
    assert rel_err(db1.cpu().numpy(), db0.cpu().numpy().astype(np.float64)) <= 1e-6
    assert rel_err(a1.to_csr_order(dw1).cpu().numpy(), dw0.cpu().numpy().astype(np.float64)) <= 1e-6
