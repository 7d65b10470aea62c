"""trspmm.nn (GCNConv, GCN) against the same model on torch.sparse FP32
(forward and every parameter gradient, learnable edge weights included) on a
2,000-node SBM subgraph, and a few optimiser steps moving the loss down.
The parity model uses tanh between the layers: with ReLU, pre-activations
within the FP16-operand rounding of the kink fall on the other side of it
than in FP32 and move the gradients that depend on them by O(1)."""
import numpy as np
import pytest
import torch

from trspmm import graphs
from trspmm.autograd import RoutedAdjacency
from trspmm.nn import GCN

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float((a - b).abs().max() / b.abs().max().clamp_min(1e-30))


def test_gcn_matches_torch_sparse(cuda):
    full = graphs.sbm_powerlaw(n=100_000, avg_degree=30, communities=1000, seed=21)
    g = graphs.subgraph(full, 2000, seed=5)
    torch.manual_seed(0)
    adj = RoutedAdjacency(g.indptr, g.indices, g.values, g.n_rows, g.n_cols, device=cuda)
    model = GCN(adj, (256, 128, 64), learn_edge_weights=True, activation=torch.tanh).to(cuda)
    x = torch.randn(g.n_rows, 256, device=cuda)
    tgt = torch.randn(g.n_rows, 64, device=cuda)
    out = model(x)
    loss = 0.5 * ((out - tgt) ** 2).sum()
    loss.backward()

    # the same model on torch.sparse (FP32), sharing the initial parameters
    ip = torch.from_numpy(g.indptr.astype(np.int64)).to(cuda)
    ix = torch.from_numpy(g.indices.astype(np.int64)).to(cuda)
    ew = model.edge_weight.detach().clone().requires_grad_(True)
    ws = [l.weight.detach().clone().requires_grad_(True) for l in model.layers]
    bs = [l.bias.detach().clone().requires_grad_(True) for l in model.layers]

    def spmm(h):
        A = torch.sparse_csr_tensor(ip, ix, ew, size=(g.n_rows, g.n_cols))
        return torch.sparse.mm(A, h)

    h = x
    for i, (w, b) in enumerate(zip(ws, bs)):
        h = spmm(h @ w) + b
        if i + 1 < len(ws):
            h = torch.tanh(h)
    ref_loss = 0.5 * ((h - tgt) ** 2).sum()
    ref_loss.backward()

    tol = 5e-3                       # FP16 operands, FP32 accumulation
    assert _rel(out.detach(), h.detach()) < tol
    assert _rel(model.edge_weight.grad, ew.grad) < tol
    for l, w, b in zip(model.layers, ws, bs):
        assert _rel(l.weight.grad, w.grad) < tol
        assert _rel(l.bias.grad, b.grad) < tol


def test_gcn_trains(cuda):
    g = graphs.chung_lu(n=4096)
    torch.manual_seed(1)
    adj = RoutedAdjacency(g.indptr, g.indices, g.values, g.n_rows, g.n_cols, device=cuda)
    model = GCN(adj, (64, 32, 16), learn_edge_weights=True).to(cuda)
    x = torch.randn(g.n_rows, 64, device=cuda)
    tgt = torch.randn(g.n_rows, 16, device=cuda)
    opt = torch.optim.Adam(model.parameters(), lr=1e-2)
    losses = []
    for _ in range(20):
        opt.zero_grad()
        loss = ((model(x) - tgt) ** 2).mean()
        loss.backward()
        opt.step()
        losses.append(float(loss))
    assert losses[-1] < 0.9 * losses[0]
