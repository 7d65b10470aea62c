"""GCN layers on the routed SpMM (graph convolution H' = A (H W) + b).

The reference's GCN driver multiplies a routed adjacency by dense features
inside its dataset/model objects (spmm/tr_csr_fp16/mdataset2_online.py:33-153,
test_tr_csr_online.py); here the same product is a torch module whose
backward is the library's adjoint (dB = A^T dC) and, with learnable edge
weights, the fused SDDMM (dval): routed_spmm of trspmm.autograd.
"""
from __future__ import annotations

import math

import torch

from .autograd import RoutedAdjacency, routed_spmm


class GCNConv(torch.nn.Module):
    """One graph convolution: H' = A (H W) + b.

    forward(adj, x, edge_weight=None): adj a RoutedAdjacency (n x n), x the
    node features [n, in_features] (FP32 or FP16), edge_weight an optional
    FP32 [nnz] tensor of A's values in A's CSR order (learnable if it
    requires grad); without it A keeps the values it was built with."""

    def __init__(self, in_features, out_features, bias=True):
        super().__init__()
        self.weight = torch.nn.Parameter(torch.empty(in_features, out_features))
        self.bias = torch.nn.Parameter(torch.zeros(out_features)) if bias else None
        bound = math.sqrt(6.0 / (in_features + out_features))     # Glorot uniform
        with torch.no_grad():
            self.weight.uniform_(-bound, bound)

    def forward(self, adj: RoutedAdjacency, x, edge_weight=None):
        h = routed_spmm(adj, x @ self.weight.to(x.dtype), edge_weight)
        return h + self.bias if self.bias is not None else h


class GCN(torch.nn.Module):
    """Stacked GCNConv layers with an activation between them (ReLU by
    default; the two-layer model of the differentiation workload:
    256 -> 128 -> 64).  With learn_edge_weights, A's values become one FP32
    parameter shared by all layers, initialised to the adjacency's values.

    The product runs on FP16 operands with FP32 accumulation, so a
    pre-activation within that rounding of ReLU's kink can fall on the other
    side of it than in an FP32 model; the gradients of the entries that
    depend on it then differ by O(1) (a property of the kink, not of the
    product: a smooth activation agrees to FP16 tolerance)."""

    def __init__(self, adj: RoutedAdjacency, sizes=(256, 128, 64), bias=True,
                 learn_edge_weights=False, activation=torch.relu):
        super().__init__()
        self.adj = adj
        self.activation = activation
        self.layers = torch.nn.ModuleList(GCNConv(a, b, bias) for a, b in zip(sizes[:-1], sizes[1:]))
        self.edge_weight = (torch.nn.Parameter(adj.values.detach().clone().to(torch.float32))
                            if learn_edge_weights else None)

    def forward(self, x):
        for i, layer in enumerate(self.layers):
            x = layer(self.adj, x, self.edge_weight)
            if i + 1 < len(self.layers):
                x = self.activation(x)
        return x
