"""Differentiable routed SpMM: C = A(w) . B with a hand-written adjoint.

``RoutedAdjacency`` holds one sparse matrix A (CSR pattern on the device plus
two routed plans built once: A for the forward, A^T for the adjoint).
``routed_spmm(adj, b, w)`` is the ``torch.autograd.Function`` front end:

  forward    C  = A(w) . B                         (routed kernel, plan of A)
  backward   dB = A(w)^T . dC                      (routed kernel, plan of A^T)
             dw[e] = <dC[row(e)], B[col(e)]>       (SDDMM on A's pattern)
             both in one pass over A^T when the adjoint plan allows
             (tr_adjoint_sddmm: each gathered row of dC feeds both products)

The reference has no backward at all; this is the differentiation path a GNN
built on the reference's operator would need.  With features="f16" (the
default) operands are FP16 on the tensor cores with FP32 accumulation; FP32
inputs and gradients are scaled by their largest magnitude before the FP16
cast (and the results scaled back), so their FP16 copies use the full
exponent range.  With features="f32" B, dC and dB stay FP32 end to end on
the FP32-feature route (tr_spmm_routed_f32 forward; tr_adjoint_sddmm_f32
for dB and the values' gradient together).  When the values ``w`` are
learnable, both plans are re-valued on the device (tr_plan_set_values)
whenever a forward or backward runs, so the pattern is routed only once.
"""
from __future__ import annotations

import numpy as np
import torch

from .core import Plan, sddmm_csr


class RoutedAdjacency:
    """Sparse A (n_rows x n_cols, CSR) with its forward and adjoint plans."""

    def __init__(self, indptr, indices, values, n_rows, n_cols, device="cuda",
                 row_scale=True, promote_min=2, reorder=False, plan_cache=None,
                 features="f16", adjoint_options=None, edge_order="csr", deterministic=False,
                 **route_kw):
        """plan_cache: None builds both plans; True or a directory takes them
        from the on-disk plan cache (trspmm.plan_cache), routing once per
        graph.  features: "f16" (FP16 operands) or "f32" (FP32 features on
        the FP32-feature route).  The other keywords shape both plans
        (Plan.build: engine, demote_below, promote_min, reorder, ...);
        adjoint_options (a dict of the same keywords) replaces them for the
        adjoint plan, e.g. a block-engine forward with the fused CUDA-core
        backward ({"demote_below": 1000}); row_scale applies to both.

        edge_order: the order of every per-entry tensor (the values w, their
        gradient, ``self.values``).  "csr": A's CSR order.  "adjoint": the
        adjoint plan's entry order (A^T's CSR order for an all-residual
        adjoint plan), which makes the backward's gradient stores and the
        adjoint plan's value upload sequential; ``edge_id[e]`` is then the
        position of A's CSR entry e, and to_edge_order / to_csr_order convert.

        deterministic: bitwise-repeatable gradients from a window adjoint plan
        (Plan.set_deterministic; block-engine plans always are)."""
        if features not in ("f16", "f32"):
            raise ValueError(f"features must be 'f16' or 'f32', not {features!r}")
        if edge_order not in ("csr", "adjoint"):
            raise ValueError(f"edge_order must be 'csr' or 'adjoint', not {edge_order!r}")
        self.features = features
        indptr = np.ascontiguousarray(indptr, dtype=np.int32)
        indices = np.ascontiguousarray(indices, dtype=np.int32)
        values = np.ascontiguousarray(values, dtype=np.float32)
        self.n_rows, self.n_cols = int(n_rows), int(n_cols)
        self.nnz = int(indices.size)
        kw = dict(row_scale=row_scale, promote_min=promote_min, reorder=reorder, **route_kw)
        akw = kw if adjoint_options is None else dict(row_scale=row_scale, **adjoint_options)
        if plan_cache:
            from .plan_cache import cached_plan
            d = None if plan_cache is True else str(plan_cache)
            self.fwd = cached_plan(indptr, indices, values, n_rows, n_cols, d, transpose=False, **kw)
            self.adj = cached_plan(indptr, indices, values, n_rows, n_cols, d, transpose=True, **akw)
        else:
            self.fwd = Plan.build(indptr, indices, values, n_rows, n_cols, transpose=False, **kw)
            self.adj = Plan.build(indptr, indices, values, n_rows, n_cols, transpose=True, **akw)
        if deterministic:
            self.adj.set_deterministic(True)
        self.device = torch.device(device)
        self.indptr = torch.from_numpy(indptr).to(self.device)
        self.indices = torch.from_numpy(indices).to(self.device)
        self.values = torch.from_numpy(values).to(self.device)
        self.edge_id = None
        if edge_order == "adjoint" and self.nnz:
            order = self.adj.entry_order(self.device)
            if bool((order < 0).any()):
                raise ValueError("edge_order='adjoint' needs an adjoint plan that holds every entry")
            new_id = torch.empty_like(order)
            new_id[order.long()] = torch.arange(self.nnz, dtype=torch.int32, device=self.device)
            self.fwd.renumber_edges(new_id)
            self.adj.renumber_edges(new_id)
            self.edge_id = new_id
            self.values = self.to_edge_order(self.values)

    def to_edge_order(self, x):
        """A per-entry tensor in A's CSR order, rearranged into this
        adjacency's edge order."""
        if self.edge_id is None:
            return x
        out = torch.empty_like(x)
        out[self.edge_id.long()] = x
        return out

    def to_csr_order(self, x):
        """A per-entry tensor in this adjacency's edge order, in A's CSR order."""
        return x if self.edge_id is None else x[self.edge_id.long()]

    def set_values(self, w):
        """Re-value both plans from FP32 entry values (CUDA tensor [nnz])."""
        w = w.detach().to(torch.float32).contiguous()
        if w.numel() != self.nnz:
            raise RuntimeError(f"expected {self.nnz} values, got {w.numel()}")
        self.fwd.set_values(w)
        self.adj.set_values(w)


def _to_half_scaled(x):
    """(FP16 copy of x / s, s) with s = max |x| (1 for FP16 input or all zeros)."""
    if x.dtype == torch.float16:
        return x.contiguous(), None
    s = x.detach().abs().amax()
    s = torch.where(s > 0, s, torch.ones_like(s)).to(torch.float32)
    return (x / s).to(torch.float16).contiguous(), s


class RoutedSpMMFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, w, b, adj):
        if w is not None:
            adj.set_values(w)
        ctx.adj = adj
        ctx.has_w = w is not None
        ctx.b_dtype = b.dtype
        if adj.features == "f32":
            b32 = b.detach().to(torch.float32).contiguous()
            ctx.save_for_backward(w if w is not None else torch.empty(0, device=b.device), b32)
            return adj.fwd.spmm(b32, out_dtype=torch.float32)
        b16, sb = _to_half_scaled(b)
        out = adj.fwd.spmm(b16, out_dtype=torch.float32)
        if sb is not None:
            out = out * sb
        ctx.save_for_backward(w if w is not None else torch.empty(0, device=b.device), b16,
                              sb if sb is not None else torch.empty(0, device=b.device))
        return out

    @staticmethod
    def backward(ctx, dc):
        adj = ctx.adj
        if adj.features == "f32":
            w, b32 = ctx.saved_tensors
            if ctx.has_w:
                adj.set_values(w)
            dc32 = dc.detach().to(torch.float32).contiguous()
            db = dw = None
            if ctx.needs_input_grad[1] and ctx.has_w and ctx.needs_input_grad[0]:
                # both gradients in one pass over A^T (tr_adjoint_sddmm_f32)
                db, dw = adj.adj.adjoint_sddmm(adj.indptr, adj.indices, dc32, b32)
                return dw, db.to(ctx.b_dtype), None
            if ctx.needs_input_grad[1]:
                db = adj.adj.spmm(dc32, out_dtype=torch.float32).to(ctx.b_dtype)
            if ctx.has_w and ctx.needs_input_grad[0]:
                dw = adj.to_edge_order(sddmm_csr(adj.indptr, adj.indices, dc32, b32))
            return dw, db, None
        w, b16, sb = ctx.saved_tensors
        if ctx.has_w:
            adj.set_values(w)
        dc16, sc = _to_half_scaled(dc.contiguous())
        db = dw = None
        scale = None
        if sc is not None:
            scale = sc
        if sb.numel():
            scale = sb if scale is None else scale * sb
        if ctx.needs_input_grad[1] and ctx.has_w and ctx.needs_input_grad[0]:
            # both gradients: one pass over A^T gathers each row of dC once
            db, dw = adj.adj.adjoint_sddmm(adj.indptr, adj.indices, dc16, b16)
            if sc is not None:
                db = db * sc
            if scale is not None:
                dw = dw * scale
            return dw, db.to(ctx.b_dtype), None
        if ctx.needs_input_grad[1]:
            db = adj.adj.spmm(dc16, out_dtype=torch.float32)
            if sc is not None:
                db = db * sc
            db = db.to(ctx.b_dtype)
        if ctx.has_w and ctx.needs_input_grad[0]:
            dw = adj.to_edge_order(sddmm_csr(adj.indptr, adj.indices, dc16, b16))
            if scale is not None:
                dw = dw * scale
        return dw, db, None


def routed_spmm(adj, b, w=None):
    """C = A . B (FP32 out).  With w (FP32 [nnz], may require grad) the values
    of A are w; without, the values A was built with."""
    return RoutedSpMMFunction.apply(w, b, adj)
