"""The headline workload at full size (200k-node SBM, 10.2M entries, K=128)
through the plans the benchmark times: the block-engine forward on
label-ordered rows and the fused CUDA-core backward, as RoutedAdjacency and
routed_spmm run them (autograd), and the block engine for the adjoint too.

Checked against FP64 on 2,000 sampled rows of C and dB and 20,000 sampled
entries of dval, and through the size-independent column-sum identities
1^T C = (1^T A) B and 1^T dB = (A 1)^T dC.  The autograd hands the FP32
gradient dC to the FP16 kernels as FP16(dC / max|dC|) and scales the outputs
back, so the FP64 references use that same dC.  Tolerances: C 1e-4 of the
largest magnitude (FP16 operands, FP32 accumulation and output), dB 2e-3
(returned in B's dtype, FP16: one rounding of the output), dval 1e-5; the
identities 1e-5 (C) and 1e-3 (dB) of the summed magnitudes.
"""
import numpy as np
import pytest
import scipy.sparse as sp
import torch

import trspmm
from helpers import rel_err
from trspmm import graphs
from trspmm.autograd import RoutedAdjacency, routed_spmm

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def workload():
    g, b = graphs.make_workload("large_routed")
    dc = graphs.dense_features(g.n_rows, b.shape[1], "normal", seed=g.seed + 101)
    return g, b, dc


def _check(g, b, dc, c, db, dval):
    # the matrix the plans multiply: FP16(v / row scale) * row scale (A's rows
    # for the forward, A^T's rows -- A's columns -- for the adjoint)
    v = g.values.astype(np.float64)
    rows = np.repeat(np.arange(g.n_rows), np.diff(g.indptr))

    def scaled(keys, n):
        s = np.zeros(n)
        np.maximum.at(s, keys, np.abs(v))
        s[s == 0] = 1
        return (v / s[keys]).astype(np.float16).astype(np.float64) * s[keys]
    A = sp.csr_matrix((scaled(rows, g.n_rows), g.indices, g.indptr), shape=(g.n_rows, g.n_cols))
    AT = sp.csr_matrix((scaled(g.indices, g.n_cols), g.indices, g.indptr),
                       shape=(g.n_rows, g.n_cols)).T.tocsr()
    s_dc = np.float32(np.abs(dc.astype(np.float32)).max())
    dc64 = (dc.astype(np.float32) / s_dc).astype(np.float16).astype(np.float64) * s_dc
    b64 = b.astype(np.float64)
    rng = np.random.default_rng(0)
    r = rng.choice(g.n_rows, 2000, replace=False)
    assert rel_err(c[r], A[r] @ b64) <= 1e-4
    r = rng.choice(g.n_cols, 2000, replace=False)
    assert rel_err(db[r], AT[r] @ dc64) <= 2e-3
    e = rng.choice(g.nnz, 20000, replace=False)
    ref = np.einsum("ij,ij->i", dc64[rows[e]], b64[g.indices[e]])
    assert rel_err(dval[e], ref) <= 1e-5
    colsum = np.asarray(A.sum(axis=0)).ravel() @ b64
    assert np.abs(c.astype(np.float64).sum(axis=0) - colsum).max() <= \
        1e-5 * (np.abs(A).sum(axis=0) @ np.abs(b64)).max()
    rowsum = np.asarray(AT.sum(axis=0)).ravel() @ dc64
    assert np.abs(db.astype(np.float64).sum(axis=0) - rowsum).max() <= \
        1e-3 * (np.abs(AT).sum(axis=0) @ np.abs(dc64)).max()


@pytest.mark.parametrize("adjoint", [{"demote_below": 1000},
                                     {"engine": "block", "reorder": True}])
def test_headline_plans_through_autograd(cuda, workload, adjoint):
    g, b, dc = workload
    adj = RoutedAdjacency(g.indptr, g.indices, g.values, g.n_rows, g.n_cols, device=cuda,
                          row_scale=True, promote_min=0, engine="block", reorder=True,
                          adjoint_options=adjoint)
    assert adj.fwd.info["engine"] == trspmm.TR_ENGINE_BLOCK
    assert adj.adj.info["engine"] == (trspmm.TR_ENGINE_BLOCK if "engine" in adjoint
                                      else trspmm.TR_ENGINE_WINDOW)
    bb = torch.from_numpy(b).to(cuda).requires_grad_(True)
    w = torch.from_numpy(g.values).to(cuda).requires_grad_(True)
    c = routed_spmm(adj, bb, w)
    c.backward(torch.from_numpy(dc).to(cuda))
    torch.cuda.synchronize()
    _check(g, b, dc, c.detach().cpu().numpy(), bb.grad.float().cpu().numpy(),
           w.grad.cpu().numpy())
