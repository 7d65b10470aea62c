"""Block-diagonal batches: one plan pair for many graphs gives the same
forward and backward as one plan pair per graph (FP64 product as the
arbiter), and the CUDA-graph replay of the batched step equals its eager
run up to summation order.  Tolerances: 1e-4 (FP32 outputs), SDDMM 1e-5,
replay vs eager 1e-6."""
import numpy as np
import pytest
import scipy.sparse as sp
import torch

import oracle
from helpers import rel_err
from trspmm import graphs
from trspmm.batched import BatchedStep, PerGraphLoop

pytestmark = pytest.mark.gpu

OPTS = [dict(demote_below=1000, promote_min=0, row_scale=True),
        dict(promote_min=2, row_scale=True),
        dict(row_scale=False)]


@pytest.mark.parametrize("opt", range(len(OPTS)))
@pytest.mark.parametrize("k", [64, 128])
def test_batched_matches_per_graph_and_fp64(cuda, opt, k):
    g = graphs.batched(num_graphs=40, seed=9)
    o = OPTS[opt]
    bs = BatchedStep(g, k, device=cuda, **o)
    loop = PerGraphLoop(g, k, device=cuda, **o)
    b = graphs.dense_features(g.n_cols, k, seed=1)
    dc = graphs.dense_features(g.n_rows, k, seed=2)
    for st in (bs, loop):
        st.b.copy_(torch.from_numpy(b))
        st.dc.copy_(torch.from_numpy(dc))
        st.run()
    torch.cuda.synchronize()
    A = sp.csr_matrix((np.asarray(g.values, np.float64), g.indices, g.indptr),
                      shape=(g.n_rows, g.n_cols))
    rows = np.repeat(np.arange(g.n_rows), np.diff(g.indptr))
    v = np.asarray(g.values, np.float32)
    if o.get("row_scale"):
        s = np.zeros(g.n_rows, np.float32)
        np.maximum.at(s, rows, np.abs(v))
        s[s == 0] = 1
        A16 = sp.csr_matrix(((v / s[rows]).astype(np.float16).astype(np.float64) * s[rows],
                             g.indices, g.indptr), shape=A.shape)
        st_ = np.zeros(g.n_cols, np.float32)
        np.maximum.at(st_, g.indices, np.abs(v))
        st_[st_ == 0] = 1
        AT16 = sp.csr_matrix(((v / st_[g.indices]).astype(np.float16).astype(np.float64)
                              * st_[g.indices], g.indices, g.indptr), shape=A.shape).T
    else:
        A16 = sp.csr_matrix((v.astype(np.float16).astype(np.float64), g.indices, g.indptr),
                            shape=A.shape)
        AT16 = A16.T
    c_ref = A16 @ b.astype(np.float64)
    db_ref = AT16 @ dc.astype(np.float64)
    dv_ref = oracle.sddmm_f64(g.indptr, g.indices, dc.astype(np.float64), b.astype(np.float64))
    for st in (bs, loop):
        assert rel_err(st.c.cpu().numpy(), c_ref) <= 1e-4
        assert rel_err(st.db.cpu().numpy(), db_ref) <= 1e-4
        assert rel_err(st.dval.cpu().numpy(), dv_ref) <= 1e-5


def test_batched_graph_replay_equals_eager(cuda):
    g = graphs.batched(num_graphs=64, seed=4)
    bs = BatchedStep(g, 64, device=cuda, demote_below=1000, promote_min=0, row_scale=True)
    bs.b.copy_(torch.from_numpy(graphs.dense_features(g.n_cols, 64, seed=3)))
    bs.dc.copy_(torch.from_numpy(graphs.dense_features(g.n_rows, 64, seed=4)))
    bs.run()
    torch.cuda.synchronize()
    ref = (bs.c.clone(), bs.db.clone(), bs.dval.clone())
    bs.c.zero_(); bs.db.zero_(); bs.dval.zero_()
    bs.capture()
    bs.c.zero_(); bs.db.zero_(); bs.dval.zero_()
    bs.replay()
    torch.cuda.synchronize()
    # the CUDA-core engine adds a row's partial sums from different warps with
    # shared-memory atomics, so the last bits may differ from run to run
    for x, y in zip((bs.c, bs.db, bs.dval), ref):
        assert rel_err(x.cpu().numpy(), y.cpu().numpy()) <= 1e-6


@pytest.mark.parametrize("opts", [dict(demote_below=1000, promote_min=0, row_scale=True),
                                  dict(engine="block", promote_min=0, row_scale=True,
                                       adjoint_options={"demote_below": 1000})])
def test_batched_all_512_graphs_fp64(cuda, opts):
    """The batched workload at full size: 512 power-law graphs (20-500
    nodes, mean degree 4-32), K = 64, forward and backward of the whole
    batch in one plan pair, against FP64 (every entry and row)."""
    g = graphs.batched(num_graphs=512)
    bs = BatchedStep(g, 64, device=cuda, **opts)
    b = graphs.dense_features(g.n_cols, 64, seed=1)
    dc = graphs.dense_features(g.n_rows, 64, seed=2)
    bs.b.copy_(torch.from_numpy(b))
    bs.dc.copy_(torch.from_numpy(dc))
    bs.run()
    torch.cuda.synchronize()
    v = np.asarray(g.values, np.float32)
    rows = np.repeat(np.arange(g.n_rows), np.diff(g.indptr))
    s = np.zeros(g.n_rows, np.float32)
    np.maximum.at(s, rows, np.abs(v))
    s[s == 0] = 1
    A16 = sp.csr_matrix(((v / s[rows]).astype(np.float16).astype(np.float64) * s[rows],
                         g.indices, g.indptr), shape=(g.n_rows, g.n_cols))
    st_ = np.zeros(g.n_cols, np.float32)
    np.maximum.at(st_, g.indices, np.abs(v))
    st_[st_ == 0] = 1
    AT16 = sp.csr_matrix(((v / st_[g.indices]).astype(np.float16).astype(np.float64)
                          * st_[g.indices], g.indices, g.indptr), shape=A16.shape).T
    assert rel_err(bs.c.cpu().numpy(), A16 @ b.astype(np.float64)) <= 1e-4
    assert rel_err(bs.db.cpu().numpy(), AT16 @ dc.astype(np.float64)) <= 1e-4
    dv_ref = oracle.sddmm_f64(g.indptr, g.indices, dc.astype(np.float64), b.astype(np.float64))
    assert rel_err(bs.dval.cpu().numpy(), dv_ref) <= 1e-5
