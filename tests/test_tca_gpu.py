"""TCA row reorder with the signatures and Jaccard similarities on the GPU
(tr_tca_order with device = 1): the same order, bit for bit, as the host
threads (which the CPU tests pin to the reference and the oracle); plans
built on the TCA order multiply correctly."""
import numpy as np
import pytest
import torch

import trspmm
from trspmm import core, graphs
from tr_csr_fp16.tr_tca_reorder import apply_tca_reorder

pytestmark = pytest.mark.gpu

GRAPHS = {
    "chung_lu_2048": lambda: graphs.chung_lu(n=2048),
    "route_mix_8192": lambda: graphs.route_mix(n=8192, target_nnz=400_000),
    "sbm_20000": lambda: graphs.sbm_powerlaw(n=20000, avg_degree=30, communities=200, seed=4),
    "ragged_500x300": lambda: graphs.random_csr(500, 300, 0.05, seed=2, empty_rows=0.4),
    "dup_300x200": lambda: graphs.random_csr(300, 200, 0.08, seed=7, dup=True),
    "sparse_wide": lambda: graphs.random_csr(3000, 20000, 0.002, seed=5, empty_rows=0.2),
}


@pytest.mark.parametrize("name", list(GRAPHS))
def test_device_order_equals_host_order(name):
    g = GRAPHS[name]()
    h, hs = core.tca_order(g.indptr, g.indices, device=False)
    d, ds = core.tca_order(g.indptr, g.indices, device=True)
    assert np.array_equal(h, d)
    assert hs == ds


def test_drop_in_uses_the_gpu_by_default():
    g = GRAPHS["chung_lu_2048"]()
    p1, i1, o1 = apply_tca_reorder(g.indptr, g.indices, g.n_rows, verbose=False)
    p0, i0, o0 = apply_tca_reorder(g.indptr, g.indices, g.n_rows, verbose=False, device=False)
    assert np.array_equal(o1, o0) and np.array_equal(p1, p0) and np.array_equal(i1, i0)


@pytest.mark.parametrize("name,k", [("sbm_20000", 128), ("route_mix_8192", 64),
                                    ("ragged_500x300", 40)])
def test_tca_ordered_plan_multiplies(name, k):
    g = GRAPHS[name]()
    dev = torch.device("cuda:0")
    order, _ = core.tca_order(g.indptr, g.indices, device=True)
    for reorder in ("tca", order):
        plan = trspmm.Plan.build(g.indptr, g.indices, g.values, g.n_rows, g.n_cols,
                                 reorder=reorder, row_scale=True)
        b = graphs.dense_features(g.n_cols, k, seed=9)
        c = plan.spmm(torch.from_numpy(b).to(dev)).cpu().numpy().astype(np.float64)
        import scipy.sparse as sp
        A = sp.csr_matrix((g.values.astype(np.float64), g.indices, g.indptr),
                          shape=(g.n_rows, g.n_cols))
        ref = A @ b.astype(np.float64)
        err = np.abs(c - ref).max() / max(np.abs(ref).max(), 1e-30)
        assert err <= 2e-3, err              # FP16 operands, FP32 accumulation
