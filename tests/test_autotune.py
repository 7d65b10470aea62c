"""The autotuner's host side (sampling, cache keys) on the CPU, and one
tuning run on the GPU: every candidate is timed, the winner's plan computes
the product (FP64 check), and the cache answers the second call."""
import numpy as np
import pytest
import scipy.sparse as sp

from trspmm import autotune, graphs


def test_sample_rows_keeps_whole_rows():
    g = graphs.chung_lu(n=4096)
    ip, ix, vv, m, n = autotune.sample_csr(g.indptr, g.indices, g.values, g.n_rows, g.n_cols,
                                           False, 10_000)
    assert n == g.n_cols and 0 < m < g.n_rows
    assert ip[-1] <= 10_000 and ip[-1] == g.indptr[m]
    assert np.array_equal(ip, g.indptr[:m + 1]) and np.array_equal(ix, g.indices[:ip[-1]])


def test_sample_columns_for_the_adjoint():
    g = graphs.sbm_powerlaw(n=3000, avg_degree=20, communities=30)
    ip, ix, vv, m, n = autotune.sample_csr(g.indptr, g.indices, g.values, g.n_rows, g.n_cols,
                                           True, 12_000)
    assert m == g.n_rows and 0 < n < g.n_cols
    A = sp.csr_matrix((g.values, g.indices, g.indptr), shape=(g.n_rows, g.n_cols))
    S = sp.csr_matrix((vv, ix, ip), shape=(m, n))
    assert (abs(S - A[:, :n]) > 0).nnz == 0
    assert ix.size <= 12_000 + A[:, n - 1].nnz


def test_small_graphs_are_not_sampled():
    g = graphs.chung_lu(n=512)
    out = autotune.sample_csr(g.indptr, g.indices, g.values, g.n_rows, g.n_cols, False, 10**9)
    assert out[0] is g.indptr and out[3] == g.n_rows


def test_cache_key_buckets():
    a = autotune.cache_key("B200", 128, 10_000_000, 200_000, False)
    b = autotune.cache_key("B200", 128, 10_100_000, 201_000, False)
    assert a == b
    assert a != autotune.cache_key("B200", 128, 10_000_000, 200_000, True)
    assert autotune.cache_key("B200", 128, 1, 1, True, backward=True).endswith("bwd")


@pytest.mark.gpu
def test_tune_small_graph(cuda, tmp_path, monkeypatch):
    import torch
    import oracle
    import trspmm
    from helpers import rel_err
    monkeypatch.setenv("TRSPMM_AUTOTUNE_CACHE", str(tmp_path / "tune.json"))
    g = graphs.sbm_powerlaw(n=6000, avg_degree=30, communities=60)
    best, rep = autotune.tune(g.indptr, g.indices, g.values, g.n_rows, g.n_cols, 128,
                              device=cuda, row_scale=True, reps=3, sample_nnz=100_000)
    assert not rep["cached"] and rep["sample"]["nnz"] <= 100_000 + 200
    timed = [r["options"] for r in rep["results"]]
    assert {"engine": "block", "reorder": True, "k_tile": 64} in timed
    assert all(r["ms"] > 0 for r in rep["results"])
    # the engine is decided at full size among each family's best layout
    fams = {r["options"].get("engine", "window") for r in rep["full"]}
    assert fams == {"window", "block"} and best in [r["options"] for r in rep["full"]]
    plan = trspmm.Plan.build(g.indptr, g.indices, g.values, g.n_rows, g.n_cols, row_scale=True,
                             **best)
    P = trspmm.host_plan(g.indptr, g.indices, g.values, g.n_rows, g.n_cols, row_scale=True, **best)
    b = graphs.dense_features(g.n_cols, 128, seed=2)
    out = plan.spmm(torch.from_numpy(b).to(cuda))
    torch.cuda.synchronize()
    assert rel_err(out.cpu().numpy(), oracle.decode_plan(P)["all"] @ b.astype(np.float64)) <= 1e-4
    best2, rep2 = autotune.tune(g.indptr, g.indices, g.values, g.n_rows, g.n_cols, 128,
                                device=cuda, row_scale=True, reps=3, sample_nnz=100_000)
    assert rep2["cached"] and best2 == best
