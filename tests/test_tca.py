"""TCA row reorder (tr_tca_order, the plan builder's reorder="tca", the
drop-in tr_csr_fp16.tr_tca_reorder.apply_tca_reorder) against the reference's
own apply_tca_reorder (golden fixture tests/golden/tca_orders.json, made by
tests/golden/make_tca_golden.py) and against the oracle's restatement
(oracle/tca.py) on seeded random graphs.  CPU only (host threads)."""
import hashlib
import json
import os

import numpy as np
import pytest

import oracle
import trspmm
from trspmm import core, graphs, plan_cache
from tr_csr_fp16.tr_tca_reorder import apply_tca_reorder

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = json.load(open(os.path.join(HERE, "golden", "tca_orders.json")))
# the fixture's graphs (same generators and seeds as make_tca_golden.py)
CASES = {
    "chung_lu_2048": lambda: graphs.chung_lu(n=2048),
    "route_mix_1024": lambda: graphs.route_mix(n=1024, target_nnz=50_000),
    "sbm_3000": lambda: graphs.sbm_powerlaw(n=3000, avg_degree=20, communities=30, seed=4),
    "ragged_500x300": lambda: graphs.random_csr(500, 300, 0.05, seed=2, empty_rows=0.4),
    "dup_300x200": lambda: graphs.random_csr(300, 200, 0.08, seed=7, dup=True),
    "batched_24": lambda: graphs.batched(num_graphs=24, seed=11),
    "rect_400x900": lambda: graphs.random_csr(400, 900, 0.02, seed=13, empty_rows=0.1),
}
_built = {}


def _graph(name):
    if name not in _built:
        _built[name] = CASES[name]()
    return _built[name]


def _checksum(g):
    return int(np.bitwise_xor.reduce((g.indices.astype(np.int64) * 2654435761
                                      + np.arange(g.nnz)) & 0xFFFFFFFF)) if g.nnz else 0


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.int32).tobytes()).hexdigest()


@pytest.mark.parametrize("t,n", [(0.2, 128), (0.5, 128), (0.8, 64), (0.1, 128), (0.35, 96)])
def test_lsh_banding_matches_oracle(t, n):
    assert core.lsh_params(t, n) == oracle.tca.lsh_params(t, n)


@pytest.mark.parametrize("name", list(CASES))
def test_order_matches_reference_golden(name):
    g = _graph(name)
    want = GOLDEN["cases"][name]
    assert (g.n_rows, g.nnz, _checksum(g)) == (want["rows"], want["nnz"], want["checksum"])
    order, st = core.tca_order(g.indptr, g.indices)
    assert order[:32].tolist() == want["order_head"]
    assert _sha(order) == want["order_sha256"]
    assert (st["pairs1"], st["clusters1"], st["pairs2"]) == (
        want["pairs1"], want["clusters1"], want["pairs2"])


@pytest.mark.parametrize("name", list(CASES))
def test_drop_in_matches_reference_golden(name):
    """apply_tca_reorder: the reference's reorder_id and new_col_ind; row
    pointers that describe the permuted rows (the reference's are all zero)."""
    g = _graph(name)
    want = GOLDEN["cases"][name]
    assert want["ref_row_ptr_last"] != g.nnz          # the reference's defect, recorded
    ptr, idx, order = apply_tca_reorder(g.indptr, g.indices, g.n_rows, verbose=False,
                                        device=False)
    assert _sha(order) == want["order_sha256"]
    assert _sha(idx) == want["col_ind_sha256"]
    deg = np.diff(g.indptr)
    assert np.array_equal(np.diff(ptr), deg[order]) and ptr[-1] == g.nnz
    for k in range(0, g.n_rows, max(1, g.n_rows // 50)):
        r = order[k]
        assert sorted(idx[ptr[k]:ptr[k + 1]]) == sorted(g.indices[g.indptr[r]:g.indptr[r + 1]])


@pytest.mark.parametrize("seed", range(6))
def test_matches_oracle_on_random_graphs(seed):
    rng = np.random.default_rng(300 + seed)
    n = int(rng.integers(20, 700))
    g = graphs.random_csr(n, int(rng.integers(5, 400)), float(rng.uniform(0.003, 0.2)), seed=seed,
                          empty_rows=float(rng.uniform(0, 0.5)), dup=bool(seed % 2))
    kw = dict(thres=int(rng.choice([1, 2, 4, 16, 40])),
              cluster_thres=int(rng.choice([1, 3, 128])),
              lsh_threshold=float(rng.choice([0.2, 0.5, 0.8])), seed=int(rng.integers(1, 1000)))
    want, wst = oracle.tca.tca_order(g.indptr, g.indices, **kw)
    got, st = core.tca_order(g.indptr, g.indices, **kw)
    assert np.array_equal(got, want)
    assert st == wst


def test_edge_cases_match_oracle():
    cases = [
        (np.array([0], np.int32), np.zeros(0, np.int32)),                     # no rows
        (np.zeros(7, np.int32), np.zeros(0, np.int32)),                       # all empty
        (np.array([0, 3], np.int32), np.array([5, 1, 5], np.int32)),          # one row, dup
        (np.array([0, 2, 4, 6], np.int32), np.array([0, 1, 0, 1, 0, 1], np.int32)),  # equal rows
        (np.array([0, 1, 2, 3, 3], np.int32), np.array([7, 8, 9], np.int32)),  # disjoint
    ]
    for ptr, idx in cases:
        got, st = core.tca_order(ptr, idx)
        want, wst = oracle.tca.tca_order(ptr, idx)
        assert np.array_equal(got, want), (ptr, idx)
        n = len(ptr) - 1
        assert sorted(got.tolist()) == list(range(n))
        if n:
            assert st == wst


def test_rejects_bad_arguments():
    g = _graph("ragged_500x300")
    with pytest.raises(trspmm.TrError, match="caps"):
        core.tca_order(g.indptr, g.indices, thres=0)
    with pytest.raises(trspmm.TrError, match="lsh_threshold"):
        core.tca_order(g.indptr, g.indices, lsh_threshold=1.0)
    with pytest.raises(trspmm.TrError, match=">= 0"):
        core.tca_order(np.array([0, 1], np.int32), np.array([-3], np.int32))
    with pytest.raises(trspmm.TrError, match="non-decreasing"):
        core.tca_order(np.array([0, 2, 1], np.int32), np.array([0, 1], np.int32))
    with pytest.raises(trspmm.TrError, match="max_pairs"):
        core.tca_order(g.indptr, g.indices, max_pairs=10)
    with pytest.raises(trspmm.TrError, match="num_perm"):
        core.lsh_params(0.2, 0)


def test_plan_rows_follow_the_tca_order():
    g = graphs.sbm_powerlaw(n=3000, avg_degree=24, communities=30, seed=6)
    order, _ = core.tca_order(g.indptr, g.indices)
    P = trspmm.host_plan(g.indptr, g.indices, g.values, g.n_rows, g.n_cols, reorder="tca")
    assert np.array_equal(P["row_out"][:g.n_rows], order)
    # the caller's permutation gives the same plan
    Q = trspmm.host_plan(g.indptr, g.indices, g.values, g.n_rows, g.n_cols, reorder=order)
    for k in ("row_out", "res_col", "res_ptr", "tile_col", "win_order", "val_slot"):
        assert np.array_equal(P[k], Q[k]), k
    # TCA puts rows that share columns together: fewer (window, column) gathers
    plain = trspmm.host_plan(g.indptr, g.indices, g.values, g.n_rows, g.n_cols, promote_min=1)
    tca = trspmm.host_plan(g.indptr, g.indices, g.values, g.n_rows, g.n_cols, promote_min=1,
                           reorder="tca")
    gathers = lambda H: int((H["tile_col"] >= 0).sum()) + len(H["res_col"])
    assert gathers(tca) < gathers(plain)


def test_given_order_is_validated():
    g = _graph("ragged_500x300")
    bad = np.arange(g.n_rows, dtype=np.int32)
    bad[3] = bad[4]
    with pytest.raises(trspmm.TrError, match="permutation"):
        trspmm.host_plan(g.indptr, g.indices, g.values, g.n_rows, g.n_cols, reorder=bad)
    with pytest.raises(ValueError, match="reorder"):
        trspmm.host_plan(g.indptr, g.indices, g.values, g.n_rows, g.n_cols, reorder="minhash")


def test_plan_cache_keys_name_the_mode():
    g = _graph("dup_300x200")
    keys = {m: plan_cache.plan_key(g.indptr, g.indices, g.values, g.n_rows, g.n_cols, reorder=m)
            for m in (False, True, "label", "tca")}
    assert keys[True] == keys["label"]
    assert len({keys[False], keys[True], keys["tca"]}) == 3
    with pytest.raises(ValueError):
        plan_cache.plan_key(g.indptr, g.indices, g.values, g.n_rows, g.n_cols,
                            reorder=np.arange(g.n_rows))


def test_loader_reorders_rows_when_asked(monkeypatch):
    """LIBRA_TCA_REORDER=1 (mdataset2_online.py:72-91): the routed CSR is the
    TCA-permuted one, with every row's columns kept."""
    from tr_csr_fp16.mdataset2_online import GCN_dataset_tcu_sptc_cuda_online as DS
    g = graphs.chung_lu(n=1000, avg_degree=8, seed=3)
    monkeypatch.setenv("LIBRA_TCA_REORDER", "1")
    d = DS.from_csr(g.indptr, g.indices, g.n_cols, 16)
    order, _ = core.tca_order(g.indptr, g.indices)
    assert np.array_equal(d.reorder_id, order)
    ptr, idx = d.row_pointers.numpy(), d.column_index.numpy()
    assert len(ptr) == d.num_nodes + 1 and ptr[-1] == g.nnz
    for k in range(0, g.n_rows, 37):
        r = order[k]
        assert sorted(idx[ptr[k]:ptr[k + 1]]) == sorted(g.indices[g.indptr[r]:g.indptr[r + 1]])
    monkeypatch.setenv("LIBRA_TCA_REORDER", "0")
    d0 = DS.from_csr(g.indptr, g.indices, g.n_cols, 16)
    assert d0.reorder_id is None and np.array_equal(d0.row_pointers.numpy()[:g.n_rows + 1], g.indptr)


def test_device_stages_without_a_gpu_raise():
    import torch
    if torch.cuda.is_available():
        pytest.skip("checks the error path of a machine without a CUDA device")
    g = _graph("dup_300x200")
    with pytest.raises(trspmm.TrError, match="TCA signatures"):
        core.tca_order(g.indptr, g.indices, device=True)
