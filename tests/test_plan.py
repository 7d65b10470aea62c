"""The native plan builder (host side, no device): the plan a kernel reads
encodes exactly A (or A^T), whatever the options — row scaling, promotion of
shared residual columns to tensor-core tiles, row clustering — and its
entry -> slot map finds every value.  Checked with the oracle's plan decoder."""
import numpy as np
import pytest
import scipy.sparse as sp

import oracle
import trspmm
from trspmm import graphs

GRAPHS = {
    "random_ragged": lambda: graphs.random_csr(300, 280, 0.05, seed=3, empty_rows=0.3),
    "chung_lu": lambda: graphs.chung_lu(n=2000, avg_degree=12, seed=4),
    "route_mix": lambda: graphs.route_mix(n=2048, target_nnz=100_000, seed=5),
    "sbm": lambda: graphs.sbm_powerlaw(n=3000, avg_degree=24, communities=30, seed=6),
    "batched": lambda: graphs.batched(num_graphs=10, seed=7),
}
OPTS = [
    dict(),
    dict(row_scale=True),
    dict(promote_min=2),
    dict(promote_min=1, row_scale=True),
    dict(transpose=True),
    dict(transpose=True, promote_min=2, row_scale=True),
    dict(reorder=True),
    dict(reorder=True, transpose=True, promote_min=2, row_scale=True),
    dict(demote_below=3),
    dict(demote_below=4, promote_min=4, reorder=True, row_scale=True),
    # every 2:4 column demoted: the group entries go straight to the residual
    dict(demote_below=1000, row_scale=True),
    dict(demote_below=17, transpose=True, promote_min=2),
    dict(demote_below=1000, reorder=True, transpose=True, row_scale=True),
    dict(reorder="tca"),
    dict(reorder="tca", transpose=True, promote_min=2, row_scale=True),
]


def _expected(g, transpose, row_scale):
    """A (or A^T) with the values the plan must hold: FP16(v / s_r) * s_r,
    s_r = max |v| over the (transposed) row in FP32, s_r = 1 without scaling."""
    A = sp.csr_matrix((np.asarray(g.values, np.float32), g.indices, g.indptr),
                      shape=(g.n_rows, g.n_cols))
    if transpose:
        A = A.T.tocsr()
    A.sort_indices()
    rows = np.repeat(np.arange(A.shape[0]), np.diff(A.indptr))
    v = A.data.astype(np.float32)
    if row_scale:
        s = np.zeros(A.shape[0], np.float32)
        np.maximum.at(s, rows, np.abs(v))
        s[s == 0] = 1
    else:
        s = np.ones(A.shape[0], np.float32)
    q = (v / s[rows]).astype(np.float16).astype(np.float64) * s[rows].astype(np.float64)
    return sp.csr_matrix((q, A.indices, A.indptr), shape=A.shape)


@pytest.mark.parametrize("opt", range(len(OPTS)), ids=lambda i: "-".join(
    f"{k}={v}" for k, v in OPTS[i].items()) or "default")
@pytest.mark.parametrize("name", list(GRAPHS))
def test_plan_encodes_matrix(name, opt):
    g = GRAPHS[name]()
    o = OPTS[opt]
    P = trspmm.host_plan(g.indptr, g.indices, g.values, g.n_rows, g.n_cols, **o)
    D = oracle.decode_plan(P)
    ref = _expected(g, o.get("transpose", False), o.get("row_scale", False))
    diff = abs(D["all"] - ref)
    assert diff.nnz == 0 or diff.max() <= 1e-12 * max(abs(ref).max(), 1)
    # every plan row lands in a distinct output row; padding rows nowhere
    ro = P["row_out"]
    n_out = ref.shape[0]
    assert np.array_equal(np.sort(ro[ro >= 0]), np.arange(n_out))
    # the entry -> slot map reads back every entry's value (exact mode)
    v = oracle.plan_value_of_entries(P)
    assert not np.isnan(v).any(), "entry without a value slot"
    w = np.asarray(g.values, np.float32)
    # the value the plan holds for entry e: compare entry by entry through A's order
    A = sp.csr_matrix((np.arange(1, g.nnz + 1, dtype=np.float64), g.indices, g.indptr),
                      shape=(g.n_rows, g.n_cols))
    if o.get("transpose"):
        rows_t = g.indices
        s = np.zeros(g.n_cols, np.float32)
        if o.get("row_scale"):
            np.maximum.at(s, rows_t, np.abs(w))
        s[s == 0] = 1
        srow = s[rows_t]
    else:
        rows = np.repeat(np.arange(g.n_rows), np.diff(g.indptr))
        s = np.zeros(g.n_rows, np.float32)
        if o.get("row_scale"):
            np.maximum.at(s, rows, np.abs(w))
        s[s == 0] = 1
        srow = s[rows]
    want = (w / srow).astype(np.float16).astype(np.float64) * srow
    assert np.allclose(v, want, rtol=0, atol=0), "plan value of an entry differs"
    # residual slot -> entry is the inverse of entry -> slot on the residual
    T = len(P["tile_col"]) // 16
    re_ = P["res_edge"]
    assert len(re_) == len(P["res_col"]) and (re_ >= 0).all()
    assert np.array_equal(P["val_slot"][re_], T * 256 + np.arange(len(re_)))
    del A


def test_promotion_moves_shared_columns_only():
    g = graphs.sbm_powerlaw(n=3000, avg_degree=24, communities=30, seed=6)
    base = trspmm.host_plan(g.indptr, g.indices, g.values, g.n_rows, g.n_cols)
    P = trspmm.host_plan(g.indptr, g.indices, g.values, g.n_rows, g.n_cols, promote_min=2)
    D = oracle.decode_plan(P)
    assert D["prom"].nnz > 0
    assert len(P["res_col"]) < len(base["res_col"])
    # a promoted column slot holds >= 2 entries of its window
    wt, prom = P["win_tile"], P["win_prom"]
    a = P["tile_a"].view(np.float16).reshape(-1, 256)
    i = np.arange(256)
    k_of = ((i % 128) // 64) * 8 + (i % 8)
    for w in range(len(wt) - 1):
        for t in range(int(prom[w]), int(wt[w + 1])):
            cnt = np.bincount(k_of[a[t] != 0], minlength=16)
            used = P["tile_col"][t * 16:(t + 1) * 16] >= 0
            assert (cnt[used] >= 2).all()
    # promote_min = 1 empties the residual (no repeated (row, col) in this graph)
    P1 = trspmm.host_plan(g.indptr, g.indices, g.values, g.n_rows, g.n_cols, promote_min=1)
    assert len(P1["res_col"]) == 0


def test_demotion_moves_thin_sptc_columns_only():
    g = graphs.route_mix(n=2048, target_nnz=100_000, seed=5)
    base = trspmm.host_plan(g.indptr, g.indices, g.values, g.n_rows, g.n_cols)
    P = trspmm.host_plan(g.indptr, g.indices, g.values, g.n_rows, g.n_cols, demote_below=4)
    assert len(P["res_col"]) > len(base["res_col"])
    Db, D = oracle.decode_plan(base), oracle.decode_plan(P)
    assert D["sptc"].nnz < Db["sptc"].nnz and D["tc"].nnz == Db["tc"].nnz
    wt, split, prom = P["win_tile"], P["win_split"], P["win_prom"]
    a = P["tile_a"].view(np.float16).reshape(-1, 256)
    i = np.arange(256)
    k_of = ((i % 128) // 64) * 8 + (i % 8)
    for w in range(len(wt) - 1):
        for t in range(int(split[w]), int(prom[w])):
            cnt = np.bincount(k_of[a[t] != 0], minlength=16)
            used = P["tile_col"][t * 16:(t + 1) * 16] >= 0
            assert used.any() and (cnt[used] >= 4).all()


def test_duplicate_entries_stay_exact():
    # repeated (row, column) entries: a tile slot holds one, the rest stay residual
    indptr = np.array([0, 4, 6], np.int32)
    indices = np.array([3, 3, 5, 3, 5, 5], np.int32)
    values = np.array([1.0, 2.0, 0.5, 4.0, 1.5, -1.0], np.float32)
    for pm in (0, 1, 2):
        P = trspmm.host_plan(indptr, indices, values, 2, 8, promote_min=pm)
        D = oracle.decode_plan(P)["all"].toarray()
        want = np.zeros((2, 8))
        np.add.at(want, (np.repeat([0, 1], [4, 2]), indices), values)
        assert np.allclose(D, want)
        assert not np.isnan(oracle.plan_value_of_entries(P)).any()


def test_reorder_clusters_communities():
    """Randomly permuted SBM: clustering rows before routing cuts the number
    of distinct (window, column) pairs, i.e. the feature rows gathered."""
    g = graphs.sbm_powerlaw(n=4000, avg_degree=30, communities=40, seed=11)

    def gathers(P):
        wt = P["win_tile"]
        n_tiles_cols = int((P["tile_col"] >= 0).sum())
        return n_tiles_cols + len(P["res_col"]), len(wt) - 1

    plain = trspmm.host_plan(g.indptr, g.indices, g.values, g.n_rows, g.n_cols, promote_min=1)
    clus = trspmm.host_plan(g.indptr, g.indices, g.values, g.n_rows, g.n_cols, promote_min=1,
                            reorder=True)
    gp, _ = gathers(plain)
    gc, _ = gathers(clus)
    assert gc * 1.3 < gp, (gc, gp)
    ro = clus["row_out"]
    assert not np.array_equal(ro[: g.n_rows], np.arange(g.n_rows))


def test_builder_rejects_malformed_csr():
    with pytest.raises(trspmm.TrError, match="out of range"):
        trspmm.host_plan(np.array([0, 1], np.int32), np.array([9], np.int32),
                         np.ones(1, np.float32), 1, 4)
    with pytest.raises(trspmm.TrError, match="non-decreasing"):
        trspmm.host_plan(np.array([0, 2, 1], np.int32), np.array([0, 1], np.int32),
                         np.ones(2, np.float32), 2, 4)
    with pytest.raises(trspmm.TrError, match="promote_min"):
        trspmm.host_plan(np.array([0, 1], np.int32), np.array([0], np.int32),
                         np.ones(1, np.float32), 1, 4, promote_min=-1)


def test_empty_matrix_plan():
    P = trspmm.host_plan(np.zeros(1, np.int32), np.zeros(0, np.int32), np.zeros(0, np.float32),
                         0, 5)
    assert len(P["win_tile"]) == 1 and len(P["val_slot"]) == 0
    P = trspmm.host_plan(np.zeros(4, np.int32), np.zeros(0, np.int32), np.zeros(0, np.float32),
                         3, 5, transpose=True, reorder=True)
    assert oracle.decode_plan(P)["all"].nnz == 0


def test_skip_sptc_routes_every_non_tc_column_to_cuda():
    """skip_sptc (set by the builder when demote_below > 16): no 2:4 groups,
    the dense-TC funnel unchanged, the CUDA parts hold every other entry."""
    g = graphs.route_mix(n=2048, target_nnz=100_000, seed=5)
    full = trspmm.route(g.indptr, g.indices, g.values, mode="exact")
    skip = trspmm.route(g.indptr, g.indices, g.values, mode="exact", skip_sptc=True)
    names = trspmm.TABLE_NAMES
    assert skip[names.index("s_column")].size == 0
    for t in ("t_column", "t_binary", "t_value"):
        assert np.array_equal(full[names.index(t)], skip[names.index(t)]), t
    dec = oracle.decode_tables(skip, g.n_rows, g.n_cols)
    A = sp.csr_matrix((np.asarray(g.values, np.float64), g.indices, g.indptr),
                      shape=(g.n_rows, g.n_cols))
    assert abs(dec["all"] - A).max() <= 1e-3 * abs(A).max()     # FP16 TC values
    assert dec["sptc"].nnz == 0


@pytest.mark.parametrize("engine", ["window", "block"])
@pytest.mark.parametrize("transpose", [False, True])
def test_memoised_label_order_builds_the_label_plan(engine, transpose):
    """reorder=True computes the label order once per matrix
    (trspmm.core.label_order, tr_label_order) and passes it on as the
    caller's permutation; the plan equals the builder's own label mode
    (TR_REORDER_LABEL) array for array."""
    import ctypes
    from trspmm import core
    g = graphs.sbm_powerlaw(n=3000, avg_degree=16, communities=30, seed=8)
    ip, ix, vv = g.indptr, g.indices, g.values
    memo = core.host_plan(ip, ix, vv, g.n_rows, g.n_cols, row_scale=True, transpose=transpose,
                          reorder=True, engine=engine, demote_below=1000)
    # the builder's own label mode, bypassing the memoised order
    rp = np.ascontiguousarray(ip, dtype=np.int32)
    ci = np.ascontiguousarray(ix, dtype=np.int32)
    va = np.ascontiguousarray(vv, dtype=np.float32)
    prm = core._params(mode="exact")
    opts, _keep = core.plan_opts(True, 0, transpose, True, 1000, engine)
    assert opts.reorder == core.TR_REORDER_LABEL
    h = ctypes.c_void_p()
    core.check(trspmm.lib().tr_plan_build_host(core._vp(rp), core._vp(ci), core._vp(va),
                                               g.n_rows, g.n_cols, ctypes.byref(prm),
                                               ctypes.byref(opts), ctypes.byref(h)))
    try:
        own = core.host_plan_arrays(h)
    finally:
        trspmm.lib().tr_host_plan_free(h)
    for name, arr in own.items():
        assert np.array_equal(memo[name], arr), name
    order = core.label_order(ip, ix, g.n_rows, g.n_cols, transpose)
    assert core.label_order(ip, ix, g.n_rows, g.n_cols, transpose) is order     # memoised
    assert np.array_equal(np.sort(order), np.arange(order.size))
    assert np.array_equal(own["row_out"][: order.size], order)


def test_label_order_edge_cases():
    """tr_label_order: no rows, no entries, at most 16 rows (kept in natural
    order, as the builder does), A^T's row count, malformed CSR refused."""
    from trspmm import core
    assert core.label_order(np.zeros(1, np.int32), np.zeros(0, np.int32), 0, 5).size == 0
    g = graphs.random_csr(40, 7, 0.0, seed=1)
    assert np.array_equal(core.label_order(g.indptr, g.indices, 40, 7), np.arange(40))
    g = graphs.random_csr(12, 30, 0.3, seed=2)
    assert np.array_equal(core.label_order(g.indptr, g.indices, 12, 30), np.arange(12))
    g = graphs.random_csr(300, 50, 0.1, seed=3)
    o = core.label_order(g.indptr, g.indices, 300, 50, transpose=True)
    assert np.array_equal(np.sort(o), np.arange(50))
    bad = g.indices.copy()
    bad[0] = 50
    with pytest.raises(trspmm.TrError):
        core.label_order(g.indptr, bad, 300, 50)
