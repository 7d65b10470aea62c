"""Block layout (engine="block") on the CPU: the plan encodes exactly A (or
A^T), every entry has one tile position and one value slot, plan files keep
block plans, and malformed block arrays are refused on load."""
import os

import numpy as np
import pytest
import scipy.sparse as sp

import oracle
import trspmm
from helpers import rel_err
from trspmm import graphs, plan_cache

CASES = {
    "chung_lu": lambda: graphs.chung_lu(n=1000),
    "dup_ragged": lambda: graphs.random_csr(300, 500, 0.05, seed=2, dup=True, empty_rows=0.2),
    "sbm": lambda: graphs.sbm_powerlaw(n=3000, communities=30),
    "rect": lambda: graphs.random_csr(257, 1000, 0.02, seed=4),
    "empty": lambda: graphs.random_csr(200, 50, 0.0, seed=1),
}


def _a(g, transpose):
    A = sp.csr_matrix((g.values.astype(np.float64), g.indices, g.indptr), shape=(g.n_rows, g.n_cols))
    return A.T.tocsr() if transpose else A


@pytest.mark.parametrize("name", list(CASES))
@pytest.mark.parametrize("transpose", [False, True])
@pytest.mark.parametrize("reorder", [False, True])
@pytest.mark.parametrize("row_scale", [False, True])
def test_block_plan_encodes_a(name, transpose, reorder, row_scale):
    g = CASES[name]()
    P = trspmm.host_plan(g.indptr, g.indices, g.values, g.n_rows, g.n_cols, engine="block",
                         transpose=transpose, reorder=reorder, row_scale=row_scale)
    A = _a(g, transpose)
    dec = oracle.decode_plan(P)["all"]          # asserts unique tile positions
    if A.nnz:
        # FP16 storage of v / row_scale: half an FP16 ulp of the largest value
        assert rel_err(dec.toarray(), A.toarray()) <= 2 ** -11
    else:
        assert dec.nnz == 0
    v = oracle.plan_value_of_entries(P)
    assert not np.isnan(v).any()
    if g.nnz:
        assert np.abs(v - g.values).max() <= 2 ** -11 * max(np.abs(g.values).max(), 1e-30)
    n_chunks = len(P["chunk_ent"]) - 1
    assert len(P["chunk_col"]) == 16 * n_chunks
    assert P["ent_src"].size == g.nnz and np.array_equal(np.sort(P["ent_src"]), np.arange(g.nnz))
    assert np.array_equal(np.sort(P["blk_order"]), np.arange(len(P["blk_chunk"]) - 1))


def test_each_column_gathered_once_per_block():
    """Without duplicate entries a block holds each of its columns in exactly
    one slot: the gather count is the number of distinct (block, column)
    pairs, padded to whole chunks."""
    g = graphs.sbm_powerlaw(n=3000, communities=30)
    P = trspmm.host_plan(g.indptr, g.indices, g.values, g.n_rows, g.n_cols, engine="block")
    bc, cc = P["blk_chunk"], P["chunk_col"]
    rows = np.repeat(np.arange(g.n_rows), np.diff(g.indptr))
    pairs = np.unique((rows // 128).astype(np.int64) * g.n_cols + g.indices).size
    assert (cc >= 0).sum() == pairs
    for b in range(len(bc) - 1):
        cols = cc[bc[b] * 16:bc[b + 1] * 16]
        cols = cols[cols >= 0]
        assert np.unique(cols).size == cols.size


def test_block_plan_file_round_trip(tmp_path):
    g = graphs.sbm_powerlaw(n=3000, communities=30)
    kw = dict(engine="block", row_scale=True, reorder=True, transpose=True)
    h, path, hit = plan_cache.cached_host_plan(g.indptr, g.indices, g.values, g.n_rows, g.n_cols,
                                               directory=str(tmp_path), **kw)
    a = trspmm.core.host_plan_arrays(h)
    trspmm.lib().tr_host_plan_free(h)
    assert not hit and os.path.exists(path)
    h2, _, hit2 = plan_cache.cached_host_plan(g.indptr, g.indices, g.values, g.n_rows, g.n_cols,
                                              directory=str(tmp_path), **kw)
    b = trspmm.core.host_plan_arrays(h2)
    trspmm.lib().tr_host_plan_free(h2)
    assert hit2
    for name in a:
        assert np.array_equal(a[name], b[name]), name
    # a different engine is a different cache entry
    assert plan_cache.plan_key(g.indptr, g.indices, g.values, g.n_rows, g.n_cols) != \
        plan_cache.plan_key(g.indptr, g.indices, g.values, g.n_rows, g.n_cols, engine="block")


def test_block_plan_file_refuses_bad_positions(tmp_path):
    """A block plan file whose tile offset lies outside the 4 KiB tile (with a
    matching checksum) is refused: the kernels would write past the tile."""
    import ctypes
    g = graphs.chung_lu(n=600)
    h, path, _ = plan_cache.cached_host_plan(g.indptr, g.indices, g.values, g.n_rows, g.n_cols,
                                             directory=str(tmp_path), engine="block")
    trspmm.lib().tr_host_plan_free(h)
    raw = bytearray(open(path, "rb").read())
    P = trspmm.host_plan(g.indptr, g.indices, g.values, g.n_rows, g.n_cols, engine="block")
    needle = P["ent_pos"][:8].tobytes()
    at = bytes(raw).find(needle)
    assert at > 0
    raw[at:at + 2] = np.uint16(5000).tobytes()
    body = bytes(raw[:-8])
    hsh = 1469598103934665603
    for x in body:
        hsh = ((hsh ^ x) * 1099511628211) & 0xFFFFFFFFFFFFFFFF
    raw[-8:] = hsh.to_bytes(8, "little")
    bad = tmp_path / "bad.trplan"
    bad.write_bytes(bytes(raw))
    out = ctypes.c_void_p()
    rc = trspmm.lib().tr_host_plan_load(str(bad).encode(), ctypes.byref(out))
    assert rc == 1 and b"inconsistent" in trspmm.lib().tr_last_error()


def test_unknown_engine_refused():
    g = graphs.chung_lu(n=200)
    with pytest.raises(ValueError):
        trspmm.host_plan(g.indptr, g.indices, g.values, g.n_rows, g.n_cols, engine="warp")
