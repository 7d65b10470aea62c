"""Plan files and the on-disk plan cache (tr_host_plan_save / _load,
trspmm.plan_cache): a saved plan loads back array for array; the cache
routes once per key and rebuilds damaged files; loading refuses files that
are not plan files, truncated or damaged ones.  The device check (a cached
plan multiplies like a freshly built one) is marked gpu."""
import ctypes
import os

import numpy as np
import pytest
import torch

import trspmm
from trspmm import graphs, plan_cache
from trspmm.core import host_plan_arrays
from trspmm._lib import check, lib

G = graphs.route_mix(n=1024, target_nnz=60_000)
OPTS = dict(row_scale=True, promote_min=2, demote_below=3)


def _load(path):
    h = ctypes.c_void_p()
    check(lib().tr_host_plan_load(str(path).encode(), ctypes.byref(h)))
    return h


def _arrays_equal(a, b):
    assert a.keys() == b.keys()
    for k in a:
        assert a[k].dtype == b[k].dtype and np.array_equal(a[k], b[k]), k


@pytest.mark.parametrize("transpose", [False, True])
def test_cache_routes_once_and_round_trips(tmp_path, transpose):
    h1, path, hit1 = plan_cache.cached_host_plan(G.indptr, G.indices, G.values, G.n_rows, G.n_cols,
                                                 str(tmp_path), transpose=transpose, **OPTS)
    h2, path2, hit2 = plan_cache.cached_host_plan(G.indptr, G.indices, G.values, G.n_rows, G.n_cols,
                                                  str(tmp_path), transpose=transpose, **OPTS)
    try:
        assert (hit1, hit2) == (False, True) and path == path2 and os.path.exists(path)
        a, b = host_plan_arrays(h1), host_plan_arrays(h2)
        _arrays_equal(a, b)
        want = trspmm.host_plan(G.indptr, G.indices, G.values, G.n_rows, G.n_cols,
                                transpose=transpose, **OPTS)
        _arrays_equal(a, {k: want[k] for k in a})
    finally:
        lib().tr_host_plan_free(h1)
        lib().tr_host_plan_free(h2)


def test_key_depends_on_graph_values_and_options():
    k = plan_cache.plan_key(G.indptr, G.indices, G.values, G.n_rows, G.n_cols, **OPTS)
    assert k == plan_cache.plan_key(G.indptr, G.indices, G.values.copy(), G.n_rows, G.n_cols, **OPTS)
    v2 = G.values.copy()
    v2[0] += 1
    assert k != plan_cache.plan_key(G.indptr, G.indices, v2, G.n_rows, G.n_cols, **OPTS)
    assert k != plan_cache.plan_key(G.indptr, G.indices, G.values, G.n_rows, G.n_cols,
                                    **dict(OPTS, demote_below=4))
    assert k != plan_cache.plan_key(G.indptr, G.indices, G.values, G.n_rows, G.n_cols, density=4,
                                    **OPTS)
    ix = G.indices.copy()
    ix[[0, 1]] = ix[[1, 0]]
    assert k != plan_cache.plan_key(G.indptr, ix, G.values, G.n_rows, G.n_cols, **OPTS)


def test_damaged_files_are_refused_and_rebuilt(tmp_path):
    h, path, hit = plan_cache.cached_host_plan(G.indptr, G.indices, G.values, G.n_rows, G.n_cols,
                                               str(tmp_path), **OPTS)
    good = host_plan_arrays(h)
    lib().tr_host_plan_free(h)
    raw = open(path, "rb").read()
    # one flipped byte in the middle
    bad = bytearray(raw)
    bad[len(bad) // 2] ^= 0x5A
    open(path, "wb").write(bytes(bad))
    with pytest.raises(trspmm.TrError, match="checksum"):
        _load(path)
    h, _, hit = plan_cache.cached_host_plan(G.indptr, G.indices, G.values, G.n_rows, G.n_cols,
                                            str(tmp_path), **OPTS)
    assert not hit                                  # rebuilt, and the file replaced
    _arrays_equal(host_plan_arrays(h), good)
    lib().tr_host_plan_free(h)
    assert open(path, "rb").read() == raw
    # truncated
    open(path, "wb").write(raw[: len(raw) // 3])
    with pytest.raises(trspmm.TrError, match="checksum"):
        _load(path)
    # not a plan file at all
    junk = tmp_path / "junk.trplan"
    junk.write_bytes(b"\x00" * 64)
    with pytest.raises(trspmm.TrError, match="not a plan file"):
        _load(junk)
    with pytest.raises(trspmm.TrError, match="cannot open"):
        _load(tmp_path / "missing.trplan")


def test_unwritable_directory_only_skips_caching(tmp_path):
    blocker = tmp_path / "file"
    blocker.write_text("x")
    h, path, hit = plan_cache.cached_host_plan(G.indptr, G.indices, G.values, G.n_rows, G.n_cols,
                                               str(blocker / "sub"), **OPTS)
    assert not hit and not os.path.exists(path)
    lib().tr_host_plan_free(h)


@pytest.mark.gpu
def test_cached_plan_multiplies_like_a_built_one(tmp_path, cuda):
    b = torch.randn(G.n_cols, 64, device=cuda).half()
    built = trspmm.Plan.build(G.indptr, G.indices, G.values, G.n_rows, G.n_cols, **OPTS)
    first = plan_cache.cached_plan(G.indptr, G.indices, G.values, G.n_rows, G.n_cols,
                                   str(tmp_path), **OPTS)
    again = plan_cache.cached_plan(G.indptr, G.indices, G.values, G.n_rows, G.n_cols,
                                   str(tmp_path), **OPTS)
    assert (first.cache_hit, again.cache_hit) == (False, True)
    assert again.info == built.info
    want = built.spmm(b)
    for p in (first, again):
        got = p.spmm(b)
        assert float((got - want).abs().max()) <= 1e-6 * float(want.abs().max())
