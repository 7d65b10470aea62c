"""The product router (libtrspmm, host C++) against the oracle and the
reference's golden tables: bit-exact in compat mode, lossless in exact mode,
with the reference's edge cases and error behaviour."""
import os

import numpy as np
import pytest
import scipy.sparse as sp
import torch

import oracle
import trspmm
from helpers import golden_files, half_csr, load_golden
from trspmm import graphs


def _same(a, b):
    bad = [n for n, x, y in zip(oracle.TABLE_NAMES[:29], a[:29], b[:29])
           if not (x.dtype == y.dtype and x.shape == y.shape and np.array_equal(x, y))]
    assert not bad, f"tables differ: {bad}"


@pytest.mark.parametrize("path", golden_files(), ids=lambda p: p.split("route_")[-1][:-4])
def test_router_matches_reference_golden(path):
    indptr, indices, values, n_cols, args, ref = load_golden(path)
    got = trspmm.route(indptr, indices, values, *args, unit_min_nnz=2, skip_tc=False)
    _same(got, ref)


CASES = [
    lambda: graphs.random_csr(1, 5, 0.6, seed=1),
    lambda: graphs.random_csr(17, 1, 0.9, seed=2),
    lambda: graphs.random_csr(300, 300, 0.1, seed=3, empty_rows=0.5),
    lambda: graphs.chung_lu(n=2000, avg_degree=12, seed=4),
    lambda: graphs.route_mix(n=2048, target_nnz=120_000, seed=5),
    lambda: graphs.sbm_powerlaw(n=4000, avg_degree=24, communities=40, seed=6),
    lambda: graphs.batched(num_graphs=12, seed=7),
]
PARAMS = [
    dict(),
    dict(density=4, tc_min_util=0.5),
    dict(partsize_t=3, partsize_c=5, shortsize=2),
    dict(density=1, partsize_t=1, partsize_c=1, shortsize=0),
    dict(window=8),
    dict(skip_tc=True),
    dict(unit_min_nnz=5),
]


@pytest.mark.parametrize("case", range(len(CASES)))
@pytest.mark.parametrize("prm", range(len(PARAMS)))
def test_router_matches_oracle(case, prm):
    g = CASES[case]()
    kw = dict(PARAMS[prm])
    kw.setdefault("unit_min_nnz", 2)
    kw.setdefault("skip_tc", False)
    window = kw.pop("window", 16)
    args = dict(partsize_t=kw.pop("partsize_t", 32), partsize_c=kw.pop("partsize_c", 32),
                shortsize=kw.pop("shortsize", 3), density=kw.pop("density", 8), window=window,
                tc_min_util=kw.pop("tc_min_util", 0.0))
    a = oracle.route(g.indptr, g.indices, g.values, **args, **kw)
    b = trspmm.route(g.indptr, g.indices, g.values, **args, **kw)
    _same(a, b)


@pytest.mark.parametrize("case", range(len(CASES)))
def test_exact_mode_is_lossless(case):
    g = CASES[case]()
    compat = trspmm.route(g.indptr, g.indices, g.values)
    exact = trspmm.route(g.indptr, g.indices, g.values, mode="exact")
    # same routing decisions: TC and SPTC tables unchanged (t_atomic may flip
    # to 1 where a window gains CUDA work from spilled entries)
    for i in [0, 1, 2, 3, 4, 6] + list(range(17, 29)):
        assert np.array_equal(compat[i], exact[i]), oracle.TABLE_NAMES[i]
    A = half_csr(g.indptr, g.indices, g.values, g.n_rows, g.n_cols)
    dec = oracle.decode_tables(exact, g.n_rows, g.n_cols)
    diff = (A - dec["all"])
    diff.eliminate_zeros()
    assert diff.nnz == 0
    assert dec["all"].nnz == A.nnz


def test_router_empty_matrix():
    indptr = np.zeros(1, dtype=np.int32)
    t = trspmm.route(indptr, np.zeros(0, np.int32), np.zeros(0, np.float32))
    o = oracle.route(indptr, np.zeros(0, np.int32), np.zeros(0, np.float32))
    _same(t, o)
    assert t[22].tolist() == [0]


def test_router_rows_without_entries():
    indptr = np.zeros(40, dtype=np.int32)
    t = trspmm.route(indptr, np.zeros(0, np.int32), np.zeros(0, np.float32))
    assert t[28].tolist() == [0, 0, 0, 0]       # 39 rows: three windows, no tiles


def test_router_threads_do_not_change_tables():
    g = graphs.sbm_powerlaw(n=6000, avg_degree=20, communities=60, seed=9)
    a = trspmm.route(g.indptr, g.indices, g.values, threads=1)
    b = trspmm.route(g.indptr, g.indices, g.values, threads=7)
    _same(a, b)


def test_router_duplicate_entries_follow_reference():
    # non-canonical CSR (a repeated column in a row): compat mode reproduces
    # the reference, exact mode keeps every entry
    indptr = np.array([0, 3, 5], dtype=np.int32)
    indices = np.array([2, 2, 7, 1, 1], dtype=np.int32)
    values = np.array([1.0, 2.0, 3.0, 4.0, 5.0], dtype=np.float32)
    a = oracle.route(indptr, indices, values, density=1)
    b = trspmm.route(indptr, indices, values, density=1)
    _same(a, b)


@pytest.mark.parametrize("bad", [
    dict(window=0), dict(window=33), dict(wide=0), dict(wide=40), dict(window=20)])
def test_router_rejects_bad_arguments(bad):
    g = graphs.random_csr(20, 20, 0.2)
    with pytest.raises(RuntimeError):
        trspmm.route(g.indptr, g.indices, g.values, **bad)


def test_router_rejects_malformed_csr():
    with pytest.raises(RuntimeError, match="non-decreasing"):
        trspmm.route(np.array([0, 3, 2], np.int32), np.zeros(3, np.int32), np.zeros(3, np.float32))
    with pytest.raises(RuntimeError, match=">= 0"):
        trspmm.route(np.array([0, 1], np.int32), np.array([-4], np.int32), np.ones(1, np.float32))


def test_env_switches(monkeypatch):
    g = graphs.route_mix(n=512, target_nnz=20_000)
    monkeypatch.setenv("LIBRA_SKIP_TC", "1")
    monkeypatch.setenv("LIBRA_SPTC_UNIT_MIN_NNZ", "3")
    a = trspmm.route(g.indptr, g.indices, g.values)
    b = oracle.route(g.indptr, g.indices, g.values, skip_tc=True, unit_min_nnz=3)
    _same(a, b)
    assert a[2].size == 0


def test_dropin_block_module_matches_reference_types():
    import Libra5BlockOnline
    g = graphs.chung_lu(n=256)
    out = Libra5BlockOnline.block_sptc_2to4_online(
        torch.from_numpy(g.indptr), torch.from_numpy(g.indices), torch.from_numpy(g.values),
        32, 32, 3, 8, 16, 16, 0.0, 0.5, 12)
    assert len(out) == 30
    ref = oracle.route(g.indptr, g.indices, g.values)
    for t, r, name in zip(out[:29], ref[:29], oracle.TABLE_NAMES):
        assert t.numpy().dtype == r.dtype and tuple(t.shape) == r.shape, name
        assert np.array_equal(t.numpy(), r), name
    assert out[29].dtype == torch.float32 and out[29].dim() == 0
    with pytest.raises(RuntimeError):
        Libra5BlockOnline.block_sptc_2to4_online(
            torch.from_numpy(g.indptr).long(), torch.from_numpy(g.indices),
            torch.from_numpy(g.values), 32, 32, 3, 8, 16, 16, 0.0, 0.5, 12)


@pytest.mark.skipif(not oracle.ref_available(), reason="reference router not compiled here")
def test_router_matches_compiled_reference_midsize():
    g = graphs.sbm_powerlaw(n=12_000, avg_degree=30, communities=120, seed=21)
    a = trspmm.route(g.indptr, g.indices, g.values)
    b = oracle.ref_route(g.indptr, g.indices, g.values, 32, 32, 3, 8, 16, 16, 0.0, 0.5, 12)
    _same(a, b)


@pytest.mark.skipif(not oracle.ref_available(), reason="reference router not compiled here")
def test_router_matches_compiled_reference_route_mix_full_size():
    """The route-mix stress matrix at its full size (65,536 rows, ~3.2M
    entries: dense 16x8 blocks on a band, 2:4-compatible rows, uniform
    scatter): all 29 tables bit for bit against the reference's router
    compiled from its own source."""
    g = graphs.route_mix(n=65_536, target_nnz=3_200_000, seed=3)
    assert g.nnz > 3_000_000
    a = trspmm.route(g.indptr, g.indices, g.values, mode="compat")
    b = oracle.ref_route(g.indptr, g.indices, g.values, 32, 32, 3, 8, 16, 16, 0.0, 0.5, 12)
    _same(a, b)
