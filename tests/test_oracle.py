"""The oracle, pinned: its restated router against the reference's own tables
(golden fixtures made by the reference router, and the compiled reference
itself where available); its table decoder and FP64 arithmetic against scipy."""
import numpy as np
import pytest
import scipy.sparse as sp

import oracle
import trspmm
from helpers import golden_files, half_csr, load_golden, rel_err
from trspmm import graphs


@pytest.mark.parametrize("path", golden_files(), ids=lambda p: p.split("route_")[-1][:-4])
def test_oracle_router_matches_reference_golden(path):
    indptr, indices, values, n_cols, args, ref = load_golden(path)
    got = oracle.route(indptr, indices, values, *args, unit_min_nnz=2, skip_tc=False)
    for name, a, b in zip(oracle.TABLE_NAMES, got[:29], ref):
        assert a.dtype == b.dtype, name
        assert a.shape == b.shape, name
        assert np.array_equal(a, b), name


@pytest.mark.skipif(not oracle.ref_available(), reason="reference router not compiled here")
@pytest.mark.parametrize("seed", range(6))
def test_oracle_router_matches_compiled_reference(seed):
    rng = np.random.default_rng(seed)
    n = int(rng.integers(20, 600))
    g = graphs.random_csr(n, int(rng.integers(10, 700)), float(rng.uniform(0.005, 0.2)), seed=seed,
                          empty_rows=float(rng.uniform(0, 0.3)))
    args = (int(rng.integers(1, 40)), int(rng.integers(1, 40)), int(rng.integers(0, 5)),
            int(rng.integers(1, 12)), 16, 16, float(rng.choice([0.0, 0.3, 0.6])), 0.5, 12)
    a = oracle.route(g.indptr, g.indices, g.values, *args, unit_min_nnz=2, skip_tc=False)
    b = oracle.ref_route(g.indptr, g.indices, g.values, *args)
    for name, x, y in zip(oracle.TABLE_NAMES[:29], a, b):
        assert np.array_equal(x, y), name


@pytest.mark.parametrize("path", golden_files(), ids=lambda p: p.split("route_")[-1][:-4])
def test_decoded_tables_are_a_minus_truncation(path):
    """What the tables encode is A without the SPTC entries beyond two per row
    and group; every other entry keeps its FP16 value."""
    indptr, indices, values, n_cols, args, ref = load_golden(path)
    n_rows = len(indptr) - 1
    window = args[4]
    if window != 16:
        pytest.skip("reference row codes assume 16-row windows")
    A = half_csr(indptr, indices, values, n_rows, n_cols)
    dec = oracle.decode_tables(ref, n_rows, n_cols, window)
    diff = (A - dec["all"]).tocoo()
    diff.eliminate_zeros()
    # every missing entry is an SPTC-group column, and nothing extra appears
    assert np.all(np.isclose(diff.data, A[diff.row, diff.col].A1))
    # the packed tiles decode to the same SPTC matrix as s_value/s_pos
    dec2 = oracle.decode_tables(ref, n_rows, n_cols, window, sptc_from="tiles")
    assert abs(dec["sptc"] - dec2["sptc"]).max() == 0


def test_spmm_f64_matches_scipy():
    g = graphs.chung_lu(n=700)
    b = graphs.dense_features(g.n_cols, 24)
    A = half_csr(g.indptr, g.indices, g.values, g.n_rows, g.n_cols)
    ref = A @ b.astype(np.float64)
    got = oracle.spmm_f64(g.indptr, g.indices, A.data, b.astype(np.float64))
    assert rel_err(got, ref) < 1e-13


def test_spmm_f16_f32_close_to_f64():
    g = graphs.sbm_powerlaw(n=3000, avg_degree=20, communities=30)
    b = graphs.dense_features(g.n_cols, 64, "normal")
    A = half_csr(g.indptr, g.indices, g.values, g.n_rows, g.n_cols)
    ref = A @ b.astype(np.float64)
    got = oracle.spmm_f16_f32(g.indptr, g.indices, g.values.astype(np.float16), b, threads=2)
    assert rel_err(got, ref) < 1e-5


def test_sddmm_f64():
    g = graphs.random_csr(50, 40, 0.2, seed=3)
    rng = np.random.default_rng(0)
    dc = rng.standard_normal((50, 8))
    b = rng.standard_normal((40, 8))
    got = oracle.sddmm_f64(g.indptr, g.indices, dc, b)
    rows = g.row_ids()
    ref = np.einsum("ij,ij->i", dc[rows], b[g.indices])
    assert np.allclose(got, ref)


def test_oracle_rejects_bad_window():
    g = graphs.random_csr(10, 10, 0.3)
    with pytest.raises(ValueError):
        oracle.route(g.indptr, g.indices, g.values, 32, 32, 3, 8, 17)


def test_reference_sptc_host_checks():
    """The one index the reference's scalar 2:4 kernel does not check
    (s_pos into a group's four columns) is refused on the host before the
    call (tests/test_reference_operator_gpu.py runs the kernel)."""
    g = graphs.random_csr(33, 50, 0.1, seed=2)
    T = dict(zip(trspmm.TABLE_NAMES, trspmm.route(g.indptr, g.indices, g.values)))
    bad = T["s_pos"].copy()
    bad.flat[0] = 4
    with pytest.raises(ValueError, match="-1..3"):
        oracle.check_sptc_tables(T["s_column"], T["s_value"], bad, T["s_window"], 16, 8,
                                 g.n_rows, g.n_cols)
    with pytest.raises(ValueError, match="shapes"):
        oracle.check_sptc_tables(T["s_column"][:-1], T["s_value"], T["s_pos"], T["s_window"], 16,
                                 8, g.n_rows, g.n_cols)


def test_reference_cuda_route_host_checks():
    """The conditions under which the reference's parallel operator runs its
    CUDA-route kernels alone and inside their buffers are refused on the
    host when broken (tests/test_reference_operator_gpu.py runs it)."""
    g = graphs.random_csr(200, 150, 0.05, seed=3)
    T = dict(zip(trspmm.TABLE_NAMES, trspmm.route(g.indptr, g.indices, g.values,
                                                  skip_tc=True, skip_sptc=True)))
    oracle.check_cuda_route_tables(T, 128, g.n_rows, g.n_cols, 32)
    with pytest.raises(ValueError, match="128 features"):
        oracle.check_cuda_route_tables(T, 64, g.n_rows, g.n_cols, 32)
    for name, edit, msg in (("c_row", lambda a: a.__setitem__(0, -1), "negative"),
                            ("c_column", lambda a: a.__setitem__(0, g.n_cols), "kOri")):
        bad = dict(T)
        bad[name] = T[name].copy()
        edit(bad[name])
        with pytest.raises(ValueError, match=msg):
            oracle.check_cuda_route_tables(bad, 128, g.n_rows, g.n_cols, 32)
    with pytest.raises(ValueError, match="partsize_c"):
        oracle.check_cuda_route_tables(T, 128, g.n_rows, g.n_cols, 8)
    full = dict(zip(trspmm.TABLE_NAMES, trspmm.route(g.indptr, g.indices, g.values)))
    if full["t_atomic"].size or full["s_column"].size:
        with pytest.raises(ValueError, match="CUDA-route parts only"):
            oracle.check_cuda_route_tables(full, 128, g.n_rows, g.n_cols, 32)
