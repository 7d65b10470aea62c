"""trspmm.datasets.load_matrix over every file format the reference's scripts
read: scipy .npz, src_li / dst_li edge lists (with 'shape' and optional
'data', or with num_nodes_src / num_nodes_dst), MatrixMarket coordinate
(real and pattern) and array files.  CPU only."""
import numpy as np
import pytest
import scipy.io
import scipy.sparse as sp

from trspmm.datasets import load_matrix

RNG = np.random.default_rng(3)
ROWS = RNG.integers(0, 40, 300)
COLS = RNG.integers(0, 25, 300)
VALS = RNG.uniform(-1, 1, 300).astype(np.float32)
WANT = sp.coo_matrix((VALS, (ROWS, COLS)), shape=(40, 25)).tocsr()
WANT.sum_duplicates()
WANT.sort_indices()


def _check(m, want=WANT, ones=False):
    assert (m.n_rows, m.n_cols) == want.shape
    assert m.indptr.dtype == np.int32 and m.indices.dtype == np.int32 and m.values.dtype == np.float32
    assert np.array_equal(m.indptr, want.indptr) and np.array_equal(m.indices, want.indices)
    if ones:
        assert np.all(m.values == 1)
    else:
        assert np.allclose(m.values, want.data.astype(np.float32), rtol=1e-6, atol=1e-7)
    for r in range(m.n_rows):                       # columns sorted within rows
        assert np.all(np.diff(m.indices[m.indptr[r]:m.indptr[r + 1]]) > 0)


def test_scipy_npz(tmp_path):
    p = tmp_path / "a.npz"
    sp.save_npz(p, WANT)
    _check(load_matrix(str(p)))


def test_edge_list_with_shape_and_data(tmp_path):
    p = tmp_path / "b.npz"
    np.savez(p, src_li=ROWS, dst_li=COLS, data=VALS, shape=np.array([40, 25]))
    _check(load_matrix(str(p)))


def test_edge_list_without_data_is_ones(tmp_path):
    p = tmp_path / "c.npz"
    np.savez(p, src_li=ROWS, dst_li=COLS, shape=np.array([40, 25]))
    want = sp.coo_matrix((np.ones(300, np.float32), (ROWS, COLS)), shape=(40, 25)).tocsr()
    want.sum_duplicates()
    want.sort_indices()
    _check(load_matrix(str(p)), want)


def test_edge_list_with_node_counts(tmp_path):
    p = tmp_path / "d.npz"
    np.savez(p, src_li=ROWS, dst_li=COLS, num_nodes_src=40, num_nodes_dst=25)
    m = load_matrix(str(p))
    assert (m.n_rows, m.n_cols) == (40, 25) and np.array_equal(m.indices, WANT.indices)


def test_matrix_market_real_pattern_and_array(tmp_path):
    p = tmp_path / "e.mtx"
    scipy.io.mmwrite(str(p), WANT)
    _check(load_matrix(str(p)))
    q = tmp_path / "f.mtx"
    scipy.io.mmwrite(str(q), WANT, field="pattern")
    _check(load_matrix(str(q)), ones=True)
    dense = WANT.toarray()
    r = tmp_path / "g.mtx"
    scipy.io.mmwrite(str(r), dense)
    _check(load_matrix(str(r)))


def test_bad_files(tmp_path):
    p = tmp_path / "h.npz"
    np.savez(p, foo=np.arange(3))
    with pytest.raises(ValueError, match="edge list"):
        load_matrix(str(p))
    q = tmp_path / "i.npz"
    np.savez(q, src_li=np.array([0, 50]), dst_li=np.array([0, 1]), shape=np.array([40, 25]))
    with pytest.raises(ValueError, match="outside"):
        load_matrix(str(q))
    with pytest.raises(ValueError, match="unsupported"):
        load_matrix(str(tmp_path / "j.csv"))
