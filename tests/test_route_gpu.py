"""The router's dense-TC funnel on the GPU against the CPU router (exact
mode): t_row_offset, t_block_offset, t_column, t_value, t_window_row and
t_binary bit for bit, on the golden fixtures' matrices, power-law and
community graphs, windows larger than the kernel's shared-memory capacity
(hub rows), parameter sweeps and empty inputs."""
import numpy as np
import pytest
import scipy.sparse as sp
import torch

import trspmm
from helpers import golden_files, load_golden
from trspmm import graphs

pytestmark = pytest.mark.gpu

NAMES = ["t_row_offset", "t_block_offset", "t_column", "t_value", "t_window_row", "t_binary"]


def _canonical(indptr, indices, values, n_rows, n_cols):
    A = sp.csr_matrix((np.asarray(values, np.float32), indices, indptr), shape=(n_rows, n_cols))
    A.sum_duplicates()
    A.sort_indices()
    return A.indptr.astype(np.int32), A.indices.astype(np.int32), A.data.astype(np.float32)


def _compare(ip, ix, vv, n_rows, cuda, **kw):
    ref = trspmm.route(ip, ix, vv, mode="exact", unit_min_nnz=2,
                       skip_tc=kw.get("skip_tc", False),
                       **{k: v for k, v in kw.items() if k != "skip_tc"})
    got = trspmm.route_tc_device(torch.from_numpy(ip).to(cuda), torch.from_numpy(ix).to(cuda),
                                 torch.from_numpy(vv).to(cuda), n_rows, **kw)
    for name in NAMES:
        want = ref[trspmm.TABLE_NAMES.index(name)]
        assert got[name].dtype == want.dtype, name
        assert np.array_equal(got[name], want), name


@pytest.mark.parametrize("path", golden_files(), ids=lambda p: p.split("route_")[-1][:-4])
def test_golden_matrices(cuda, path):
    indptr, indices, values, n_cols, args, _ = load_golden(path)
    n_rows = len(indptr) - 1
    ip, ix, vv = _canonical(indptr, indices, values, n_rows, n_cols)
    _compare(ip, ix, vv, n_rows, cuda)


CASES = {
    "chung_lu": lambda: graphs.chung_lu(n=4096),
    "sbm": lambda: graphs.sbm_powerlaw(n=6000, avg_degree=30, communities=60, seed=4),
    "route_mix": lambda: graphs.route_mix(n=2048, target_nnz=120_000),
    "batched": lambda: graphs.batched(num_graphs=30, seed=3),
    "ragged": lambda: graphs.random_csr(500, 300, 0.05, seed=2, empty_rows=0.4),
}


@pytest.mark.parametrize("name", list(CASES))
@pytest.mark.parametrize("kw", [dict(), dict(density=4), dict(density=2, tc_min_util=0.3),
                                dict(partsize_t=3), dict(skip_tc=True)],
                         ids=["default", "d4", "d2u03", "pt3", "skip"])
def test_graphs(cuda, name, kw):
    g = CASES[name]()
    _compare(g.indptr, g.indices, np.asarray(g.values, np.float32), g.n_rows, cuda, **kw)


def test_hub_windows_beyond_shared_memory(cuda):
    """Rows with thousands of entries: windows whose keys do not fit the
    kernel's shared memory run on the global scratch path."""
    rng = np.random.default_rng(5)
    n, n_cols = 64, 20000
    rows, cols = [], []
    for r in range(n):
        deg = 3000 if r in (3, 17, 40) else int(rng.integers(1, 40))
        c = rng.choice(n_cols // 4 if r < 32 else n_cols, size=deg, replace=False)
        rows.append(np.full(deg, r))
        cols.append(c)
    # a dense band of shared columns so TC groups exist in the hub windows
    for r in range(16):
        rows.append(np.full(40, r))
        cols.append(np.arange(100, 140))
    A = sp.coo_matrix((rng.uniform(-1, 1, sum(len(x) for x in rows)).astype(np.float32),
                       (np.concatenate(rows), np.concatenate(cols))), shape=(n, n_cols)).tocsr()
    ip, ix, vv = _canonical(A.indptr, A.indices, A.data, n, n_cols)
    assert np.diff(ip)[3] > 2048
    _compare(ip, ix, vv, n, cuda)
    _compare(ip, ix, vv, n, cuda, density=2)


def test_empty(cuda):
    ip = np.zeros(33, np.int32)
    got = trspmm.route_tc_device(torch.from_numpy(ip).to(cuda), torch.zeros(0, dtype=torch.int32, device=cuda),
                                 torch.zeros(0, dtype=torch.float32, device=cuda), 32)
    assert got["t_column"].size == 0 and np.array_equal(got["t_row_offset"], [0])
