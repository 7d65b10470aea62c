"""The GPU online matcher (tr_match_2to4_online, drop-in
matching_utils_online.match_2to4_online) against the host restatement of the
same rules (tr_match_2to4 with TR_MATCH_ONLINE): every counter equal, on
graphs with windows past the kernel's 2048-entry capacity (counted on the
host), ragged and duplicated entries, and the parameter corners (t_max
negative, zero and past 16; dense_threshold 1 and large)."""
import numpy as np
import pytest

import matching_utils_online
import trspmm
from trspmm import graphs

pytestmark = pytest.mark.gpu


def _hubs():
    rng = np.random.default_rng(11)
    rows, cols = [], []
    for r in range(64):
        deg = 3000 if r in (2, 20) else int(rng.integers(1, 60))
        rows.append(np.full(deg, r))
        cols.append(rng.choice(20000, size=deg, replace=False))
    import scipy.sparse as sp
    A = sp.coo_matrix((np.ones(sum(len(c) for c in cols), np.float32),
                       (np.concatenate(rows), np.concatenate(cols))), shape=(64, 20000)).tocsr()
    A.sort_indices()
    return graphs.Graph(A.indptr.astype(np.int32), A.indices.astype(np.int32),
                        A.data.astype(np.float32), 64, 20000)


CASES = {
    "chung_lu": lambda: graphs.chung_lu(n=4096),
    "route_mix": lambda: graphs.route_mix(n=2048, target_nnz=120_000),
    "sbm": lambda: graphs.sbm_powerlaw(n=6000, avg_degree=30, communities=60, seed=4),
    "ragged": lambda: graphs.random_csr(500, 300, 0.05, seed=2, empty_rows=0.4),
    "dup": lambda: graphs.random_csr(300, 200, 0.08, seed=7, dup=True),
    "hubs": _hubs,
}


@pytest.mark.parametrize("name", list(CASES))
@pytest.mark.parametrize("dt,tm", [(8, 8), (1, 0), (4, -1), (32, 20)])
def test_gpu_equals_host_rules(cuda, name, dt, tm):
    g = CASES[name]()
    want = trspmm.match_2to4(g.indptr, g.indices, "online", 16, dt, tm)
    got = trspmm.core.match_2to4_online(g.indptr, g.indices, 16, dt, tm)
    assert got == want


def test_drop_in_keys(cuda):
    g = CASES["chung_lu"]()
    d = matching_utils_online.match_2to4_online(g.indptr, g.indices, g.values)
    for k in ("total_rows", "total_cols", "total_nnz", "num_sptc_groups", "num_tc_blocks",
              "dense_to_tc_cols", "dense_to_sptc_cols", "fine_fb", "coarse_fb_cols",
              "num_16x16_blocks", "block_padding_groups", "fake_zeros"):
        assert k in d, k
    assert d["block_padding_groups"] == d["num_16x16_blocks"] * 4 - d["num_sptc_groups"]
    with pytest.raises(trspmm.TrError, match="16-row windows"):
        matching_utils_online.match_2to4_online(g.indptr, g.indices, g.values, window_size=8)
