"""2:4 matching statistics (tr_match_2to4 and the drop-in modules
matching_utils, matching_utils_hash, matching_utils_bucket) against the
reference's own matching extensions: the golden fixture made from them
(tests/golden/matching_stats.json), and the compiled reference itself on
randomised matrices where oracle/_ref has been built.  CPU only."""
import json
import os

import numpy as np
import pytest

import oracle
import matching_utils
import matching_utils_bucket
import matching_utils_hash
import trspmm
from trspmm import graphs

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = json.load(open(os.path.join(HERE, "golden", "matching_stats.json")))
DROP_IN = {"sliding": matching_utils.match_2to4, "hash": matching_utils_hash.match_2to4_hash,
           "bucket": matching_utils_bucket.match_2to4_bucket}
REF = {"sliding": ("matching_utils", "match_2to4"),
       "hash": ("matching_utils_hash", "match_2to4_hash"),
       "bucket": ("matching_utils_bucket", "match_2to4_bucket")}
GRAPHS = {
    "chung_lu_4096": lambda: graphs.chung_lu(n=4096),
    "route_mix_2048": lambda: graphs.route_mix(n=2048, target_nnz=120_000),
    "sbm_6000": lambda: graphs.sbm_powerlaw(n=6000, avg_degree=30, communities=60, seed=4),
    "ragged_500x300": lambda: graphs.random_csr(500, 300, 0.05, seed=2, empty_rows=0.4),
    "dup_300x200": lambda: graphs.random_csr(300, 200, 0.08, seed=7, dup=True),
}
_built = {}


def _graph(name):
    if name not in _built:
        _built[name] = GRAPHS[name]()
    return _built[name]


def _checksum(g):
    return int(np.bitwise_xor.reduce((g.indices.astype(np.int64) * 2654435761
                                      + np.arange(g.nnz)) & 0xFFFFFFFF)) if g.nnz else 0


def _same(got, want):
    for k, v in want.items():
        assert k in got, k
        if isinstance(v, float):
            assert got[k] == pytest.approx(v, rel=1e-12), k
        else:
            assert got[k] == v, k


@pytest.mark.parametrize("name", list(GRAPHS))
def test_fixture_graphs_unchanged(name):
    g = _graph(name)
    meta = GOLDEN["graphs"][name]
    assert (g.nnz, g.n_rows, _checksum(g)) == (meta["nnz"], meta["rows"], meta["checksum"])


@pytest.mark.parametrize("case", GOLDEN["cases"],
                         ids=lambda c: f"{c['graph']}-{c['variant']}-" +
                         "-".join(f"{k}{v}" for k, v in c["kwargs"].items()))
def test_drop_in_matches_reference_golden(case):
    g = _graph(case["graph"])
    got = DROP_IN[case["variant"]](g.indptr, g.indices, g.values, **case["kwargs"])
    _same(got, case["expect"])


@pytest.mark.skipif(not oracle.ref_match_available("matching_utils_bucket"),
                    reason="reference matching modules not compiled here")
@pytest.mark.parametrize("seed", range(8))
@pytest.mark.parametrize("variant", ["sliding", "hash", "bucket"])
def test_matches_compiled_reference(variant, seed):
    rng = np.random.default_rng(100 + seed)
    n = int(rng.integers(17, 900))
    g = graphs.random_csr(n, int(rng.integers(5, 600)), float(rng.uniform(0.002, 0.3)), seed=seed,
                          empty_rows=float(rng.uniform(0, 0.4)), dup=bool(seed % 2))
    kw = {"window_size": int(rng.choice([1, 3, 8, 16, 20, 64]))}
    if variant == "sliding":
        kw.update(dense_threshold=int(rng.integers(1, 12)), t_max=int(rng.integers(0, 16)))
    mod, fn = REF[variant]
    want = oracle.ref_match(mod, fn, g.indptr, g.indices, g.values, **kw)
    _same(DROP_IN[variant](g.indptr, g.indices, g.values, **kw), want)


def test_keys_of_every_variant():
    """Each variant's dict carries its reference keys and the other variants'
    names for the same counters (the reference's comparison script mixes them)."""
    g = _graph("chung_lu_4096")
    for v, fn in DROP_IN.items():
        d = fn(g.indptr, g.indices, g.values)
        for k in ("total_rows", "total_cols", "total_nnz", "sparsity", "num_row_panels",
                  "num_groups", "num_sptc_groups", "num_tc_blocks", "num_16x16_blocks",
                  "block_padding_groups", "fine_fallback", "coarse_fallback", "fake_zeros"):
            assert k in d, (v, k)
        assert d["block_padding_groups"] == d["num_16x16_blocks"] * 4 - d["num_groups"]
        if v != "sliding":
            assert d["num_tc_blocks"] == 0


def test_rejects_bad_arguments():
    g = _graph("ragged_500x300")
    for ws in (0, 65):
        with pytest.raises(trspmm.TrError, match="window_size"):
            matching_utils.match_2to4(g.indptr, g.indices, g.values, window_size=ws)
    with pytest.raises(trspmm.TrError, match="dense_threshold"):
        matching_utils.match_2to4(g.indptr, g.indices, g.values, dense_threshold=0)
    with pytest.raises(trspmm.TrError, match="empty matrix"):
        matching_utils_hash.match_2to4_hash(np.zeros(5, np.int32), np.zeros(0, np.int32),
                                            np.zeros(0, np.float32))


@pytest.mark.parametrize("name", ["chung_lu_4096", "route_mix_2048", "sbm_6000", "dup_300x200"])
def test_online_rules_are_the_sliding_decisions(name):
    """The online variant (host restatement) takes the sliding variant's
    decisions; only the group size behind fake_zeros differs (32 slots,
    against 2 x window rows), which shows in windows of fewer than 16 rows."""
    g = _graph(name)
    a = trspmm.match_2to4(g.indptr, g.indices, "sliding", 16)
    b = trspmm.match_2to4(g.indptr, g.indices, "online", 16)
    for k in a:
        if k != "fake_zeros":
            assert a[k] == b[k], k
    if g.n_rows % 16 == 0:
        assert a["fake_zeros"] == b["fake_zeros"]
    assert b["dense_to_tc_cols"] == b["num_tc_blocks"] * 8
    with pytest.raises(trspmm.TrError, match="16-row windows"):
        trspmm.match_2to4(g.indptr, g.indices, "online", 8)
