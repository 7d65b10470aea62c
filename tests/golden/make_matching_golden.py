"""Regenerates tests/golden/matching_stats.json: the 2:4 matching statistics
that the REFERENCE's matching extensions report for small seeded matrices.

The reference's matching_utils (TR-source/Block/block_matching_window_para_dr.cpp),
matching_utils_hash (block_matching_hash.cpp) and matching_utils_bucket
(block_matching_bucket.cpp) are compiled from their own sources into
oracle/_ref by ``make -C oracle ref`` and called through their own Python
bindings.  The matrices are regenerated from the seeded generators named in
each case (trspmm.graphs); the fixture stores the matrix's nnz and a
checksum of its indices so a changed generator is noticed.

Run from the repository root, where the reference tree is available:
    python tests/golden/make_matching_golden.py
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tr-spmm_b200"))

import oracle  # noqa: E402
from trspmm import graphs  # noqa: E402

GRAPHS = {
    "chung_lu_4096": lambda: graphs.chung_lu(n=4096),
    "route_mix_2048": lambda: graphs.route_mix(n=2048, target_nnz=120_000),
    "sbm_6000": lambda: graphs.sbm_powerlaw(n=6000, avg_degree=30, communities=60, seed=4),
    "ragged_500x300": lambda: graphs.random_csr(500, 300, 0.05, seed=2, empty_rows=0.4),
    "dup_300x200": lambda: graphs.random_csr(300, 200, 0.08, seed=7, dup=True),
}
# (graph, variant, keyword arguments of the reference function)
CASES = [(g, v, {"window_size": w}) for g in GRAPHS for v in ("sliding", "hash", "bucket")
         for w in (16, 8)]
CASES += [("chung_lu_4096", v, {"window_size": 32}) for v in ("sliding", "hash", "bucket")]
CASES += [("route_mix_2048", "sliding", {"window_size": 16, "dense_threshold": 4, "t_max": 2}),
          ("sbm_6000", "sliding", {"window_size": 16, "dense_threshold": 16, "t_max": 0})]
REF = {"sliding": ("matching_utils", "match_2to4"),
       "hash": ("matching_utils_hash", "match_2to4_hash"),
       "bucket": ("matching_utils_bucket", "match_2to4_bucket")}


def checksum(g):
    return int(np.bitwise_xor.reduce((g.indices.astype(np.int64) * 2654435761
                                      + np.arange(g.nnz)) & 0xFFFFFFFF)) if g.nnz else 0


def main():
    built = {name: f() for name, f in GRAPHS.items()}
    out = {"graphs": {n: {"nnz": int(g.nnz), "rows": int(g.n_rows), "checksum": checksum(g)}
                      for n, g in built.items()},
           "cases": []}
    for gname, variant, kw in CASES:
        g = built[gname]
        mod, fn = REF[variant]
        res = oracle.ref_match(mod, fn, g.indptr, g.indices, g.values, **kw)
        out["cases"].append({"graph": gname, "variant": variant, "kwargs": kw, "expect": res})
    with open(os.path.join(HERE, "matching_stats.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
    print(f"{len(out['cases'])} cases")


if __name__ == "__main__":
    main()
