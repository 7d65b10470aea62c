"""Regenerates the golden route-table fixtures in this directory.

Each fixture holds a small seeded CSR matrix and the 29 route tables that the
REFERENCE router produced for it: TR-source/Block/block_online.cpp compiled
from its own source into oracle/_ref by ``make -C oracle ref`` and called
through its own Python binding (``Libra5BlockOnline.block_sptc_2to4_online``).
The reference ships no golden vectors of its own, so these pin both the CPU
oracle and this library's router to the reference's actual behaviour.

Run from the repository root, where the reference tree is available:
    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tr-spmm_b200"))

import oracle  # noqa: E402
from trspmm import graphs  # noqa: E402

# (name, generator, router arguments: partsize_t, partsize_c, shortsize, density,
#  window, wide, tc_min_util, sptc_min_util, sptc_threshold)
DEFAULT = (32, 32, 3, 8, 16, 16, 0.0, 0.5, 12)
CASES = [
    ("random_64x80", lambda: graphs.random_csr(64, 80, 0.3, seed=1), DEFAULT),
    ("random_ragged", lambda: graphs.random_csr(203, 170, 0.05, seed=4, empty_rows=0.2), DEFAULT),
    ("chung_lu_512", lambda: graphs.chung_lu(n=512, avg_degree=16, seed=11), DEFAULT),
    ("route_mix_1024", lambda: graphs.route_mix(n=1024, target_nnz=50_000, seed=12), DEFAULT),
    ("route_mix_1024_d4", lambda: graphs.route_mix(n=1024, target_nnz=50_000, seed=12),
     (4, 8, 2, 4, 16, 16, 0.25, 0.5, 12)),
    ("sbm_2048", lambda: graphs.sbm_powerlaw(n=2048, avg_degree=20, communities=20, seed=13),
     DEFAULT),
    ("dense_band_256", lambda: graphs.route_mix(n=256, target_nnz=20_000, frac_dense=0.9,
                                                frac_24=0.05, seed=14), DEFAULT),
    ("window8", lambda: graphs.random_csr(100, 64, 0.2, seed=15),
     (32, 32, 3, 4, 8, 16, 0.0, 0.5, 12)),
]


def main():
    if not oracle.ref_available():
        raise SystemExit("oracle/_ref is not built (make -C oracle ref)")
    for name, gen, args in CASES:
        g = gen()
        tabs = oracle.ref_route(g.indptr, g.indices, g.values, *args)
        arrays = {"indptr": g.indptr, "indices": g.indices, "values": g.values,
                  "n_cols": np.int64(g.n_cols), "args": np.array(args, dtype=np.float64)}
        for tname, t in zip(oracle.TABLE_NAMES[:29], tabs[:29]):
            arrays[tname] = t
        np.savez_compressed(os.path.join(HERE, f"route_{name}.npz"), **arrays)
        print(name, g.n_rows, g.nnz)


if __name__ == "__main__":
    main()
