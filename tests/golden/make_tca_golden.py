"""Makes tests/golden/tca_orders.json: row orders of the reference's own TCA
reorder (spmm/tr_csr_fp16/tr_tca_reorder.py, apply_tca_reorder) on seeded
synthetic graphs.

The reference imports datasketch, which is not installed here.  This script
runs the reference's unmodified function with two stand-ins, so that its
result is defined and reproducible:
  * a ``datasketch`` module whose MinHash / MinHashLSH hash with the library's
    hash family (128 permutations; LSH bands from the same false-positive /
    false-negative criterion) and whose query returns keys in ascending order;
  * ``queue.PriorityQueue`` with first-queued-first ties among equal
    similarities (the reference's Pair orders by similarity only).
Everything else -- candidate queueing, Jaccard, both clustering levels, the
final order, the rebuilt column array -- is the reference's code.  The
reference's rebuilt row pointers are recorded only by their last value: its
loop leaves every row empty (row_ptr all zeros), a defect the library does
not reproduce.  Run from the repository root with the reference checkout's
root directory as the argument (or in TR_REFERENCE_ROOT):
    python tests/golden/make_tca_golden.py <reference root>
"""
import contextlib
import hashlib
import heapq
import importlib.util
import io
import itertools
import json
import os
import queue
import re
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tr-spmm_b200"))
from oracle import tca as otca           # noqa: E402  (hash family of the stand-in)
from trspmm import graphs                # noqa: E402

REF_FILE = os.path.join("spmm", "tr_csr_fp16", "tr_tca_reorder.py")


class _MinHash:
    def __init__(self, num_perm=128):
        assert num_perm == otca.N_PERM
        self.cols, self.sig = [], None

    def update(self, b):
        self.cols.append(int(b.decode("utf-8")))
        self.sig = None

    def signature(self):
        if self.sig is None:
            c = np.asarray(self.cols, dtype=np.int64)
            self.sig = otca.signatures(np.asarray([0, c.size]), c)[0]
        return self.sig


class _MinHashLSH:
    _params = {}

    def __init__(self, threshold=0.9, num_perm=128):
        if (threshold, num_perm) not in self._params:
            self._params[(threshold, num_perm)] = otca.lsh_params(threshold, num_perm)
        self.b, self.r = self._params[(threshold, num_perm)]
        self.tables = [dict() for _ in range(self.b)]

    def _digests(self, m):
        return otca.band_digests(m.signature()[None, :], self.b, self.r)[0]

    def insert(self, key, m):
        for t, d in zip(self.tables, self._digests(m)):
            t.setdefault(int(d), []).append(key)

    def query(self, m):
        out = set()
        for t, d in zip(self.tables, self._digests(m)):
            out.update(t.get(int(d), []))
        return sorted(out, key=int)


class _StablePQ:
    """queue.PriorityQueue with ties (neither item less) popped in put order."""

    class _E:
        __slots__ = ("item", "seq")

        def __init__(self, item, seq):
            self.item, self.seq = item, seq

        def __lt__(self, other):
            if self.item < other.item:
                return True
            if other.item < self.item:
                return False
            return self.seq < other.seq

    def __init__(self):
        self.h, self.c = [], itertools.count()

    def put(self, item):
        heapq.heappush(self.h, self._E(item, next(self.c)))

    def get(self):
        return heapq.heappop(self.h).item

    def empty(self):
        return not self.h

    def qsize(self):
        return len(self.h)


CASES = {
    "chung_lu_2048": lambda: graphs.chung_lu(n=2048),
    "route_mix_1024": lambda: graphs.route_mix(n=1024, target_nnz=50_000),
    "sbm_3000": lambda: graphs.sbm_powerlaw(n=3000, avg_degree=20, communities=30, seed=4),
    "ragged_500x300": lambda: graphs.random_csr(500, 300, 0.05, seed=2, empty_rows=0.4),
    "dup_300x200": lambda: graphs.random_csr(300, 200, 0.08, seed=7, dup=True),
    "batched_24": lambda: graphs.batched(num_graphs=24, seed=11),
    "rect_400x900": lambda: graphs.random_csr(400, 900, 0.02, seed=13, empty_rows=0.1),
}


def checksum(g):
    return int(np.bitwise_xor.reduce((g.indices.astype(np.int64) * 2654435761
                                      + np.arange(g.nnz)) & 0xFFFFFFFF)) if g.nnz else 0


def main():
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("TR_REFERENCE_ROOT")
    if not root:
        sys.exit("usage: make_tca_golden.py <reference root> (or set TR_REFERENCE_ROOT)")
    ref = os.path.join(root, REF_FILE)
    sys.modules["datasketch"] = types.SimpleNamespace(MinHash=_MinHash, MinHashLSH=_MinHashLSH)
    queue.PriorityQueue = _StablePQ
    spec = importlib.util.spec_from_file_location("tr_tca_reorder_ref", ref)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    out = {"source": "spmm/tr_csr_fp16/tr_tca_reorder.py apply_tca_reorder(thres=16)",
           "cases": {}}
    for name, make in CASES.items():
        g = make()
        log = io.StringIO()
        with contextlib.redirect_stdout(log):
            ptr, idx, order = mod.apply_tca_reorder(g.indptr.astype(np.int32),
                                                   g.indices.astype(np.int32), g.n_rows,
                                                   thres=16, verbose=True)
        text = log.getvalue()
        order = np.asarray(order, dtype=np.int32)
        out["cases"][name] = {
            "rows": g.n_rows, "nnz": g.nnz, "checksum": checksum(g),
            "order_sha256": hashlib.sha256(order.tobytes()).hexdigest(),
            "order_head": order[:32].tolist(),
            # the reference's new_col_ind; its new_row_ptr is not usable: the
            # rebuild loop (tr_tca_reorder.py:342-350) overwrites each row's
            # end pointer with its start when it moves to the next row
            "col_ind_sha256": hashlib.sha256(np.asarray(idx, np.int32).tobytes()).hexdigest(),
            "ref_row_ptr_last": int(np.asarray(ptr)[-1]),
            "pairs1": int(re.search(r"LSH query \+ Jaccard time = .*queue size = (\d+)", text)[1]),
            "clusters1": int(re.search(r"row-level clusters = (\d+)", text)[1]),
            "pairs2": int(re.search(r"cluster-level queue size = (\d+)", text)[1]),
        }
        print(name, out["cases"][name]["pairs1"], out["cases"][name]["clusters1"])
    with open(os.path.join(HERE, "tca_orders.json"), "w") as f:
        json.dump(out, f, indent=1)
        f.write("\n")


if __name__ == "__main__":
    main()
