"""ORACLE — test infrastructure only (see oracle/__init__.py).

CPU restatement of the reference's TCA row reorder,
spmm/tr_csr_fp16/tr_tca_reorder.py:44-357 (apply_tca_reorder), in plain
Python + numpy, written step for step after the reference:

  :84-99    MinHash of every row's column set, inserted into an LSH index
  :103-134  query every non-empty row, queue each new pair with its Jaccard
  :143-186  pop most similar first; merge roots (smaller into larger, a
            cluster of >= thres rows is closed); non-root pairs re-queue
            their roots with the Jaccard of the root rows' own sets
  :191-203  clusters in order of first appearance
  :208-297  the same over clusters (set = union of member sets, cap 128)
  :299-313  final order: groups, their clusters, each cluster's rows

The reference depends on datasketch (MinHash, MinHashLSH), which is not
installed here, and leaves two orders to its containers (query results come
out of a Python set; equal similarities leave a heap unordered).  This
restatement fixes them the way the library does (candidates ascending,
equal similarities first-queued first) and uses the library's MinHash hash
family (splitmix64-mixed column keys, multiply-add-shift permutations),
written independently here with numpy.  Parity is therefore pinned against
this restatement only: against the reference itself it is unpinned
(datasketch's SHA-1 hashing is absent, and the reference's own tie order is
not deterministic).
"""
from __future__ import annotations

import heapq
import itertools

import numpy as np

M64 = (1 << 64) - 1
GOLDEN = 0x9E3779B97F4A7C15
N_PERM = 128


def lsh_params(threshold, num_perm):
    """(bands, rows): b * r <= num_perm minimising 0.5 * false-positive +
    0.5 * false-negative probability integrals (MinHashLSH's documented
    criterion), integrated with scipy's adaptive quadrature."""
    from scipy.integrate import quad
    best = None
    for b in range(1, num_perm + 1):
        for r in range(1, num_perm // b + 1):
            fp = quad(lambda s: 1 - (1 - s ** r) ** b, 0.0, threshold)[0]
            fn = quad(lambda s: (1 - s ** r) ** b, threshold, 1.0)[0]
            e = 0.5 * fp + 0.5 * fn
            if best is None or e < best[0]:
                best = (e, b, r)
    return best[1], best[2]


def _mix64(z):
    """splitmix64 output function on a uint64 array (wrapping arithmetic)."""
    z = np.asarray(z, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


def _perm_coeffs(seed):
    i = np.arange(N_PERM, dtype=np.uint64)
    with np.errstate(over="ignore"):
        a = _mix64(np.uint64(seed) + np.uint64(GOLDEN) * (np.uint64(2) * i + np.uint64(1)))
        b = _mix64(np.uint64(seed) + np.uint64(GOLDEN) * (np.uint64(2) * i + np.uint64(2)))
    return a | np.uint64(1), b


def signatures(indptr, indices, seed=1):
    """uint32 [n, 128] MinHash signatures (empty rows: all 0xFFFFFFFF)."""
    n = len(indptr) - 1
    keys = (_mix64(np.asarray(indices, dtype=np.int64).astype(np.uint64) & np.uint64(0xFFFFFFFF))
            >> np.uint64(32))
    a, b = _perm_coeffs(seed)
    sig = np.full((n, N_PERM), 0xFFFFFFFF, dtype=np.uint64)
    starts = np.asarray(indptr[:-1], dtype=np.int64)
    live = np.flatnonzero(np.diff(np.asarray(indptr, dtype=np.int64)) > 0)
    if keys.size:
        for i in range(N_PERM):
            with np.errstate(over="ignore"):
                h = (a[i] * keys + b[i]) >> np.uint64(32)
            sig[live, i] = np.minimum.reduceat(h, starts[live])
    return sig.astype(np.uint32)


def band_digests(sig, bands, rows):
    """uint64 [n, bands]: the digest of each band of each signature."""
    n = sig.shape[0]
    out = np.empty((n, bands), dtype=np.uint64)
    v = sig.astype(np.uint64)
    with np.errstate(over="ignore"):
        for j in range(bands):
            d = np.full(n, _mix64(np.uint64(0x5BD1E9955BD1E995) + np.uint64(j)), dtype=np.uint64)
            for k in range(rows):
                d = _mix64(d ^ (v[:, j * rows + k] + np.uint64(GOLDEN)))
            out[:, j] = d
    return out


def _candidates(dig, live):
    """Per item, the sorted other items sharing a band digest (live items)."""
    cand = [set() for _ in range(dig.shape[0])]
    for j in range(dig.shape[1]):
        buckets = {}
        for i in live:
            buckets.setdefault(int(dig[i, j]), []).append(i)
        for members in buckets.values():
            for x in members:
                cand[x].update(members)
    return [sorted(c) for c in cand]


def _jaccard(s1, s2):
    if not s1 or not s2:
        return 0.0
    inter = len(s1 & s2)
    union = len(s1 | s2)
    return float(inter) / union if union > 0 else 0.0


def _cluster(sets, dig, cap):
    """Queue, pop and merge (tr_tca_reorder.py:103-186 / :235-297); returns
    the root of every item and the number of queued candidate pairs."""
    m = len(sets)
    live = [i for i in range(m) if sets[i]]
    cand = _candidates(dig, live)
    key = lambda x, y: (x, y) if x < y else (y, x)
    heap, queued, seq = [], set(), itertools.count()
    for i in live:
        for item in cand[i]:
            if item == i or key(i, item) in queued:
                continue
            heapq.heappush(heap, (-_jaccard(sets[i], sets[item]), next(seq), i, item))
            queued.add(key(i, item))
    n_pairs = len(queued)
    cid = list(range(m))
    sz = [1] * m
    deleted = [0] * m
    num = m

    def root(i):
        while i != cid[i]:
            cid[i] = cid[cid[i]]
            i = cid[i]
        return i

    while heap and num > 0:
        _, _, p1, p2 = heapq.heappop(heap)
        queued.discard(key(p1, p2))
        if p1 == cid[p1] and p2 == cid[p2]:
            if deleted[p1] or deleted[p2]:
                continue
            if sz[p1] < sz[p2]:
                cid[p1] = p2
                num -= 1
                sz[p2] += sz[p1]
                if sz[p2] >= cap:
                    deleted[p2] = 1
                    num -= 1
            else:
                cid[p2] = p1
                num -= 1
                sz[p1] += sz[p2]
                if sz[p1] >= cap:
                    deleted[p1] = 1
                    num -= 1
        else:
            r1, r2 = root(p1), root(p2)
            if deleted[r1] or deleted[r2]:
                continue
            if r1 != r2 and key(r1, r2) not in queued:
                heapq.heappush(heap, (-_jaccard(sets[r1], sets[r2]), next(seq), r1, r2))
                queued.add(key(r1, r2))
    return [root(i) for i in range(m)], n_pairs


def _groups(roots):
    """{root: members} in order of first appearance, members ascending."""
    out = {}
    for i, r in enumerate(roots):
        out.setdefault(r, []).append(i)
    return out


def tca_order(indptr, indices, n_rows=None, thres=16, cluster_thres=128, lsh_threshold=0.2,
              seed=1):
    """(order: new position -> old row, stats dict)."""
    indptr = np.asarray(indptr, dtype=np.int64)
    indices = np.asarray(indices, dtype=np.int64)
    n = len(indptr) - 1 if n_rows is None else int(n_rows)
    indptr = indptr[:n + 1]
    indices = indices[:indptr[-1]] if n > 0 else indices[:0]
    if n == 0:
        return np.zeros(0, dtype=np.int32), {}
    bands, rows = lsh_params(lsh_threshold, N_PERM)
    sets = [set(indices[indptr[i]:indptr[i + 1]].tolist()) for i in range(n)]
    sig = signatures(indptr, indices, seed)
    roots1, pairs1 = _cluster(sets, band_digests(sig, bands, rows), thres)
    clusters = _groups(roots1)
    keys = list(clusters)
    # level 2: each cluster's set is the union of its rows' sets, hashed
    # afresh (tr_tca_reorder.py:211-223)
    csets = [set().union(*(sets[r] for r in clusters[k])) for k in keys]
    cptr = np.concatenate([[0], np.cumsum([len(c) for c in csets])])
    ccol = np.asarray([c for cs in csets for c in sorted(cs)], dtype=np.int64)
    csig = signatures(cptr, ccol, seed)
    roots2, pairs2 = _cluster(csets, band_digests(csig, bands, rows), cluster_thres)
    groups = _groups(roots2)
    order = [row for g in groups.values() for c in g for row in clusters[keys[c]]]
    seen = set(order)
    order += [i for i in range(n) if i not in seen]
    stats = {"bands": bands, "rows_per_band": rows, "pairs1": pairs1, "clusters1": len(keys),
             "pairs2": pairs2, "clusters2": len(groups)}
    return np.asarray(order, dtype=np.int32), stats
