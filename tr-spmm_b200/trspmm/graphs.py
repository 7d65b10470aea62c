"""Seeded synthetic sparse operands for the routed SpMM workloads.

The reference ships no datasets (its loader reads ``<name>.npz`` files with
``src_li``/``dst_li`` arrays, spmm/tr_csr_fp16/mdataset2_online.py:52-70), so
these generators stand in for them with the shapes, sizes and value
distributions of the five workloads:

  chung_lu         power-law (exponent 2.1) graph, GCN-normalised, + self loops
  sbm_powerlaw     stochastic block model with power-law degrees, 70 % of edges
                   inside ~100-node communities, nodes randomly permuted
  route_mix        banded 16x8 dense blocks + 2:4-compatible row patterns +
                   uniform scatter (exercises all three routes)
  batched          block-diagonal union of many small power-law graphs

Every generator returns a canonical CSR (sorted, duplicate-free columns per
row, int32 indices) and FP32 values; callers round to FP16.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


@dataclass
class Graph:
    indptr: np.ndarray          # int32 [n_rows + 1]
    indices: np.ndarray         # int32 [nnz]
    values: np.ndarray          # float32 [nnz]
    n_rows: int
    n_cols: int
    name: str = ""
    seed: int = 0
    offsets: np.ndarray | None = None   # block-diagonal batches: node offset per graph
    meta: dict = field(default_factory=dict)

    @property
    def nnz(self) -> int:
        return int(self.indices.shape[0])

    def row_ids(self) -> np.ndarray:
        return np.repeat(np.arange(self.n_rows, dtype=np.int64), np.diff(self.indptr))


def _sorted_unique(x):
    """Sorted distinct values (sort + adjacent difference; faster than np.unique here)."""
    a = np.sort(x, kind="stable")
    if a.shape[0] == 0:
        return a
    keep = np.empty(a.shape[0], dtype=bool)
    keep[0] = True
    np.not_equal(a[1:], a[:-1], out=keep[1:])
    return a[keep]


def _csr_from_edges(rows, cols, n_rows, n_cols):
    """Canonical CSR pattern (sorted, unique) from an edge list."""
    key = rows.astype(np.int64) * n_cols + cols.astype(np.int64)
    key = _sorted_unique(key)
    r = (key // n_cols).astype(np.int64)
    c = (key % n_cols).astype(np.int32)
    indptr = np.zeros(n_rows + 1, dtype=np.int64)
    indptr[1:] = np.bincount(r, minlength=n_rows)
    indptr = np.cumsum(indptr).astype(np.int32)
    return indptr, c, r


def _unique_undirected(sample, target, n, max_rounds=12):
    """Draws edge batches from ``sample(count) -> (u, v)`` until ``target``
    distinct undirected non-loop pairs exist (or the rounds run out)."""
    keys = np.zeros(0, dtype=np.int64)
    need = target
    for _ in range(max_rounds):
        u, v = sample(int(need * 1.25) + 16)
        keep = u != v
        a = np.minimum(u[keep], v[keep]).astype(np.int64)
        b = np.maximum(u[keep], v[keep]).astype(np.int64)
        keys = _sorted_unique(np.concatenate([keys, a * n + b]))
        need = target - keys.shape[0]
        if need <= 0:
            break
    if keys.shape[0] > target:                     # trim the overshoot, deterministically
        keys = np.sort(np.random.default_rng(keys.shape[0]).choice(keys, size=target,
                                                                    replace=False))
    return keys // n, keys % n


def gcn_normalise(indptr, indices, n):
    """Symmetric GCN values 1/sqrt(d_i d_j), computed in FP32 (degrees of the
    pattern as given, which already holds the self loops)."""
    deg = np.diff(indptr).astype(np.float32)
    deg_c = np.bincount(indices, minlength=n).astype(np.float32)
    rows = np.repeat(np.arange(len(indptr) - 1), np.diff(indptr))
    d_r = np.maximum(deg[rows], 1.0)
    d_c = np.maximum(deg_c[indices], 1.0)
    return (1.0 / np.sqrt(d_r * d_c)).astype(np.float32)


def _powerlaw_weights(rng, n, exponent, mean_degree, max_frac=0.05):
    # Expected-degree sequence w_i ~ i^{-1/(gamma-1)}, scaled to the mean, capped.
    idx = np.arange(1, n + 1, dtype=np.float64)
    w = idx ** (-1.0 / (exponent - 1.0))
    w = w / w.mean() * mean_degree
    w = np.minimum(w, max_frac * n)
    w = w / w.mean() * mean_degree
    return rng.permutation(w)


def chung_lu(n=4096, avg_degree=16, exponent=2.1, seed=1, self_loops=True, gcn=True):
    rng = np.random.default_rng(seed)
    w = _powerlaw_weights(rng, n, exponent, avg_degree)
    p = w / w.sum()
    m = int(n * avg_degree / 2)
    u, v = _unique_undirected(lambda c: (rng.choice(n, size=c, p=p), rng.choice(n, size=c, p=p)),
                              m, n)
    rows = np.concatenate([u, v] + ([np.arange(n)] if self_loops else []))
    cols = np.concatenate([v, u] + ([np.arange(n)] if self_loops else []))
    indptr, indices, _ = _csr_from_edges(rows, cols, n, n)
    vals = gcn_normalise(indptr, indices, n) if gcn else rng.random(indices.shape[0], dtype=np.float32)
    return Graph(indptr, indices, vals, n, n, "chung_lu", seed,
                 meta={"avg_degree": avg_degree, "exponent": exponent})


def sbm_powerlaw(n=200_000, avg_degree=50, communities=2000, p_intra=0.7, exponent=2.1,
                 seed=2, permute=True, self_loops=True):
    """SBM with ~n/communities nodes per block, power-law expected degrees and a
    fraction p_intra of edge endpoints drawn inside the source's community."""
    rng = np.random.default_rng(seed)
    block = rng.integers(0, communities, size=n)
    w = _powerlaw_weights(rng, n, exponent, avg_degree)
    m = int(n * avg_degree / 2)
    p = w / w.sum()
    order = np.argsort(block, kind="stable")
    bstart = np.searchsorted(block[order], np.arange(communities + 1))
    cw = np.concatenate([[0.0], np.cumsum(w[order])])

    def sample(cnt):
        u = rng.choice(n, size=cnt, p=p)
        intra = rng.random(cnt) < p_intra
        v = np.empty(cnt, dtype=np.int64)
        # inter-community endpoints: degree-weighted over all nodes
        v[~intra] = rng.choice(n, size=int((~intra).sum()), p=p)
        # intra-community endpoints: degree-weighted inside the source's block
        ui = u[intra]
        bu = block[ui]
        lo, hi = cw[bstart[bu]], cw[bstart[bu + 1]]
        pos = np.searchsorted(cw, lo + rng.random(ui.shape[0]) * (hi - lo), side="right") - 1
        v[intra] = order[np.clip(pos, bstart[bu], bstart[bu + 1] - 1)]
        return u, v

    u, v = _unique_undirected(sample, m, n)
    if permute:
        perm = rng.permutation(n)
        u, v = perm[u], perm[v]
        block = block[np.argsort(perm)]
    rows = np.concatenate([u, v] + ([np.arange(n)] if self_loops else []))
    cols = np.concatenate([v, u] + ([np.arange(n)] if self_loops else []))
    indptr, indices, _ = _csr_from_edges(rows, cols, n, n)
    vals = gcn_normalise(indptr, indices, n)
    return Graph(indptr, indices, vals, n, n, "sbm_powerlaw", seed,
                 meta={"avg_degree": avg_degree, "communities": communities,
                       "p_intra": p_intra, "block": block})


def route_mix(n=65_536, target_nnz=3_200_000, band=256, seed=3, frac_dense=0.4, frac_24=0.3):
    """Banded 16x8 dense blocks (frac_dense of nnz), 2:4-compatible row patterns
    (frac_24) and uniform scatter (rest); values U[0,1]."""
    rng = np.random.default_rng(seed)
    nwin = n // 16
    rows_l, cols_l = [], []
    # dense 16x8 blocks on the band
    n_blocks = int(target_nnz * frac_dense / 128)
    bw = rng.integers(0, nwin, size=n_blocks)
    off = rng.integers(-band // 2, band // 2, size=n_blocks)
    c0 = np.clip(bw * 16 + off, 0, n - 8)
    rr = (bw[:, None] * 16 + np.arange(16)[None, :])            # [b,16]
    cc = (c0[:, None] + np.arange(8)[None, :])                  # [b,8]
    rows_l.append(np.repeat(rr, 8, axis=1).ravel())
    cols_l.append(np.tile(cc, (1, 16)).ravel())
    # 2:4 row patterns: 4-column groups where every row of the window takes 2 of 4
    n_groups = int(target_nnz * frac_24 / 32)
    gw = rng.integers(0, nwin, size=n_groups)
    gc = rng.integers(0, n // 4, size=n_groups) * 4
    pick = np.argsort(rng.random((n_groups, 16, 4)), axis=2)[:, :, :2]   # 2 of 4 per row
    rows_l.append(np.repeat(gw[:, None] * 16 + np.arange(16)[None, :], 2, axis=1).ravel())
    cols_l.append((gc[:, None, None] + pick).reshape(n_groups, 32).ravel())
    # uniform scatter
    n_sc = int(target_nnz * (1 - frac_dense - frac_24))
    rows_l.append(rng.integers(0, n, size=n_sc))
    cols_l.append(rng.integers(0, n, size=n_sc))
    indptr, indices, _ = _csr_from_edges(np.concatenate(rows_l), np.concatenate(cols_l), n, n)
    vals = rng.random(indices.shape[0], dtype=np.float32)
    return Graph(indptr, indices, vals, n, n, "route_mix", seed,
                 meta={"band": band, "frac_dense": frac_dense, "frac_24": frac_24})


def batched(num_graphs=512, nodes=(20, 500), degree=(4, 32), exponent=2.1, seed=5):
    """Block-diagonal union of independent power-law graphs (with self loops,
    GCN values); ``offsets`` holds each graph's first node."""
    rng = np.random.default_rng(seed)
    sizes = rng.integers(nodes[0], nodes[1] + 1, size=num_graphs)
    degs = rng.uniform(degree[0], degree[1], size=num_graphs)
    offsets = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
    rows_l, cols_l = [], []
    for g in range(num_graphs):
        n = int(sizes[g])
        w = _powerlaw_weights(rng, n, exponent, degs[g], max_frac=0.5)
        p = w / w.sum()
        m = max(1, min(int(n * degs[g] / 2), n * (n - 1) // 4))
        u, v = _unique_undirected(lambda c: (rng.choice(n, size=c, p=p), rng.choice(n, size=c, p=p)),
                                  m, n, max_rounds=6)
        o = offsets[g]
        rows_l += [u + o, v + o, np.arange(n) + o]
        cols_l += [v + o, u + o, np.arange(n) + o]
    total = int(offsets[-1])
    indptr, indices, _ = _csr_from_edges(np.concatenate(rows_l), np.concatenate(cols_l), total, total)
    vals = gcn_normalise(indptr, indices, total)
    return Graph(indptr, indices, vals, total, total, "batched", seed,
                 offsets=offsets, meta={"num_graphs": num_graphs})


def subgraph(g, n_nodes, seed=0):
    """Induced subgraph on n_nodes nodes of a square graph: whole communities
    (``meta['block']``) in random order when the graph has them, else a
    breadth-first region; nodes renumbered in their original order, GCN
    values recomputed on the subgraph's pattern."""
    rng = np.random.default_rng(seed)
    n = g.n_rows
    if "block" in g.meta:
        block = np.asarray(g.meta["block"])
        picked = []
        for b in rng.permutation(block.max() + 1):
            picked.append(np.nonzero(block == b)[0])
            if sum(x.size for x in picked) >= n_nodes:
                break
        nodes = np.concatenate(picked)[:n_nodes]
    else:
        seen = np.zeros(n, bool)
        order = []
        frontier = [int(rng.integers(n))]
        while len(order) < n_nodes and frontier:
            nxt = []
            for u in frontier:
                if seen[u]:
                    continue
                seen[u] = True
                order.append(u)
                nxt.extend(g.indices[g.indptr[u]:g.indptr[u + 1]].tolist())
            frontier = nxt
        nodes = np.array(order[:n_nodes])
    nodes = np.sort(nodes)
    new = np.full(n, -1, np.int64)
    new[nodes] = np.arange(nodes.size)
    rows = np.repeat(np.arange(n), np.diff(g.indptr))
    keep = (new[rows] >= 0) & (new[g.indices] >= 0)
    m = nodes.size
    indptr, indices, _ = _csr_from_edges(new[rows[keep]], new[g.indices[keep]], m, m)
    vals = gcn_normalise(indptr, indices, m)
    return Graph(indptr, indices, vals, m, m, g.name + "_sub", seed)


def random_csr(n_rows, n_cols, density, seed=0, dup=False, empty_rows=0.0):
    """Small uniform random CSR for edge-case tests (optionally with empty rows)."""
    rng = np.random.default_rng(seed)
    m = max(0, int(n_rows * n_cols * density))
    r = rng.integers(0, n_rows, size=m)
    c = rng.integers(0, n_cols, size=m)
    if empty_rows > 0:
        dead = rng.random(n_rows) < empty_rows
        keep = ~dead[r]
        r, c = r[keep], c[keep]
    indptr, indices, _ = _csr_from_edges(r, c, n_rows, n_cols)
    vals = rng.uniform(-1, 1, size=indices.shape[0]).astype(np.float32)
    return Graph(indptr, indices, vals, n_rows, n_cols, "random", seed)


def dense_features(n, k, dist="uniform", seed=0):
    rng = np.random.default_rng(seed + 7919)
    if dist == "normal":
        x = rng.standard_normal((n, k), dtype=np.float32)
    else:
        x = rng.uniform(-1, 1, size=(n, k)).astype(np.float32)
    return x.astype(np.float16)


# The five workloads, by the names used in tests and bench.py.
WORKLOADS = {
    "plain_small":   dict(gen="chung_lu", k=64, b="uniform"),
    "large_routed":  dict(gen="sbm_powerlaw", k=128, b="normal"),
    "route_mix":     dict(gen="route_mix", k=256, b="uniform"),
    "gcn_diff":      dict(gen="sbm_gcn", k=256, b="normal"),
    "batched":       dict(gen="batched", k=64, b="uniform"),
}


def make_workload(name: str, scale: float = 1.0):
    """Graph + FP16 features for a named workload; ``scale`` < 1 shrinks the
    node count for quick tests (same generator, same seed)."""
    spec = WORKLOADS[name]
    k = spec["k"]
    if name == "plain_small":
        g = chung_lu(n=max(64, int(4096 * scale)))
    elif name == "large_routed":
        n = max(2048, int(200_000 * scale))
        g = sbm_powerlaw(n=n, communities=max(20, n // 100))
    elif name == "route_mix":
        n = max(1024, int(65_536 * scale)) // 16 * 16
        g = route_mix(n=n, target_nnz=int(3_200_000 * n / 65_536))
    elif name == "gcn_diff":
        n = max(2048, int(100_000 * scale))
        g = sbm_powerlaw(n=n, avg_degree=30, communities=max(20, n // 100), seed=4)
    elif name == "batched":
        g = batched(num_graphs=max(4, int(512 * scale)))
    else:
        raise KeyError(name)
    b = dense_features(g.n_cols, k, spec["b"], seed=g.seed)
    return g, b
