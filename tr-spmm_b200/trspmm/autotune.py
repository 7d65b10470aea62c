"""Autotuner for routed plans.

The reference fixes its routing by constants (16-row windows, dense-TC
column threshold 8, 2:4 units of 2+ entries; TR-source/Block/block_online.cpp
:545-567, LIBRA_* switches) that were chosen for mma.sync on an RTX 3090.  On
sm_100a the split that pays depends on the graph: a gathered feature row only
earns its place in a tcgen05 tile when several rows of its window use it.
This tuner times the candidate plan shapes on the device and keeps the
fastest:

  engine         the row-window height and layout: "window" = the
                 reference's three routes over 16-row windows; "block" =
                 every entry on the tensor cores over 128-row blocks, each
                 distinct column of a block gathered once
  k_tile         block engine: features per tensor-core launch (the MMA's
                 N; 64..256), timed on one built plan
  reorder        cluster rows sharing columns into the same windows / blocks
  density        the router's dense-TC column threshold (rows of a window
                 using a column before it is a TC candidate; reference: 8)
  demote_below   2:4 tile columns with fewer entries go to the CUDA cores
  promote_min    CUDA-core columns with at least this many entries in a
                 window become tensor-core tiles

With backward=True the tuner times the whole backward of C = A(w) . B
(dB = A^T dC and the edge-value gradient) for candidate adjoint plans: the
fused CUDA-core pass of all-residual window plans against the block
engine's tensor-core backward, each with its edges numbered in its own
entry order, as RoutedAdjacency(edge_order="adjoint") runs it.

Large graphs are tuned on a sample (sample_nnz, default 2.5M entries): a
contiguous slice of A's rows for the forward, of A's columns (A^T's rows)
for the adjoint and the backward, so every kept row has its full degree and
the natural order's locality; plans are built once per distinct layout and
every launch setting (k_tile) is timed on it.

Results are cached as JSON keyed by device name, K, the power-of-two
buckets of nnz and rows, and the plan kind (forward, adjoint or backward),
in $TRSPMM_AUTOTUNE_CACHE or ~/.cache/trspmm/autotune.json.
"""
from __future__ import annotations

import json
import math
import os
import time

import numpy as np

from ._lib import TR_ENGINE_BLOCK, TrError
from .core import Plan

CANDIDATES = [
    {},                                                   # the reference's routing, exact
    {"demote_below": 3, "promote_min": 3},
    {"demote_below": 1000},                               # dense TC tiles + CUDA cores
    {"reorder": True, "demote_below": 4, "promote_min": 4},
    {"reorder": True, "demote_below": 1000},
    {"promote_min": 1},                                   # every column on the tensor cores
    {"density": 4, "demote_below": 1000},                 # looser dense-TC threshold
    {"engine": "block"},                                  # 128-row blocks, all tensor cores
    {"engine": "block", "reorder": True},
    {"engine": "block", "reorder": True, "k_tile": 64},
    {"engine": "block", "reorder": True, "k_tile": 128},
]

BACKWARD_CANDIDATES = [
    {"demote_below": 1000},                               # fused CUDA-core dB + dval
    {"reorder": True, "demote_below": 1000},
    {"engine": "block"},                                  # block dB, then the SDDMM
    {"engine": "block", "reorder": True},
]


def cache_path():
    return os.environ.get("TRSPMM_AUTOTUNE_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "trspmm",
                                       "autotune.json"))


def cache_key(device_name, k, nnz, n_rows, transpose, backward=False):
    b = lambda x: int(round(math.log2(max(int(x), 1))))
    kind = "bwd" if backward else ("adj" if transpose else "fwd")
    return f"{device_name}|K{int(k)}|nnz2^{b(nnz)}|rows2^{b(n_rows)}|{kind}"


def _load_cache(path):
    try:
        with open(path) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _store_cache(path, data):
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        tmp = path + ".tmp"
        with open(tmp, "w") as f:
            json.dump(data, f, indent=1, sort_keys=True)
        os.replace(tmp, path)
    except OSError:
        pass


def sample_csr(indptr, indices, values, n_rows, n_cols, transpose, target):
    """(indptr, indices, values, n_rows, n_cols) of a slice of A holding about
    `target` entries: its first rows (forward) or, for A^T's plans, its
    first columns (every row of A keeping the entries in those columns)."""
    ip = np.asarray(indptr, dtype=np.int64)
    ix = np.asarray(indices, dtype=np.int32)
    vv = None if values is None else np.asarray(values, dtype=np.float32)
    nnz = ix.shape[0]
    if nnz <= target:
        return indptr, indices, values, n_rows, n_cols
    if not transpose:
        m = int(np.searchsorted(ip, target, side="right")) - 1
        m = max(1, min(n_rows, m))
        e = int(ip[m])
        return (ip[:m + 1].astype(np.int32), ix[:e], None if vv is None else vv[:e], m, n_cols)
    counts = np.bincount(ix, minlength=n_cols)
    c = int(np.searchsorted(np.cumsum(counts), target, side="right"))
    c = max(1, min(n_cols, c))
    keep = ix < c
    rows = np.repeat(np.arange(n_rows), np.diff(ip))
    ptr = np.zeros(n_rows + 1, np.int64)
    np.add.at(ptr, rows[keep] + 1, 1)
    return (np.cumsum(ptr).astype(np.int32), ix[keep], None if vv is None else vv[keep],
            n_rows, c)


def _time_candidates(indptr, indices, values, n_rows, n_cols, k, cands, dev, transpose,
                     row_scale, reps, flush, backward):
    """Median device time of each candidate (plans built once per layout;
    launch settings such as k_tile timed on the same plan)."""
    import torch
    nnz = int(np.asarray(indices).shape[0])
    rows_b = n_cols if transpose else n_rows
    cols_b = n_rows if transpose else n_cols
    rng = np.random.default_rng(0)
    b = torch.from_numpy(rng.standard_normal((cols_b, k)).astype(np.float16)).to(dev)
    out = torch.empty((rows_b, k), dtype=torch.float32, device=dev)
    if backward:
        # the backward reads B [A cols, K] besides dC [A rows, K] (= b above)
        bb = torch.from_numpy(rng.standard_normal((n_cols, k)).astype(np.float16)).to(dev)
        ip = torch.from_numpy(np.ascontiguousarray(indptr, dtype=np.int32)).to(dev)
        ix = torch.from_numpy(np.ascontiguousarray(indices, dtype=np.int32)).to(dev)
        dval = torch.empty(nnz, dtype=torch.float32, device=dev)
    results = []
    plans = {}                       # layout options -> (plan, build seconds)
    try:
        for opts in cands:
            layout = {kk: v for kk, v in opts.items() if kk != "k_tile"}
            lkey = json.dumps(layout, sort_keys=True)
            if lkey not in plans:
                t0 = time.perf_counter()
                plans[lkey] = (Plan.build(indptr, indices, values, n_rows, n_cols,
                                          transpose=transpose, row_scale=row_scale, **layout),
                               time.perf_counter() - t0)
            plan, build_s = plans[lkey]
            if plan.info["engine"] == TR_ENGINE_BLOCK:
                plan.set_k_tile(opts.get("k_tile", 0))
            if backward and not getattr(plan, "_renumbered", False):
                # time the backward as RoutedAdjacency(edge_order="adjoint")
                # runs it: edges in the plan's own entry order, dval stored
                # sequentially (plans with tensor-core tiles have no such order)
                try:
                    order = plan.entry_order(dev)
                    new_id = torch.empty_like(order)
                    new_id[order.long()] = torch.arange(order.numel(), dtype=torch.int32,
                                                        device=dev)
                    plan.renumber_edges(new_id)
                except TrError:
                    pass
                plan._renumbered = True
            if backward:
                def run():
                    plan.adjoint_sddmm(ip, ix, b, bb, db=out, dval=dval)
            else:
                def run():
                    plan.spmm(b, out=out)
            for _ in range(2):
                run()
            ts = []
            for _ in range(reps):
                flush.fill_(1.0)
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record()
                run()
                e1.record()
                torch.cuda.synchronize()
                ts.append(e0.elapsed_time(e1))
            results.append({"options": opts, "ms": float(np.median(ts)), "build_s": build_s,
                            "info": dict(plan.info)})
    finally:
        for plan, _ in plans.values():
            plan.close()
    return results


def _finalists(results):
    """Per engine family the best layout on the sample, with every launch
    setting timed for that layout."""
    best = {}
    for r in results:
        fam = r["options"].get("engine", "window")
        if fam not in best or r["ms"] < best[fam]["ms"]:
            best[fam] = r
    out = []
    for r in best.values():
        layout = {kk: v for kk, v in r["options"].items() if kk != "k_tile"}
        out += [x["options"] for x in results
                if {kk: v for kk, v in x["options"].items() if kk != "k_tile"} == layout]
    return out


def tune(indptr, indices, values, n_rows, n_cols, k, device="cuda", candidates=None,
         transpose=False, row_scale=False, reps=5, use_cache=True, flush_mb=256,
         backward=False, sample_nnz=2_500_000):
    """Time each candidate's routed product at feature width k on `device`
    (L2 flushed before every timed launch, median of `reps`) and return
    (best_options, report).  report = {"key", "cached", "sample", "results",
    "full"}: per candidate its options, median ms, plan build seconds and
    plan info.  backward=True times the adjoint plan's whole backward (dB
    and the values' gradient, Plan.adjoint_sddmm) over BACKWARD_CANDIDATES.

    A graph above sample_nnz entries is tuned in two stages: every candidate
    on a slice of about that size (sample_csr), then, at full size, each
    engine family's best layout on the slice with its launch settings, the
    winner chosen among those.  The engines respond differently to a slice
    (the block engine's column reuse per block and work per CTA shrink with
    it), so the engine is decided at full size; within an engine the
    slice's ranking is kept.
    sample_nnz=None times every candidate at full size."""
    import torch
    dev = torch.device(device)
    name = torch.cuda.get_device_name(dev)
    nnz = int(np.asarray(indices).shape[0])
    if backward:
        transpose = True
    key = cache_key(name, k, nnz, n_rows, transpose, backward)
    path = cache_path()
    cache = _load_cache(path) if use_cache else {}
    if use_cache and key in cache:
        c = cache[key]
        return dict(c["best"]), {"key": key, "cached": True, "sample": c.get("sample"),
                                 "results": c.get("results", []), "full": c.get("full", [])}
    if candidates is not None:
        cands = candidates
    else:
        cands = BACKWARD_CANDIDATES if backward else CANDIDATES
    # a k_tile at or above K is the default launch: drop the duplicates
    cands = [c for c in cands if not (c.get("k_tile", 0) and c["k_tile"] >= k)]
    flush = torch.empty(flush_mb * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    sampled = bool(sample_nnz) and nnz > sample_nnz
    sample = None
    if sampled:
        s_ip, s_ix, s_v, s_m, s_n = sample_csr(indptr, indices, values, n_rows, n_cols,
                                               transpose, sample_nnz)
        sample = {"n_rows": int(s_m), "n_cols": int(s_n), "nnz": int(np.asarray(s_ix).shape[0]),
                  "of": {"n_rows": int(n_rows), "n_cols": int(n_cols), "nnz": nnz}}
        results = _time_candidates(s_ip, s_ix, s_v, s_m, s_n, k, cands, dev, transpose,
                                   row_scale, reps, flush, backward)
        full = _time_candidates(indptr, indices, values, n_rows, n_cols, k,
                                _finalists(results), dev, transpose, row_scale, reps, flush,
                                backward)
    else:
        results = _time_candidates(indptr, indices, values, n_rows, n_cols, k, cands, dev,
                                   transpose, row_scale, reps, flush, backward)
        full = results
    best = min(full, key=lambda r: r["ms"])["options"]
    if use_cache:
        cache = _load_cache(path)
        cache[key] = {"best": best, "results": results, "full": full, "sample": sample}
        _store_cache(path, cache)
    return dict(best), {"key": key, "cached": False, "sample": sample, "results": results,
                        "full": full}
