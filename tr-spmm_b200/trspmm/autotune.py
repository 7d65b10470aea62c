"""Autotuner for routed plans.

The reference fixes its routing by constants (16-row windows, dense-TC
column threshold 8, 2:4 units of 2+ entries; TR-source/Block/block_online.cpp
:545-567, LIBRA_* switches) that were chosen for mma.sync on an RTX 3090.  On
sm_100a the split that pays depends on the graph: a gathered feature row only
earns its place in a tcgen05 tile when several rows of its window use it.
This tuner times the candidate plan shapes on the device and keeps the
fastest:

  engine         "window": the reference's three routes over 16-row windows;
                 "block": every entry on the tensor cores over 128-row
                 blocks, each distinct column of a block gathered once
  reorder        cluster rows sharing columns into the same windows / blocks
  demote_below   2:4 tile columns with fewer entries go to the CUDA cores
  promote_min    CUDA-core columns with at least this many entries in a
                 window become tensor-core tiles

With backward=True the tuner times the whole backward of C = A(w) . B
(dB = A^T dC and the edge-value gradient) for candidate adjoint plans: the
fused CUDA-core pass of all-residual window plans against the block engine's
dB followed by the SDDMM.

The window height (16 rows, the reference's tables; 128-row blocks for the
block engine) and the feature chunk are fixed by the kernels; the kernel
for the full product is chosen by the library from K.

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

from .core import Plan

CANDIDATES = [
    {},                                                   # the reference's routing, exact
    {"demote_below": 3, "promote_min": 3},
    {"demote_below": 1000},                               # dense TC tiles + CUDA cores
    {"reorder": True, "demote_below": 4, "promote_min": 4},
    {"reorder": True, "demote_below": 1000},
    {"promote_min": 1},                                   # every column on the tensor cores
    {"engine": "block"},                                  # 128-row blocks, all tensor cores
    {"engine": "block", "reorder": True},
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


def tune(indptr, indices, values, n_rows, n_cols, k, device="cuda", candidates=None,
         transpose=False, row_scale=False, reps=5, use_cache=True, flush_mb=256,
         backward=False):
    """Time each candidate's routed product at feature width k on `device`
    (L2 flushed before every timed launch, median of `reps`) and return
    (best_options, report).  report = {"key", "cached", "results": [...]} with
    per candidate its options, median ms, plan build seconds and plan info.
    backward=True times the adjoint plan's whole backward (dB and the values'
    gradient, Plan.adjoint_sddmm) over BACKWARD_CANDIDATES."""
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
        return dict(cache[key]["best"]), {"key": key, "cached": True,
                                          "results": cache[key].get("results", [])}
    if candidates is not None:
        cands = candidates
    else:
        cands = BACKWARD_CANDIDATES if backward else CANDIDATES
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
    flush = torch.empty(flush_mb * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    results = []
    for opts in cands:
        t0 = time.perf_counter()
        plan = Plan.build(indptr, indices, values, n_rows, n_cols, transpose=transpose,
                          row_scale=row_scale, **opts)
        build_s = time.perf_counter() - t0
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
        plan.close()
    best = min(results, key=lambda r: r["ms"])["options"]
    if use_cache:
        cache = _load_cache(path)
        cache[key] = {"best": best, "results": results}
        _store_cache(path, cache)
    return dict(best), {"key": key, "cached": False, "results": results}
