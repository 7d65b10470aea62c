"""On-disk plan cache: routing and layout are paid once per graph.

The reference routes the graph on every run (the router is called from the
dataset object's constructor, TR-source/spmm/tr_csr_fp16/mdataset2_online.py
:100-153).  Here a built host plan (everything a device plan is uploaded
from) is written to a plan file (tr_host_plan_save: versioned binary with a
checksum) under a key that hashes the CSR, its values, the plan options and
the routing parameters; a later run with the same key loads the file
(tr_host_plan_load, which refuses damaged or inconsistent files) and only
uploads it.  A damaged file is rebuilt and replaced; a directory that cannot
be written only costs the caching.

Files live in $TRSPMM_PLAN_CACHE, else ~/.cache/trspmm/plans.
"""
from __future__ import annotations

import ctypes
import hashlib
import json
import os

import numpy as np

from . import core
from ._lib import TrError, check, lib

FORMAT = 1          # bump when the plan layout or the key's meaning changes


def default_dir():
    return os.environ.get("TRSPMM_PLAN_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "trspmm", "plans"))


def _options(row_scale=False, promote_min=0, transpose=False, reorder=False, demote_below=0,
             mode="exact", engine="window", **route_kw):
    if not (isinstance(reorder, (str, bool)) or reorder is None):
        raise ValueError("the plan cache takes named reorder modes (False, True / 'label', 'tca')")
    if reorder not in core.REORDER_MODES:
        raise ValueError(f"unknown reorder mode {reorder!r}")
    # False / True as before ('none' / 'label'), 'tca' by name
    reorder = {0: False, 1: True, 2: "tca"}[core.REORDER_MODES[reorder]]
    opts = {"row_scale": bool(row_scale), "promote_min": int(promote_min),
            "transpose": bool(transpose), "reorder": reorder,
            "demote_below": int(demote_below), "mode": mode}
    if engine != "window":              # keys of window plans stay as they were
        if engine not in core.ENGINES:
            raise ValueError(f"unknown plan engine {engine!r}")
        opts["engine"] = engine
    return opts, route_kw


def plan_key(indptr, indices, values, n_rows, n_cols, **plan_kw):
    """Hex key of a plan: SHA-256 over the CSR arrays, the values, the sizes,
    the plan options and the routing parameters."""
    opts, route_kw = _options(**plan_kw)
    h = hashlib.sha256()
    for a, dt in ((indptr, np.int32), (indices, np.int32), (values, np.float32)):
        if a is None:
            h.update(b"none")
        else:
            h.update(np.ascontiguousarray(a, dtype=dt).tobytes())
        h.update(b"|")
    h.update(json.dumps({"n_rows": int(n_rows), "n_cols": int(n_cols), "opts": opts,
                         "route": {k: route_kw[k] for k in sorted(route_kw)},
                         "format": FORMAT}, sort_keys=True).encode())
    return h.hexdigest()


def _build_host(indptr, indices, values, n_rows, n_cols, **plan_kw):
    opts, route_kw = _options(**plan_kw)
    rp = np.ascontiguousarray(indptr, dtype=np.int32)
    ci = np.ascontiguousarray(indices, dtype=np.int32)
    vv = None if values is None else np.ascontiguousarray(values, dtype=np.float32)
    prm = core._params(mode=opts["mode"], **route_kw)
    reorder = core._resolve_reorder(opts["reorder"], rp, ci, n_rows, n_cols, opts["transpose"])
    po, _keep = core.plan_opts(opts["row_scale"], opts["promote_min"], opts["transpose"],
                               reorder, opts["demote_below"], opts.get("engine", "window"))
    h = ctypes.c_void_p()
    check(lib().tr_plan_build_host(core._vp(rp), core._vp(ci), core._vp(vv), int(n_rows),
                                   int(n_cols), ctypes.byref(prm), ctypes.byref(po),
                                   ctypes.byref(h)))
    return h


def cached_host_plan(indptr, indices, values, n_rows, n_cols, directory=None, **plan_kw):
    """(host plan handle, path, hit): loaded from the cache when a valid plan
    file exists for this key, otherwise built and written.  The caller frees
    the handle (tr_host_plan_free)."""
    d = directory or default_dir()
    path = os.path.join(d, plan_key(indptr, indices, values, n_rows, n_cols, **plan_kw) + ".trplan")
    L = lib()
    if os.path.exists(path):
        h = ctypes.c_void_p()
        try:
            check(L.tr_host_plan_load(path.encode(), ctypes.byref(h)))
            return h, path, True
        except TrError:
            pass                                   # damaged: rebuild below
    h = _build_host(indptr, indices, values, n_rows, n_cols, **plan_kw)
    try:
        os.makedirs(d, exist_ok=True)
        check(L.tr_host_plan_save(h, path.encode()))
    except (OSError, TrError):
        pass                                       # the plan is still good, just not cached
    return h, path, False


def cached_plan(indptr, indices, values, n_rows, n_cols, directory=None, **plan_kw):
    """Device plan (core.Plan) through the cache; same options as
    core.Plan.build.  The plan's ``cache_hit`` says whether routing was
    skipped.  ``k_tile`` (a launch setting, not part of the file) is applied
    after the upload."""
    k_tile = plan_kw.pop("k_tile", 0)
    h, path, hit = cached_host_plan(indptr, indices, values, n_rows, n_cols, directory, **plan_kw)
    L = lib()
    try:
        p = ctypes.c_void_p()
        check(L.tr_host_plan_upload(h, ctypes.byref(p)))
    finally:
        L.tr_host_plan_free(h)
    plan = core.Plan(p)
    plan.cache_hit, plan.cache_path = hit, path
    if k_tile:
        plan.set_k_tile(k_tile)
    return plan
