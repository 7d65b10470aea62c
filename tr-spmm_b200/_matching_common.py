"""Shared body of the matching-stats drop-in modules (matching_utils,
matching_utils_hash, matching_utils_bucket): argument handling like the
reference's pybind11 wrappers (int32 / float32 arrays, forcecast), and the
returned dict, which carries the reference's keys for the variant plus the
other variants' names for the same counters (the reference's own comparison
script reads num_groups from the sliding variant and num_sptc_groups /
num_tc_blocks from the others)."""
from __future__ import annotations

import numpy as np

from trspmm import core


def run(variant, row_ptr, col_ind, values, window_size, dense_threshold=8, t_max=8):
    rp = np.ascontiguousarray(np.asarray(row_ptr), dtype=np.int32)
    ci = np.ascontiguousarray(np.asarray(col_ind), dtype=np.int32)
    np.ascontiguousarray(np.asarray(values), dtype=np.float32)     # checked like the reference; unused
    st = core.match_2to4(rp, ci, variant, window_size, dense_threshold, t_max)
    out = {k: int(st[k]) for k in ("total_rows", "total_cols", "total_nnz", "num_row_panels")}
    out["sparsity"] = float(st["sparsity"])
    out["num_groups"] = out["num_sptc_groups"] = int(st["num_groups"])
    out["num_tc_blocks"] = int(st["num_tc_blocks"])
    for k in ("num_16x16_blocks", "block_padding_groups", "fine_fallback", "coarse_fallback",
              "fake_zeros"):
        out[k] = int(st[k])
    return out
