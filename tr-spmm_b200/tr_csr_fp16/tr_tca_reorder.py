"""TCA row reorder (mirrors spmm/tr_csr_fp16/tr_tca_reorder.py).

``apply_tca_reorder`` keeps the reference's signature and return values:
the row order comes from libtrspmm's tr_tca_order (MinHash-LSH candidate
pairs, exact Jaccard, two levels of capped clustering, native threads, or
the GPU for the signatures and similarities), and the CSR is rebuilt the way
the reference rebuilds it (tr_tca_reorder.py:318-357: entries relabelled by
new row, ``np.argsort`` of the new row ids, row pointers from the sorted
rows), so that the within-row column order matches too.
"""
from __future__ import annotations

import time

import numpy as np

from trspmm import core


def apply_tca_reorder(row_ptr, col_ind, num_nodes, thres=16, verbose=True, device=None):
    """(new_row_ptr int32 [num_nodes+1], new_col_ind int32 [nnz],
    reorder_id int32 [num_nodes], new position -> old row).  Only the first
    ``num_nodes`` rows are reordered (the reference is called with the
    unpadded node count).  ``device``: None uses the GPU when one is
    present, True / False force it."""
    t0 = time.time()
    row_ptr = np.asarray(row_ptr)
    col_ind = np.asarray(col_ind)
    n = int(num_nodes)
    rp = np.ascontiguousarray(row_ptr[:n + 1], dtype=np.int32)
    nnz = int(rp[n]) if n >= 0 else 0
    ci = np.ascontiguousarray(col_ind[:nnz], dtype=np.int32)
    if device is None:
        import torch
        device = torch.cuda.is_available()
    order, st = core.tca_order(rp, ci, n, thres=thres, device=device)
    if verbose:
        print(f"TCA: {n} rows, LSH {st['bands']} bands x {st['rows_per_band']} rows, "
              f"{st['pairs1']} candidate row pairs -> {st['clusters1']} row-level clusters, "
              f"{st['pairs2']} cluster pairs -> {st['clusters2']} groups")
    old_to_new = np.empty(n, dtype=np.int32)
    old_to_new[order] = np.arange(n, dtype=np.int32)
    # int32 row ids and numpy's default sort, as in the reference: equal ids
    # (one row's entries) come out in the order that sort leaves them
    new_src = old_to_new[np.repeat(np.arange(n), np.diff(rp.astype(np.int64)))]
    sort_idx = np.argsort(new_src)
    new_col_ind = ci[sort_idx].astype(np.int32)
    new_row_ptr = np.zeros(n + 1, dtype=np.int32)
    new_row_ptr[1:] = np.cumsum(np.bincount(new_src, minlength=n))
    if verbose:
        print(f"TCA: total reorder time = {time.time() - t0:.2f}s")
    return new_row_ptr, new_col_ind, order.astype(np.int32)
