"""Sparse-matrix files as CSR (int32 indptr / indices, float32 values).

Formats the reference's scripts read:
  .npz, scipy.sparse.save_npz           (keys 'format' / 'indices' ...)
  .npz, edge lists src_li, dst_li with 'shape' and optional 'data'
                                        (TR-source/test_24_matching.py:80-106)
  .npz, edge lists src_li, dst_li with num_nodes_src / num_nodes_dst
                                        (spmm/tr_csr_fp16/mdataset2_online.py:52-70)
  .mtx, MatrixMarket (coordinate real / integer / pattern, or array)
                                        (TR-source/test_24_matching.py:109-146)
Duplicate (row, col) edges are summed (as a COO -> CSR conversion does),
column indices are sorted within rows, pattern files get value 1.
"""
from __future__ import annotations

import os
from dataclasses import dataclass

import numpy as np


@dataclass
class CsrMatrix:
    indptr: np.ndarray     # int32 [n_rows + 1]
    indices: np.ndarray    # int32 [nnz]
    values: np.ndarray     # float32 [nnz]
    n_rows: int
    n_cols: int

    @property
    def nnz(self) -> int:
        return int(self.indices.shape[0])


def _from_scipy(m) -> CsrMatrix:
    import scipy.sparse as sp
    m = sp.csr_matrix(m)
    m.sum_duplicates()
    m.sort_indices()
    return CsrMatrix(m.indptr.astype(np.int32), m.indices.astype(np.int32),
                     m.data.astype(np.float32), int(m.shape[0]), int(m.shape[1]))


def _edge_list(raw) -> CsrMatrix:
    import scipy.sparse as sp
    src = np.asarray(raw["src_li"]).astype(np.int64)
    dst = np.asarray(raw["dst_li"]).astype(np.int64)
    if "shape" in raw:
        shape = tuple(int(x) for x in np.asarray(raw["shape"]).tolist())
    elif "num_nodes_src" in raw:
        shape = (int(raw["num_nodes_src"]), int(raw["num_nodes_dst"]))
    else:
        n = int(max(src.max(initial=-1), dst.max(initial=-1)) + 1)
        shape = (n, n)
    val = (np.asarray(raw["data"]).astype(np.float32) if "data" in raw
           else np.ones(src.shape[0], dtype=np.float32))
    if src.size and (src.min() < 0 or dst.min() < 0 or src.max() >= shape[0] or
                     dst.max() >= shape[1]):
        raise ValueError(f"edge endpoints outside the {shape[0]} x {shape[1]} matrix")
    return _from_scipy(sp.coo_matrix((val, (src, dst)), shape=shape))


def load_matrix(path: str) -> CsrMatrix:
    """CSR of the sparse matrix stored at ``path`` (formats in the module
    docstring)."""
    ext = os.path.splitext(path)[1].lower()
    if ext == ".npz":
        import scipy.sparse as sp
        with np.load(path, allow_pickle=False) as raw:
            keys = set(raw.keys())
            if "format" in keys or "indices" in keys:
                return _from_scipy(sp.load_npz(path))
            if "src_li" in keys and "dst_li" in keys:
                return _edge_list({k: raw[k] for k in keys})
        raise ValueError(f"{path}: neither a scipy sparse .npz nor an src_li / dst_li edge list")
    if ext == ".mtx":
        from scipy.io import mminfo, mmread
        field = mminfo(path)[4]
        m = mmread(path)
        if isinstance(m, np.ndarray):
            import scipy.sparse as sp
            m = sp.csr_matrix(m)
        out = _from_scipy(m)
        if field == "pattern":
            out.values = np.ones(out.nnz, dtype=np.float32)
        return out
    raise ValueError(f"unsupported matrix file format: {ext} (use .npz or .mtx)")
