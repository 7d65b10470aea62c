"""Shared test utilities: golden fixtures, reference matrices, error norms."""
import glob
import os

import numpy as np
import scipy.sparse as sp

HERE = os.path.dirname(os.path.abspath(__file__))
TABLES = None


def golden_files():
    return sorted(glob.glob(os.path.join(HERE, "golden", "route_*.npz")))


def load_golden(path):
    import oracle
    z = np.load(path)
    args = tuple(z["args"].tolist())
    args = tuple(int(a) if i not in (6, 7) else float(a) for i, a in enumerate(args))
    tabs = [z[n] for n in oracle.TABLE_NAMES[:29]]
    return z["indptr"], z["indices"], z["values"], int(z["n_cols"]), args, tabs


def half_csr(indptr, indices, values, n_rows, n_cols):
    """A with FP16-rounded values, stored as float64."""
    v = np.asarray(values, dtype=np.float32).astype(np.float16).astype(np.float64)
    return sp.csr_matrix((v, indices, indptr), shape=(n_rows, n_cols))


def rel_err(out, ref):
    """Max abs error normalised by max |ref| (the reported 'max relative error')."""
    out = np.asarray(out, dtype=np.float64)
    ref = np.asarray(ref, dtype=np.float64)
    scale = max(np.abs(ref).max(), 1e-30) if ref.size else 1.0
    return float(np.abs(out - ref).max() / scale) if ref.size else 0.0


def spmm_ref(A, b16):
    """FP64 C = A . B (B given as FP16)."""
    return np.asarray(A @ np.asarray(b16, dtype=np.float64))
