"""Where the drop-in loader finds graphs and writes results.

Callers of the reference's loader configure it through four environment
variables, kept here with the same meaning (spmm/tr_csr_fp16/tr_paths.py):
TR_ROOT (the project directory), TR_DATA_ROOT (graph files), TR_DATA_CSV (the
dataset index) and TR_RESULTS_DIR (result files).  Everything resolves
through one table of locations; graph files are read by
``trspmm.datasets.load_matrix``'s edge-list reader, so the reference's
``src_li`` / ``dst_li`` / ``num_nodes_*`` archives load the same way here.
"""
from __future__ import annotations

import os
from pathlib import Path

import numpy as np

# environment variable -> location used when it is unset (relative to TR_ROOT)
_LOCATIONS = {
    "TR_DATA_ROOT": "dgl_dataset",
    "TR_RESULTS_DIR": "res",
}
_INDEX_NAMES = ("data_filter.csv", "data.csv")


def _location(var: str) -> Path:
    if var == "TR_ROOT":
        fallback = Path(__file__).resolve().parent.parent.parent
    else:
        fallback = _location("TR_ROOT") / _LOCATIONS[var]
    return Path(os.environ.get(var) or fallback).resolve()


def project_root() -> Path:
    return _location("TR_ROOT")


def data_root() -> Path:
    return _location("TR_DATA_ROOT")


def dataset_path(data_path: str, data: str) -> Path:
    """``<data_path>/<data>.npz``; a relative ``data_path`` hangs off data_root()."""
    folder = Path(data_path)
    return ((folder if folder.is_absolute() else data_root() / folder) / (data + ".npz")).resolve()


def load_graph_npz(data_path: str, data: str):
    """The arrays of the graph archive ``data`` as a dict (src_li, dst_li and
    the node counts or shape, as the reference's loader reads them)."""
    path = dataset_path(data_path, data)
    if not path.is_file():
        raise FileNotFoundError(f"graph '{data}' not found at {path} (set TR_DATA_ROOT)")
    with np.load(path, allow_pickle=False) as raw:
        return {key: raw[key] for key in raw.files}


def index_csv(default_name: str = "data_filter.csv") -> Path:
    """The dataset index: TR_DATA_CSV if set, else the first index file present
    in the project directory, else ``default_name`` there."""
    if os.environ.get("TR_DATA_CSV"):
        return Path(os.environ["TR_DATA_CSV"]).resolve()
    root = project_root()
    present = [root / n for n in dict.fromkeys((default_name,) + _INDEX_NAMES) if (root / n).exists()]
    return (present[0] if present else root / default_name).resolve()


def results_root() -> Path:
    out = _location("TR_RESULTS_DIR")
    out.mkdir(parents=True, exist_ok=True)
    return out


def result_path(*parts: str) -> Path:
    """A file under results_root(), its folder created."""
    target = results_root().joinpath(*parts)
    target.parent.mkdir(parents=True, exist_ok=True)
    return target
