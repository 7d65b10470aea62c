"""Dataset paths (mirrors spmm/tr_csr_fp16/tr_paths.py: TR_ROOT, TR_DATA_ROOT,
TR_DATA_CSV, TR_RESULTS_DIR)."""
from pathlib import Path
import os

import numpy as np


def project_root() -> Path:
    return Path(os.environ.get("TR_ROOT", Path(__file__).resolve().parents[2])).resolve()


def data_root() -> Path:
    return Path(os.environ.get("TR_DATA_ROOT", project_root() / "dgl_dataset")).resolve()


def dataset_path(data_path: str, data: str) -> Path:
    base = Path(data_path)
    if not base.is_absolute():
        base = data_root() / data_path
    return (base / f"{data}.npz").resolve()


def load_graph_npz(data_path: str, data: str):
    """``<data_root>/<data_path>/<data>.npz`` with src_li, dst_li, num_nodes_src,
    num_nodes_dst (the reference's format, mdataset2_online.py:52-70)."""
    path = dataset_path(data_path, data)
    if not path.exists():
        raise FileNotFoundError(f"Cannot find tr dataset '{data}' at {path}. Set TR_DATA_ROOT.")
    return np.load(path)


def index_csv(default_name: str = "data_filter.csv") -> Path:
    explicit = os.environ.get("TR_DATA_CSV")
    if explicit:
        return Path(explicit).resolve()
    root = project_root()
    for name in (default_name, "data_filter.csv", "data.csv"):
        if (root / name).exists():
            return (root / name).resolve()
    return (root / default_name).resolve()


def results_root() -> Path:
    root = Path(os.environ.get("TR_RESULTS_DIR", project_root() / "res")).resolve()
    root.mkdir(parents=True, exist_ok=True)
    return root


def result_path(*parts: str) -> Path:
    path = results_root().joinpath(*parts)
    path.parent.mkdir(parents=True, exist_ok=True)
    return path
