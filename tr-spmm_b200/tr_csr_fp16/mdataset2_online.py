"""Dataset object of the routed path (mirrors spmm/tr_csr_fp16/mdataset2_online.py).

``GCN_dataset_tcu_sptc_cuda_online`` loads a graph, pads its rows to a
multiple of ``window`` (mdataset2_online.py:58-63), builds the CSR, routes it
with ``Libra5BlockOnline.block_sptc_2to4_online`` and keeps the 30 tables as
attributes under the reference's names, with the TC / CUDA values cast to
FP16 and random FP16 features ``x`` (mdataset2_online.py:100-167).

Besides the reference's ``.npz`` loader, ``from_csr`` accepts an in-memory
CSR (the synthetic workloads use it; the reference ships no datasets).
LIBRA_TCA_REORDER=1 reorders the rows first (tr_tca_reorder.apply_tca_reorder),
as the reference's loader does (mdataset2_online.py:72-91).
"""
from __future__ import annotations

import os

import numpy as np
import scipy.sparse as sp
import torch

import Libra5BlockOnline
from tr_csr_fp16.tr_paths import load_graph_npz
from tr_csr_fp16.tr_tca_reorder import apply_tca_reorder

_NAMES = [
    "t_rowNew_offsetTensor", "t_blockTensor", "t_columnTensor", "t_valueTensor",
    "t_window_rowTensor", "t_atomicTensor", "t_binaryTensor",
    "c_row_offsetTensor", "c_rowTensor", "c_atomicTensor", "c_colTensor", "c_valueTensor",
    "c_row_offsetTensor_short", "c_rowTensor_short", "c_atomicTensor_short",
    "c_colTensor_short", "c_valueTensor_short",
    "s_columnTensor", "s_maskTensor", "s_valueTensor", "s_posTensor", "s_windowTensor",
    "s_offsetTensor", "s_tile_windowTensor", "s_tile_groupTensor", "s_tile_columnTensor",
    "s_packed_aTensor", "s_packed_metaTensor", "s_window_tile_offsetTensor", "duration",
]


class GCN_dataset_tcu_sptc_cuda_online(torch.nn.Module):
    """tr SpMM online split: dense TC blocks, strict SPTC 2:4 groups, CUDA rows."""

    def __init__(self, data, dimN, density, partsize_t, partsize_c, shortsize, data_path,
                 window, wide, tc_min_util=0.0, sptc_min_util=0.50, sptc_threshold=12,
                 values=None, mode="compat", verbose=True):
        super().__init__()
        self.graph = load_graph_npz(data_path, data) if isinstance(data, str) else data
        self.num_features = dimN
        self.window = window
        self.mode = mode
        self.verbose = verbose
        self._values = values
        self.init_edges(density, partsize_t, partsize_c, shortsize, window, wide, tc_min_util,
                        sptc_min_util, sptc_threshold)
        self.init_embedding()

    @classmethod
    def from_csr(cls, indptr, indices, n_cols, dimN, values=None, density=8, partsize_t=32,
                 partsize_c=32, shortsize=3, window=16, wide=16, tc_min_util=0.0,
                 sptc_min_util=0.5, sptc_threshold=12, mode="compat", verbose=False):
        n = len(indptr) - 1
        rows = np.repeat(np.arange(n), np.diff(indptr))
        graph = {"src_li": rows, "dst_li": np.asarray(indices), "num_nodes_src": n,
                 "num_nodes_dst": n_cols}
        return cls(graph, dimN, density, partsize_t, partsize_c, shortsize, None, window, wide,
                   tc_min_util, sptc_min_util, sptc_threshold, values=values, mode=mode,
                   verbose=verbose)

    def init_edges(self, density, partsize_t, partsize_c, shortsize, window, wide, tc_min_util,
                   sptc_min_util, sptc_threshold):
        self.num_nodes_ori = int(self.graph["num_nodes_src"])
        self.num_nodes_dst = int(self.graph["num_nodes_dst"])
        self.num_nodes = self.num_nodes_ori
        if self.num_nodes_ori % window != 0:
            self.num_nodes = self.num_nodes_ori + window - self.num_nodes_ori % window
        src_li = np.asarray(self.graph["src_li"])
        dst_li = np.asarray(self.graph["dst_li"])
        self.edge_index = np.stack([src_li, dst_li])
        self.reorder_id = None
        tca = os.environ.get("LIBRA_TCA_REORDER", "0") == "1"
        if self._values is None:
            val = np.ones(len(src_li), dtype=np.float32)
            adj = sp.coo_matrix((val, self.edge_index),
                                shape=(self.num_nodes, self.num_nodes_dst)).tocsr()
            if tca:
                # mdataset2_online.py:72-91: rows of the first num_nodes_ori
                # rows reordered, edge_index and CSR rebuilt from the result
                # (here from correct row pointers: the reference's are all zero)
                rptr, ridx, self.reorder_id = apply_tca_reorder(
                    adj.indptr, adj.indices, self.num_nodes_ori, thres=16, verbose=self.verbose)
                new_src = np.repeat(np.arange(self.num_nodes_ori), np.diff(rptr))
                self.edge_index = np.stack([new_src, ridx])
                adj = sp.coo_matrix((np.ones(len(ridx), dtype=np.float32), (new_src, ridx)),
                                    shape=(self.num_nodes, self.num_nodes_dst)).tocsr()
            self.column_index = torch.IntTensor(adj.indices)
            self.row_pointers = torch.IntTensor(adj.indptr)
            self.num_edges = self.column_index.numel()
            self.degrees = torch.randn(self.num_edges)            # mdataset2_online.py:98
        else:
            # caller-provided values, one per (src_li, dst_li) pair; sorted into CSR order
            order = np.lexsort((dst_li, src_li))
            rows, cols = src_li[order], dst_li[order]
            vals = np.asarray(self._values, dtype=np.float32)[order]
            indptr = np.zeros(self.num_nodes + 1, dtype=np.int64)
            indptr[1:] = np.cumsum(np.bincount(rows, minlength=self.num_nodes))
            if tca:
                _, _, self.reorder_id = apply_tca_reorder(indptr, cols, self.num_nodes_ori,
                                                          thres=16, verbose=self.verbose)
                perm = np.concatenate([self.reorder_id,
                                       np.arange(self.num_nodes_ori, self.num_nodes)])
                new_of = np.empty_like(perm)
                new_of[perm] = np.arange(perm.size)
                keep = np.lexsort((np.arange(rows.size), new_of[rows]))
                rows, cols, vals = new_of[rows][keep], cols[keep], vals[keep]
                indptr[1:] = np.cumsum(np.bincount(rows, minlength=self.num_nodes))
            self.column_index = torch.from_numpy(cols.astype(np.int32))
            self.row_pointers = torch.from_numpy(indptr.astype(np.int32))
            self.num_edges = self.column_index.numel()
            self.degrees = torch.from_numpy(vals)

        tensors = Libra5BlockOnline.block_sptc_2to4_online(
            self.row_pointers, self.column_index, self.degrees, partsize_t, partsize_c, shortsize,
            density, window, wide, float(tc_min_util), float(sptc_min_util), int(sptc_threshold),
            mode=self.mode)
        for name, t in zip(_NAMES, tensors):
            setattr(self, name, t)
        self.parts_t = self.t_atomicTensor.shape[0]
        self.parts_c = self.c_atomicTensor.shape[0]
        self.parts_c_short = self.c_atomicTensor_short.shape[0]
        self.partsize_c = partsize_c
        self.t_valueTensor = self.t_valueTensor.half()
        self.c_valueTensor = self.c_valueTensor.half()
        self.c_valueTensor_short = self.c_valueTensor_short.half()
        if self.verbose:
            tcu_nnz = self.t_valueTensor.numel()
            sptc_nnz = int((self.s_posTensor >= 0).sum().item())
            cuda_nnz = self.c_valueTensor.numel() + self.c_valueTensor_short.numel()
            print(f"tcu: {tcu_nnz};   sptc: {sptc_nnz};   cuda: {cuda_nnz}")
            print(f"parts_t: {self.parts_t};   parts_c: {self.parts_c};   parts_c_short: "
                  f"{self.parts_c_short};   sptc_groups: {self.s_columnTensor.shape[0]};   "
                  f"sptc_tiles: {self.s_tile_windowTensor.shape[0]}")

    def init_embedding(self):
        self.x = torch.randn(self.num_nodes_dst, self.num_features).half()
