"""Drop-in for the reference's ``Libra5BlockOnline`` extension module.

``block_sptc_2to4_online`` keeps the reference signature and return list
(TR-source/Block/block_online.cpp:545-549, :844-870): CPU int32 row_ptr /
column, CPU float32 values in; 30 CPU tensors out (29 route tables plus the
routing time).  The tables are bit-identical to the reference's, including
its per-row truncation inside 4-column SPTC groups; pass ``mode="exact"`` to
have the truncated entries moved into the CUDA residual instead.
"""
from __future__ import annotations

import numpy as np
import torch

from trspmm import core


def block_sptc_2to4_online(row1, column1, values1, partSize_t, partSize_c, shortSize, density,
                           window, wide, tc_min_util, sptc_min_util, sptc_threshold,
                           mode="compat"):
    if not (row1.dtype == torch.int32 and column1.dtype == torch.int32):
        raise RuntimeError("Expected row1.dtype() == torch::kInt32 && column1.dtype() == torch::kInt32")
    if values1.dtype != torch.float32:
        raise RuntimeError("Expected values1.dtype() == torch::kFloat32")
    if not (0 < window <= 32 and 0 < wide <= 32):
        raise RuntimeError("Expected window > 0 && window <= 32 && wide > 0 && wide <= 32")
    tabs = core.route(row1.cpu().numpy(), column1.cpu().numpy(), values1.cpu().numpy(),
                      partSize_t, partSize_c, shortSize, density, window, wide, tc_min_util,
                      sptc_min_util, sptc_threshold, mode=mode)
    out = [torch.from_numpy(np.ascontiguousarray(t)) for t in tabs[:29]]
    out.append(torch.tensor(float(tabs[29]), dtype=torch.float32))
    return out
