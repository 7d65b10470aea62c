"""Drop-in for the reference's ``matching_utils_online`` extension (the CUDA
dual-routing matcher, TR-source/Block/block_matching_online.cu:554-668): same
function, arguments and dict keys, computed on the GPU by
tr_match_2to4_online with a deterministic column order (the reference's
depends on hash-slot arrival).  Like the reference's, each call copies the
matrix to the device and waits for the result."""
from trspmm import core


def match_2to4_online(row_ptr, col_ind, values, window_size=16, dense_threshold=8, t_max=8):
    import numpy as np
    np.ascontiguousarray(np.asarray(values), dtype=np.float32)     # checked like the reference; unused
    st = core.match_2to4_online(row_ptr, col_ind, window_size, dense_threshold, t_max)
    out = {k: int(st[k]) for k in ("total_rows", "total_cols", "total_nnz", "num_tc_blocks",
                                   "dense_to_tc_cols", "dense_to_sptc_cols", "num_16x16_blocks",
                                   "block_padding_groups", "fake_zeros", "num_row_panels")}
    out["num_sptc_groups"] = out["num_groups"] = int(st["num_groups"])
    out["fine_fb"] = out["fine_fallback"] = int(st["fine_fallback"])
    out["coarse_fb_cols"] = out["coarse_fallback"] = int(st["coarse_fallback"])
    out["sparsity"] = float(st["sparsity"])
    return out
