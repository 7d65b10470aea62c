"""Drop-in for the reference's ``matching_utils`` extension (sliding-window
dual-routing 2:4 matching statistics,
TR-source/Block/block_matching_window_para_dr.cpp:346-441): same function,
arguments and dict keys, computed by tr_match_2to4 (TR_MATCH_SLIDING)."""
from _matching_common import run


def match_2to4(row_ptr, col_ind, values, window_size=16, dense_threshold=8, t_max=8):
    return run("sliding", row_ptr, col_ind, values, window_size, dense_threshold, t_max)
