"""Drop-in for the reference's ``matching_utils_bucket`` extension
(high/low-half bucketed 2:4 matching statistics,
TR-source/Block/block_matching_bucket.cpp:430-480): same function,
arguments and dict keys, computed by tr_match_2to4 (TR_MATCH_BUCKET)."""
from _matching_common import run


def match_2to4_bucket(row_ptr, col_ind, values, window_size=16):
    return run("bucket", row_ptr, col_ind, values, window_size)
