"""Drop-in for the reference's ``matching_utils_hash`` extension
(exact-complement hash + sliding-window 2:4 matching statistics,
TR-source/Block/block_matching_hash.cpp:373-420): same function, arguments
and dict keys, computed by tr_match_2to4 (TR_MATCH_HASH)."""
from _matching_common import run


def match_2to4_hash(row_ptr, col_ind, values, window_size=16):
    return run("hash", row_ptr, col_ind, values, window_size)
