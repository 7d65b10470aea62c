"""The no-alloc device router entry point, called through the C ABI.

Some callers cannot let a library allocate GPU memory: code that runs inside
a caller-owned memory pool or arena, or under a framework allocator that
must account for every byte, where a cudaMalloc / cudaFree inside the
library would synchronise the device or break that accounting.  For them
tr_route_tc_device_noalloc takes caller-allocated output buffers and keeps
its own scratch in a static device array.  These tests check that its
tables equal those of the allocating entry point (tr_route_tc_device), bit
for bit (the tolerance the router tests use), on two calls in a row — the
second call must not see anything the first left in the shared scratch —
and that it refuses sizes beyond its stated limits with clear errors.

This file is collected last on purpose: if it fails, a run that stops at
the first failure has already run every other test.
"""
import ctypes

import numpy as np
import pytest
import torch

import trspmm
from trspmm import graphs
from trspmm._lib import check, lib
from trspmm.core import _params

pytestmark = pytest.mark.gpu


def _noalloc(g, cuda, cap_sub=None, cap_val=None, **kw):
    """Call the entry point with buffers the caller (this test) allocates."""
    ip = torch.from_numpy(np.ascontiguousarray(g.indptr, np.int32)).to(cuda)
    ix = torch.from_numpy(np.ascontiguousarray(g.indices, np.int32)).to(cuda)
    vv = torch.from_numpy(np.ascontiguousarray(g.values, np.float32)).to(cuda)
    if cap_sub is None:
        cap_sub = g.nnz + 1               # every sub-block holds at least one entry
    if cap_val is None:
        cap_val = g.nnz
    t_column = torch.full((cap_sub * 8,), -7, dtype=torch.int32, device=cuda)
    t_binary = torch.zeros(cap_sub * 2, dtype=torch.int64, device=cuda)
    t_value = torch.zeros(cap_val, dtype=torch.float32, device=cuda)
    t_block = torch.zeros(cap_sub + 1, dtype=torch.int32, device=cuda)
    n_sub, n_val = ctypes.c_int64(-1), ctypes.c_int64(-1)
    prm = _params(mode="exact", skip_tc=False, **kw)
    stream = torch.cuda.current_stream(cuda).cuda_stream
    rc = lib().tr_route_tc_device_noalloc(
        ctypes.c_void_p(ip.data_ptr()), ctypes.c_void_p(ix.data_ptr()),
        ctypes.c_void_p(vv.data_ptr()), int(g.n_rows), ctypes.byref(prm),
        ctypes.c_void_p(t_column.data_ptr()), ctypes.c_void_p(t_binary.data_ptr()),
        ctypes.c_void_p(t_value.data_ptr()), ctypes.c_void_p(t_block.data_ptr()),
        ctypes.c_int64(cap_sub), ctypes.c_int64(cap_val), ctypes.byref(n_sub), ctypes.byref(n_val),
        ctypes.c_void_p(stream))
    check(rc)
    s, v = n_sub.value, n_val.value
    return {"t_column": t_column[:s * 8].cpu().numpy(), "t_binary": t_binary[:s * 2].cpu().numpy(),
            "t_value": t_value[:v].cpu().numpy(), "t_block_offset": t_block[:s + 1].cpu().numpy()}


def _allocating(g, cuda, **kw):
    return trspmm.route_tc_device(torch.from_numpy(g.indptr).to(cuda),
                                  torch.from_numpy(g.indices).to(cuda),
                                  torch.from_numpy(np.asarray(g.values, np.float32)).to(cuda),
                                  g.n_rows, **kw)


def _same(a, b):
    for name in ("t_column", "t_binary", "t_value", "t_block_offset"):
        assert a[name].dtype == b[name].dtype, name
        assert np.array_equal(a[name], b[name]), name


def test_two_calls_match_the_allocating_entry_point(cuda):
    first = graphs.route_mix(n=2048, target_nnz=120_000)        # many dense-TC sub-blocks
    second = graphs.chung_lu(n=4096)                            # few
    got1 = _noalloc(first, cuda)
    got2 = _noalloc(second, cuda, density=4)
    assert len(got1["t_value"]) > 0 and len(got2["t_value"]) > 0
    _same(got1, _allocating(first, cuda))
    _same(got2, _allocating(second, cuda, density=4))
    # and the first graph again, after the second left its contents behind
    _same(_noalloc(first, cuda), _allocating(first, cuda))


def test_refuses_sizes_beyond_its_limits(cuda):
    g = graphs.route_mix(n=2048, target_nnz=120_000)
    with pytest.raises(trspmm.TrError, match="capacity too small"):
        _noalloc(g, cuda, cap_sub=1, cap_val=1)
    # a window with more entries than the kernel keeps in shared memory
    ip = np.array([0, 3000] + [3000] * 15, np.int32)
    big = graphs.Graph(ip, np.arange(3000, dtype=np.int32), np.ones(3000, np.float32), 16, 5000)
    with pytest.raises(trspmm.TrError, match="more than 2048 entries"):
        _noalloc(big, cuda)
    # more rows than the scratch has windows for
    n = 1_048_576 + 16
    huge = graphs.Graph(np.zeros(n + 1, np.int32), np.zeros(0, np.int32), np.zeros(0, np.float32),
                        n, 4)
    with pytest.raises(trspmm.TrError, match="at most 1048576 rows"):
        _noalloc(huge, cuda)
    # still correct after the refusals
    _same(_noalloc(g, cuda), _allocating(g, cuda))
