"""The whole router on the GPU (tr_route_device) against the host router,
all 29 tables item for item (dtype, shape and bits), in both modes.

The host router is itself pinned to the reference's compiled router (golden
fixtures, tests/test_router.py), so equality here carries that pin to the
device.  Inputs have their rows sorted by column (duplicates kept), which
the device router requires; on golden matrices whose rows already are, the
device tables are also compared with the reference's own output directly.
"""
import numpy as np
import pytest
import torch

import oracle
import trspmm
from helpers import golden_files, load_golden
from trspmm import graphs

pytestmark = pytest.mark.gpu


def _sorted_rows(indptr, indices, values):
    """Rows sorted by column (stable: duplicates keep their order)."""
    ip = np.asarray(indptr, np.int32)
    ix = np.asarray(indices, np.int32)
    vv = np.asarray(values, np.float32)
    rows = np.repeat(np.arange(len(ip) - 1), np.diff(ip))
    o = np.lexsort((ix, rows))
    return ip, ix[o].copy(), vv[o].copy()


def _same(a, b):
    bad = [n for n, x, y in zip(oracle.TABLE_NAMES[:29], a[:29], b[:29])
           if not (x.dtype == y.dtype and x.shape == y.shape and np.array_equal(x, y))]
    assert not bad, f"tables differ: {bad}"


def _compare(ip, ix, vv, cuda, **kw):
    kw.setdefault("unit_min_nnz", 2)
    kw.setdefault("skip_tc", False)
    host = trspmm.route(ip, ix, vv, **kw)
    dev = trspmm.route_device(torch.from_numpy(ip).to(cuda), torch.from_numpy(ix).to(cuda),
                              torch.from_numpy(vv).to(cuda), **kw)
    _same(dev, host)
    return dev


@pytest.mark.parametrize("mode", ["compat", "exact"])
@pytest.mark.parametrize("path", golden_files(), ids=lambda p: p.split("route_")[-1][:-4])
def test_golden_matrices(cuda, path, mode):
    indptr, indices, values, n_cols, args, ref = load_golden(path)
    ip, ix, vv = _sorted_rows(indptr, indices, values)
    kw = dict(zip(["partsize_t", "partsize_c", "shortsize", "density", "window", "wide",
                   "tc_min_util", "sptc_min_util", "sptc_threshold"], args))
    dev = _compare(ip, ix, vv, cuda, mode=mode, **kw)
    if mode == "compat" and np.array_equal(ix, np.asarray(indices, np.int32)):
        _same(dev, ref)


CASES = {
    "chung_lu": lambda: graphs.chung_lu(n=4096),
    "sbm": lambda: graphs.sbm_powerlaw(n=6000, avg_degree=30, communities=60, seed=4),
    "route_mix": lambda: graphs.route_mix(n=2048, target_nnz=120_000),
    "batched": lambda: graphs.batched(num_graphs=30, seed=3),
    "ragged_dup": lambda: graphs.random_csr(500, 300, 0.05, seed=2, dup=True, empty_rows=0.4),
}


@pytest.mark.parametrize("name", list(CASES))
@pytest.mark.parametrize("mode", ["compat", "exact"])
@pytest.mark.parametrize("kw", [dict(), dict(density=4), dict(density=2, tc_min_util=0.3),
                                dict(partsize_t=3, partsize_c=5, shortsize=2),
                                dict(skip_tc=True), dict(skip_sptc=True), dict(unit_min_nnz=5),
                                dict(window=8), dict(window=5, density=3)],
                         ids=["default", "d4", "d2u03", "parts", "skip_tc", "skip_sptc", "umin5",
                              "w8", "w5"])
def test_graphs(cuda, name, mode, kw):
    g = CASES[name]()
    ip, ix, vv = _sorted_rows(g.indptr, g.indices, g.values)
    _compare(ip, ix, vv, cuda, mode=mode, **kw)


@pytest.mark.parametrize("mode", ["compat", "exact"])
def test_hub_windows_beyond_shared_memory(cuda, mode):
    """Windows of up to ~40k entries run in the global scratch slices."""
    g = graphs.random_csr(64, 5000, 0.5, seed=7, dup=True)
    ip, ix, vv = _sorted_rows(g.indptr, g.indices, g.values)
    assert np.diff(ip[::16]).max() > 1024
    _compare(ip, ix, vv, cuda, mode=mode, density=4)


def test_empty_inputs(cuda):
    for n_rows, n_cols, dens in ((1, 1, 0.0), (40, 7, 0.0), (1, 300, 0.5), (17, 1, 0.9)):
        g = graphs.random_csr(n_rows, n_cols, dens, seed=3)
        ip, ix, vv = _sorted_rows(g.indptr, g.indices, g.values)
        for mode in ("compat", "exact"):
            _compare(ip, ix, vv, cuda, mode=mode)


@pytest.mark.parametrize("mode", ["compat", "exact"])
def test_route_mix_full_size(cuda, mode):
    """The route-mix stress matrix at its full size (65,536 rows, ~3.2M
    entries), where the reference's router is pinned bit for bit."""
    g = graphs.route_mix(n=65_536, target_nnz=3_200_000, seed=3)
    ip, ix, vv = _sorted_rows(g.indptr, g.indices, g.values)
    _compare(ip, ix, vv, cuda, mode=mode)


def test_headline_graph_full_size(cuda):
    """The 200k-node SBM of the benchmark (10.2M entries)."""
    g, _ = graphs.make_workload("large_routed")
    ip, ix, vv = _sorted_rows(g.indptr, g.indices, g.values)
    dev = _compare(ip, ix, vv, cuda, mode="compat")
    assert dev[-1] > 0


def test_refusals(cuda):
    g = graphs.random_csr(40, 30, 0.2, seed=1)
    ip, ix, vv = _sorted_rows(g.indptr, g.indices, g.values)
    bad = ix.copy()
    bad[3] = -2
    with pytest.raises(RuntimeError, match=">= 0"):
        trspmm.route_device(ip, bad, vv)
    with pytest.raises(RuntimeError, match="window"):
        trspmm.route_device(ip, ix, vv, window=17)
    with pytest.raises(RuntimeError, match="partsize"):
        trspmm.route_device(ip, ix, vv, partsize_c=0)


@pytest.mark.parametrize("mode", ["compat", "exact"])
def test_device_resident_tables(cuda, mode):
    """out="torch": the tables as CUDA tensors (never copied to the host by
    the router) equal the host router's; the raw C call refuses device
    addresses for a host-built route."""
    g = CASES["sbm"]()
    ip, ix, vv = _sorted_rows(g.indptr, g.indices, g.values)
    host = trspmm.route(ip, ix, vv, mode=mode, unit_min_nnz=2, skip_tc=False)
    dev = trspmm.route_device(ip, ix, vv, mode=mode, unit_min_nnz=2, skip_tc=False, out="torch")
    assert all(t.is_cuda for t in dev[:29])
    _same([t.cpu().numpy() for t in dev[:29]], host)
    import ctypes
    from trspmm.core import _params, _vp
    L = trspmm.lib()
    h = ctypes.c_void_p()
    prm = _params(mode=mode)
    assert L.tr_route_build(_vp(ip), _vp(ix), _vp(vv), len(ip) - 1, ctypes.byref(prm),
                            ctypes.byref(h)) == 0
    data, n = ctypes.c_void_p(), ctypes.c_int64()
    TR_ERR_UNSUPPORTED = 5
    assert L.tr_route_table_device(h, 3, ctypes.byref(data), ctypes.byref(n)) == TR_ERR_UNSUPPORTED
    L.tr_route_free(h)
