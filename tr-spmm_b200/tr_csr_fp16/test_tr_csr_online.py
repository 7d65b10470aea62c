"""Routed forward driver (mirrors spmm/tr_csr_fp16/test_tr_csr_online.py).

``kernel_tcu_sptc_cuda_online`` dispatches on the reference's switches
LIBRA_SPTC_KERNEL / LIBRA_SPTC_PARALLEL (test_tr_csr_online.py:83-181) and
calls the drop-in ``Libra6SpMMOnline`` operators; ``test_tcu_sptc_cuda_online``
builds the dataset, runs the forward and prints the timings.
"""
import os

import torch

import Libra6SpMMOnline
from tr_csr_fp16.mdataset2_online import GCN_dataset_tcu_sptc_cuda_online


# The nine SPTC tensors of the parallel operator, in argument order; the
# offset tables keep their length when the route is switched off (every
# window then owns no group and no tile), the others become empty.
_SPTC_NAMES = ("s_columnTensor", "s_valueTensor", "s_posTensor", "s_offsetTensor",
               "s_tile_windowTensor", "s_tile_columnTensor", "s_packed_aTensor",
               "s_packed_metaTensor", "s_window_tile_offsetTensor")
_SPTC_OFFSETS = {"s_offsetTensor", "s_window_tile_offsetTensor"}


def _zero_sptc_like(inputInfo):
    """The SPTC arguments of a run without the SPTC route."""
    return tuple(torch.zeros_like(t) if n in _SPTC_OFFSETS else t.new_empty((0,) + tuple(t.shape[1:]))
                 for n, t in ((n, getattr(inputInfo, n)) for n in _SPTC_NAMES))


def _parallel_call(inputInfo, epoches, sptc):
    (s_column, s_value, s_pos, s_offsets, s_tile_window, s_tile_column, s_packed_a,
     s_packed_meta, s_window_tile_offset) = sptc
    return Libra6SpMMOnline.forward_fp16_tcu_cuda_sptc_mma_parallel_online(
        inputInfo.t_rowNew_offsetTensor, inputInfo.t_blockTensor, inputInfo.t_columnTensor,
        inputInfo.t_valueTensor, inputInfo.t_window_rowTensor, inputInfo.t_atomicTensor,
        inputInfo.t_binaryTensor,
        inputInfo.c_row_offsetTensor, inputInfo.c_rowTensor, inputInfo.c_atomicTensor,
        inputInfo.c_colTensor, inputInfo.c_valueTensor,
        inputInfo.c_row_offsetTensor_short, inputInfo.c_rowTensor_short,
        inputInfo.c_atomicTensor_short, inputInfo.c_colTensor_short,
        inputInfo.c_valueTensor_short,
        s_column, s_value, s_pos, s_offsets, s_tile_window, s_tile_column, s_packed_a,
        s_packed_meta, s_window_tile_offset,
        inputInfo.x,
        inputInfo.parts_t, inputInfo.parts_c, inputInfo.partsize_c, inputInfo.parts_c_short,
        inputInfo.window, inputInfo.x.size(1), inputInfo.num_nodes_ori, inputInfo.num_nodes_dst,
        epoches)


def _full_sptc(inputInfo):
    return tuple(getattr(inputInfo, n) for n in _SPTC_NAMES)


def _base_tcu_cuda_profile_online(inputInfo, epoches):
    x_base, ms_base, ms_tc, ms_cuda_long, ms_cuda_short, _ = _parallel_call(
        inputInfo, epoches, _zero_sptc_like(inputInfo))
    return x_base, ms_base, ms_tc, ms_cuda_long, ms_cuda_short


def kernel_tcu_sptc_cuda_online(inputInfo, epoches):
    sptc_kernel = os.environ.get("LIBRA_SPTC_KERNEL", "mma").lower()
    sptc_parallel = os.environ.get("LIBRA_SPTC_PARALLEL", "1") == "1"
    if sptc_parallel and sptc_kernel != "cuda":
        x, ms, ms_tc, ms_cl, ms_cs, ms_s = _parallel_call(inputInfo, epoches, _full_sptc(inputInfo))
        inputInfo.profile_times = {"base_tc_cuda": ms, "tc": ms_tc, "cuda_long": ms_cl,
                                   "cuda_short": ms_cs, "sptc": ms_s}
        return x, ms, torch.tensor(0.0), "parallel_mma"

    x_base, ms_base, ms_tc, ms_cl, ms_cs = _base_tcu_cuda_profile_online(inputInfo, epoches)
    if sptc_kernel == "cuda":
        x_sptc, ms_sptc = Libra6SpMMOnline.forward_fp16_sptc_online(
            inputInfo.s_columnTensor, inputInfo.s_valueTensor, inputInfo.s_posTensor,
            inputInfo.s_windowTensor, inputInfo.x, inputInfo.window, inputInfo.x.size(1),
            inputInfo.num_nodes_ori, inputInfo.num_nodes_dst, epoches)
    else:
        sptc_kernel = "mma_packed"
        x_sptc, ms_sptc = Libra6SpMMOnline.forward_fp16_sptc_mma_packed_online(
            inputInfo.s_tile_columnTensor, inputInfo.s_packed_aTensor,
            inputInfo.s_packed_metaTensor, inputInfo.s_window_tile_offsetTensor, inputInfo.x,
            inputInfo.window, inputInfo.x.size(1), inputInfo.num_nodes_ori,
            inputInfo.num_nodes_dst, epoches)
    inputInfo.profile_times = {"base_tc_cuda": ms_base, "tc": ms_tc, "cuda_long": ms_cl,
                               "cuda_short": ms_cs, "sptc": ms_sptc}
    return x_base + x_sptc, ms_base, ms_sptc, sptc_kernel


def test_tcu_sptc_cuda_online(data, epoches, dimN, density, partsize_t, partsize_c, shortsize,
                              data_path, window, wide, tc_min_util=0.0, sptc_min_util=0.50,
                              sptc_threshold=12):
    inputInfo = GCN_dataset_tcu_sptc_cuda_online(
        data, dimN, density, partsize_t, partsize_c, shortsize, data_path, window, wide,
        tc_min_util, sptc_min_util, sptc_threshold)
    _, ms_base, ms_sptc, sptc_kernel = kernel_tcu_sptc_cuda_online(inputInfo, epoches)
    execution_time = round(ms_base.item() + ms_sptc.item(), 4)
    name = data if isinstance(data, str) else "graph"
    print(f"{dimN}-{name} online-tcu-sptc-cuda-{density}-{execution_time}")
    if sptc_kernel == "parallel_mma":
        print(f"parallel_tc_cuda_sptc_mma={round(ms_base.item(), 4)}")
    else:
        print(f"base_tc_cuda={round(ms_base.item(), 4)}, sptc_{sptc_kernel}={round(ms_sptc.item(), 4)}")
    prof = getattr(inputInfo, "profile_times", None)
    if prof is not None:
        cuda_ms = max(prof["cuda_long"].item(), prof["cuda_short"].item())
        print(f"kernel_breakdown: tc={round(prof['tc'].item(), 4)}, cuda={round(cuda_ms, 4)}, "
              f"cuda_long={round(prof['cuda_long'].item(), 4)}, "
              f"cuda_short={round(prof['cuda_short'].item(), 4)}, sptc={round(prof['sptc'].item(), 4)}")
    return execution_time, inputInfo.duration
