// Device router: the dense-TC funnel (route_gpu.cu).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

namespace trs {

struct RouteGpuParams {
  int32_t window = 16;       // rows per window (fixed at 16 here)
  int32_t density = 8;       // TC column threshold
  float tc_min_util = 0.f;
  int32_t partsize_t = 32;
  int32_t skip_tc = 0;
};

// The TC tables of the reference router (TR-source/Block/block_online.cpp
// :844-870 items 0-4 and 6; t_atomic excluded) plus each value's CSR entry.
struct TcTables {
  std::vector<int32_t> t_row_offset{0}, t_block_offset{0}, t_column;
  std::vector<float> t_value;
  std::vector<int32_t> t_window_row;
  std::vector<int64_t> t_binary;
  std::vector<int32_t> t_edge;
};

// Device CSR in (rows sorted by column), host tables out.
int route_tc_gpu(const int32_t* d_indptr, const int32_t* d_indices, const float* d_values,
                 int32_t n_rows, const RouteGpuParams& p, TcTables& out, std::string& err);

// The same funnel without any allocation: scratch in a static device array,
// tables into caller buffers (see tr_route_tc_device_noalloc).
int route_tc_gpu_noalloc(const int32_t* d_indptr, const int32_t* d_indices, const float* d_values,
                         int32_t n_rows, const RouteGpuParams& p, int32_t* t_column,
                         int64_t* t_binary, float* t_value, int32_t* t_block_offset,
                         int64_t cap_sub, int64_t cap_val, int64_t* n_sub_out,
                         int64_t* n_val_out, cudaStream_t stream);

}  // namespace trs
