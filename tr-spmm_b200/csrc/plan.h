// Routed operand laid out for the fused sm_100a kernel.
//
// HBM layout (one allocation, window-major, 256-byte aligned sections):
//   win_tile[W+1]    tensor-core tiles of window w: [win_tile[w], win_tile[w+1])
//   win_split[W]     first 2:4 tile of window w; tiles before it come from the
//                    dense TC route, tiles from it on from the SPTC route
//   tile_col[T*16]   column of B gathered for each K slot of a tile (-1: none)
//   tile_a[T*256]    16x16 FP16 A tile, stored in the tcgen05 K-major,
//                    no-swizzle core-matrix order (N = window row, K = slot):
//                    element (n, k) at (n/8)*128 + (k/8)*64 + (n%8)*8 + k%8
//   res_ptr[W*16+1]  CUDA-core residual as CSR over the padded rows
//   res_col[R], res_val[R] (FP16)
//   win_order[W]     windows in decreasing cost order (launch order)
//   err[4]           device error flags (bounded-wait timeouts)
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/trspmm.h"

namespace trs {

struct PlanView {
  int32_t n_rows, n_cols, n_windows;
  const int32_t* win_tile;
  const int32_t* win_split;
  const int32_t* tile_col;
  const uint16_t* tile_a;
  const int32_t* res_ptr;
  const int32_t* res_col;
  const uint16_t* res_val;
  const int32_t* win_order;
  int* err;
};

struct HostPlan {
  int32_t n_rows = 0, n_cols = 0, n_windows = 0;
  std::vector<int32_t> win_tile{0}, win_split, tile_col;
  std::vector<uint16_t> tile_a;
  std::vector<int32_t> res_ptr, res_col;
  std::vector<uint16_t> res_val;
  std::vector<int32_t> win_order;
  int64_t tc_tiles = 0, sptc_tiles = 0, nnz = 0;
};

}  // namespace trs

struct tr_plan {
  trs::PlanView view;
  void* block = nullptr;        // the single device allocation
  int64_t bytes = 0;
  int device = 0;
  tr_plan_info info{};
};

namespace trs {

// Host construction from the reference's tables (validates every index).
int plan_from_tables(const tr_tables& t, int32_t n_rows, int32_t n_cols, int32_t window,
                     HostPlan& hp, std::string& err);
// SPTC-only plans from the unpacked group tables (s_column/s_value/s_pos),
// windows given either per group (s_window) or as offsets (s_offsets).
int plan_from_groups(const int32_t* s_column, const float* s_value, const int8_t* s_pos,
                     int64_t groups, const int32_t* s_window, const int32_t* s_offsets,
                     int64_t n_offsets, int32_t window, int32_t n_rows, int32_t n_cols,
                     HostPlan& hp, std::string& err);
int plan_upload(const HostPlan& hp, tr_plan** out);

}  // namespace trs
