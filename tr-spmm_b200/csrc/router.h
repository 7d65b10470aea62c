// Host router: CSR -> the reference's route tables (see router.cpp).
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/trspmm.h"

namespace trs {

// The reference's 29 tables (TR-source/Block/block_online.cpp:844-870),
// FP32 values as the reference returns them.
struct RouteTables {
  std::vector<int32_t> t_row_offset{0}, t_block_offset{0}, t_column;
  std::vector<float> t_value;
  std::vector<int32_t> t_window_row, t_atomic;
  std::vector<int64_t> t_binary;
  std::vector<int32_t> c_row_offset{0}, c_row, c_atomic, c_column;
  std::vector<float> c_value;
  std::vector<int32_t> cs_row_offset{0}, cs_row, cs_atomic, cs_column;
  std::vector<float> cs_value;
  std::vector<int32_t> s_column;
  std::vector<uint8_t> s_mask;
  std::vector<float> s_value;
  std::vector<int8_t> s_pos;
  std::vector<int32_t> s_window, s_offsets{0};
  std::vector<int32_t> s_tile_window, s_tile_group, s_tile_column, s_packed_a, s_packed_meta;
  std::vector<int32_t> s_window_tile_offset{0};
  // Provenance of every table value: the CSR entry it came from (-1: padding).
  // Parallel to t_value, s_value, c_value and cs_value.
  std::vector<int32_t> t_edge, s_edge, c_edge, cs_edge;
  int window = 16;
  int64_t dropped = 0;     // entries the compat tables leave out
  double seconds = 0.0;
};

int build_route(const int32_t* indptr, const int32_t* indices, const float* values,
                int32_t n_rows, const tr_route_params& p, RouteTables& out, std::string& err);

}  // namespace trs
