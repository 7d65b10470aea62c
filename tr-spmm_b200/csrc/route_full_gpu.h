// Device router: every stage of the three-stage router (route_full_gpu.cu).
#pragma once
#include <cstdint>
#include <string>

#include "router.h"

namespace trs {

struct RouteFullParams {
  int32_t window = 16;        // rows per window, 1..16
  int32_t density = 8;        // TC column threshold
  float tc_min_util = 0.f;
  int32_t partsize_t = 32;
  int32_t partsize_c = 32;
  int32_t shortsize = 3;
  int32_t unit_min_nnz = 2;
  int32_t skip_tc = 0;
  int32_t skip_sptc = 0;
  int32_t mode = TR_ROUTE_COMPAT;
};

// Device pointers of the tables the filling launch writes; offsets (row,
// block, part, group and tile offsets) are prefix sums the host forms from
// the per-item counts (t_part_cnt, t_subcnt, c_cnt, cs_cnt) and the
// per-window counts.
struct FullTables {
  int32_t *t_part_cnt, *t_window_row, *t_atomic, *t_subcnt, *t_column, *t_edge;
  int64_t* t_binary;
  float* t_value;
  int32_t *s_window, *s_column, *s_edge, *s_tile_window, *s_tile_group, *s_tile_column,
      *s_packed_a, *s_packed_meta;
  uint8_t* s_mask;
  float* s_value;
  int8_t* s_pos;
  int32_t *c_cnt, *c_row, *c_atomic, *c_column, *c_edge;
  float* c_value;
  int32_t *cs_cnt, *cs_row, *cs_atomic, *cs_column, *cs_edge;
  float* cs_value;
};

// The router's 29 tables on the device, in the reference's return order
// (TR-source/Block/block_online.cpp:844-870), in one allocation the struct
// owns; plus each value's CSR entry (t_edge, s_edge, c_edge, cs_edge).
struct DeviceTables {
  void* block = nullptr;
  const void* ptr[29] = {};
  int64_t count[29] = {};      // items
  int elem[29] = {};           // bytes per item
  const int32_t *t_edge = nullptr, *s_edge = nullptr, *c_edge = nullptr, *cs_edge = nullptr;
  DeviceTables() = default;
  DeviceTables(const DeviceTables&) = delete;
  DeviceTables& operator=(const DeviceTables&) = delete;
  ~DeviceTables();
};

// Device CSR in (rows sorted by column), the router's 29 tables out on the
// device, equal item for item to build_route's for the same parameters.
// `host` receives the small tables the host forms anyway (the six offset
// tables), `dropped` and `seconds`; the others stay empty there.
int route_full_gpu(const int32_t* d_indptr, const int32_t* d_indices, const float* d_values,
                   int32_t n_rows, const RouteFullParams& p, DeviceTables& dev, RouteTables& host,
                   std::string& err);

}  // namespace trs
