// Routed operand laid out for the sm_100a kernels.
//
// HBM layout (one allocation, window-major, 256-byte aligned sections):
//   win_tile[W+1]    tensor-core tiles of window w: [win_tile[w], win_tile[w+1])
//   win_split[W]     first 2:4 tile of window w; tiles before it come from the
//                    dense TC route
//   win_prom[W]      first promoted tile of window w: tiles from it on hold
//                    residual columns that the plan moved onto the tensor
//                    cores (columns gathered once, used by several rows)
//   tile_col[T*16]   column of B gathered for each K slot of a tile (-1: none)
//   tile_a[T*256]    16x16 FP16 A tile, stored in the tcgen05 K-major,
//                    no-swizzle core-matrix order (N = window row, K = slot):
//                    element (n, k) at (n/8)*128 + (k/8)*64 + (n%8)*8 + k%8
//   res_ptr[W*16+1]  CUDA-core residual as CSR over the padded rows
//   res_col[R], res_val[R] (FP16)
//   res_edge[R]      CSR entry of the source matrix behind each residual
//                    entry (-1: unknown), for the fused adjoint + SDDMM
//   win_order[W]     windows in decreasing cost order (launch order)
//   row_scale[W*16]  FP32 factor re-applied to each plan row in the epilogue
//                    (values are stored as FP16(v / row_scale))
//   row_out[W*16]    output row of each plan row (-1: padding); the identity
//                    unless the plan was built on reordered rows
//   val_slot[E]      for each CSR entry of the source matrix, its value slot:
//                    tile_a index (< T*256) or T*256 + residual index; -1 if
//                    the entry is not multiplied (compat-mode truncation)
//   edge_row[E]      plan row of each CSR entry (row scale of learnable values)
//   err[4]           device error flags (bounded-wait timeouts)
//
// Block layout (the block engine, opts.engine == TR_ENGINE_BLOCK): the plan's
// rows in blocks of 128 (eight windows); every distinct column a block
// touches is one K slot of a 16-column chunk, so each feature row of B is
// gathered once per block and multiplied by the tensor cores against all 128
// rows at once (tcgen05.mma M = 128 rows, N = K features, K = 16 slots):
//   blk_chunk[NB+1]  chunks of block b: [blk_chunk[b], blk_chunk[b+1]), a
//                    multiple of 8 (trailing chunks without entries pad it)
//   chunk_col[NC*16] row of B gathered into each slot of a chunk (-1: none)
//   chunk_ent[NC+1]  entries of chunk c: [chunk_ent[c], chunk_ent[c+1])
//   ent_pos[E]       byte offset of the entry in the chunk's 128x16 FP16 A
//                    tile (tcgen05 K-major, no swizzle: row m, slot k at
//                    (m/8)*256 + (k/8)*128 + (m%8)*16 + (k%8)*2)
//   ent_val[E]       FP16 value (FP16(v / row_scale) when row-scaled)
//   ent_src[E]       CSR entry of the caller's A behind the entry
//   blk_order[NB]    blocks in decreasing chunk count (launch order)
// row_scale / row_out cover NB*128 rows (n_windows = NB*8); the window
// sections are empty, and val_slot indexes ent_val.  On the device each
// entry is one 32-bit word, ent_pv[e] = ent_val[e] << 16 | ent_pos[e], and
// the device val_slot is 2e + 1 (the value's 16-bit half of that word).
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
  const int32_t* win_prom;
  const int32_t* tile_col;
  const uint16_t* tile_a;
  const int32_t* res_ptr;
  const int32_t* res_col;
  const uint16_t* res_val;
  const int32_t* res_edge;
  const int32_t* win_order;
  const float* row_scale;
  const int32_t* row_out;
  int* err;
  // block layout (n_blocks == 0 for window plans)
  int32_t n_blocks;
  const int32_t* blk_chunk;
  const int32_t* chunk_col;
  const int32_t* chunk_ent;
  const uint32_t* ent_pv;         // per entry: FP16 value bits << 16 | ent_pos
  const int32_t* ent_src;
  const int32_t* blk_order;
  // launch schedule of the block kernels (device only, made at upload for the
  // device's SM count): CTA c takes blocks cta_blk[cta_ptr[c] .. cta_ptr[c+1])
  int32_t n_sched;
  const int32_t* cta_ptr;
  const int32_t* cta_blk;
};

struct HostPlan {
  int32_t n_rows = 0, n_cols = 0, n_windows = 0;
  std::vector<int32_t> win_tile{0}, win_split, win_prom, tile_col;
  std::vector<uint16_t> tile_a;
  std::vector<int32_t> res_ptr, res_col;
  std::vector<uint16_t> res_val;
  std::vector<int32_t> res_edge;
  std::vector<int32_t> win_order;
  std::vector<float> row_scale;
  std::vector<int32_t> row_out;
  std::vector<int32_t> val_slot, edge_row;
  bool row_scaled = false, reordered = false;
  int64_t tc_tiles = 0, sptc_tiles = 0, prom_tiles = 0, nnz = 0;
  // block layout
  bool block = false;
  std::vector<int32_t> blk_chunk, chunk_col, chunk_ent, ent_src, blk_order;
  std::vector<uint16_t> ent_pos, ent_val;
};

// Rows per block of the block layout, K slots per chunk, and chunks per
// group (every block holds a whole number of groups).
constexpr int kBlkRows = 128;
constexpr int kChunkCols = 16;
constexpr int kChunkGroup = 8;

// A CSR matrix on its way through the builder; src[e] is the entry of the
// caller's A behind entry e.
struct Csr {
  int32_t n_rows = 0, n_cols = 0;
  std::vector<int32_t> ptr, idx;
  std::vector<float> val;
  std::vector<int32_t> src;
};

}  // namespace trs

struct tr_plan {
  trs::PlanView view;
  void* block = nullptr;        // the single device allocation
  int64_t bytes = 0;
  int device = 0;
  int64_t n_edges = 0;          // entries of the source CSR (val_slot / edge_row length)
  int32_t* val_slot = nullptr;
  int32_t* edge_row = nullptr;
  float* row_scale = nullptr;   // writable alias of view.row_scale
  uint16_t* tile_a = nullptr;   // writable aliases for re-valuing
  uint16_t* res_val = nullptr;
  int64_t n_tile_vals = 0;      // T*256
  bool row_scaled = false;
  bool blocked = false;         // block layout (the block engine)
  int32_t max_sched_blocks = 0; // most blocks any CTA of the block schedule takes
  int32_t k_tile = 0;           // block engine: features per tensor-core launch (0: 256)
  bool deterministic = false;   // window plans: the fused backward combines cut rows in order
  // Edge numbering.  Edges start numbered as A's CSR entries; after
  // tr_plan_renumber_edges, val_slot / edge_row / res_edge / ent_src use the
  // caller's numbering and edge_id[e] (own allocation) is the current number
  // of A's CSR entry e (the SDDMM over A's CSR writes through it).
  int32_t* edge_id = nullptr;
  // the kernels' entry stream map (res_edge of window plans, ent_src of
  // block plans) is the identity: the backward stores dval at the entry's
  // own position and reads no map
  bool res_edge_identity = false;
  tr_plan_info info{};
};

namespace trs {

struct RouteTables;

// Plan-shaping options of the native builder.
struct PlanOptions {
  bool row_scale = false;       // per-row FP32 scale, FP16(v / scale) stored
  int promote_min = 0;          // residual columns used by >= this many rows of a
                                // window become tensor-core tiles (0: never)
  int demote_below = 0;         // 2:4 tile columns with fewer entries than this
                                // go to the CUDA-core residual (0, 1: never)
};

// Host construction from the reference's tables (validates every index).
int plan_from_tables(const tr_tables& t, int32_t n_rows, int32_t n_cols, int32_t window,
                     HostPlan& hp, std::string& err);
// Construction from this library's route tables, which record the CSR entry
// behind every value; fills val_slot / edge_row over n_edges entries.
int plan_from_route(const RouteTables& T, int32_t n_rows, int32_t n_cols, int64_t n_edges,
                    const PlanOptions& opt, HostPlan& hp, std::string& err);
// SPTC-only plans from the unpacked group tables (s_column/s_value/s_pos),
// windows given either per group (s_window) or as offsets (s_offsets).
int plan_from_groups(const int32_t* s_column, const float* s_value, const int8_t* s_pos,
                     int64_t groups, const int32_t* s_window, const int32_t* s_offsets,
                     int64_t n_offsets, int32_t window, int32_t n_rows, int32_t n_cols,
                     HostPlan& hp, std::string& err);
int plan_upload(const HostPlan& hp, tr_plan** out);
// Block layout of a (transposed / reordered) CSR: fills hp's block arrays,
// row_scale / row_out (identity; the caller maps reordered rows), val_slot /
// edge_row over n_edges entries of the caller's A.
int plan_blocks(const Csr& a, bool row_scale, int64_t n_edges, HostPlan& hp, std::string& err);
// Native builder (builder.cpp): validate, transpose / reorder as asked, route, lay out.
int validate_csr(const int32_t* indptr, const int32_t* indices, int32_t n_rows, int32_t n_cols,
                 std::string& err);
int build_plan(const int32_t* indptr, const int32_t* indices, const float* values, int32_t n_rows,
               int32_t n_cols, const tr_route_params& params, const tr_plan_opts& opts,
               HostPlan& hp, std::string& err);
// The row order TR_REORDER_LABEL gives build_plan for A (or A^T), alone.
int label_order(const int32_t* indptr, const int32_t* indices, int32_t n_rows, int32_t n_cols,
                bool transpose_first, int32_t* order, std::string& err);

}  // namespace trs
