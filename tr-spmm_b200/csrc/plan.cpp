// Plan construction: reference route tables -> the fused kernel's layout.
//
// Semantics of the tables follow the reference's kernels:
//  * dense TC sub-blocks (16 rows x 8 columns): bit (r*8 + k) of binary_lo
//    for rows 0-7 / binary_hi for rows 8-15, value index = rank of the bit
//    (popcount below it, binary_hi ranks after all of binary_lo), rows from
//    t_window_row (TR-source/SpMM/mGCNkernel_online.cu:106-204);
//  * packed 2:4 tiles: per row group g and chunk c, one half2 word for row g
//    and one for row g+8, positions from the 4-bit meta nibble
//    (TR-source/Block/block_online.cpp:797-841);
//  * CUDA parts: c_row / c_row_offset / c_column / c_value, long and short
//    alike (TR-source/SpMM/spmm_utils/compute.h:27-88, :176-240).
// Every index is range-checked here so the kernels can trust the plan.
#include "plan.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <numeric>

#include "common.cuh"

namespace trs {
namespace {

inline int a_index(int n, int k) { return (n / 8) * 128 + (k / 8) * 64 + (n % 8) * 8 + (k % 8); }

inline uint16_t f2h(float f) {
  _Float16 h = (_Float16)f;
  uint16_t b;
  std::memcpy(&b, &h, 2);
  return b;
}

// Per-window staging before flattening.
struct WinTiles {
  std::vector<int32_t> col;        // 16 per tile
  std::vector<uint16_t> a;         // 256 per tile
  int n = 0;
  void add_empty() {
    col.insert(col.end(), 16, -1);
    a.insert(a.end(), 256, 0);
    n++;
  }
};

void finish(HostPlan& hp, std::vector<WinTiles>& tc, std::vector<WinTiles>& sp,
            const std::vector<std::vector<std::pair<int32_t, std::pair<int32_t, uint16_t>>>>& res) {
  const int W = hp.n_windows;
  hp.win_tile.assign(1, 0);
  hp.win_split.resize(W);
  hp.tile_col.clear();
  hp.tile_a.clear();
  for (int w = 0; w < W; ++w) {
    hp.tile_col.insert(hp.tile_col.end(), tc[w].col.begin(), tc[w].col.end());
    hp.tile_a.insert(hp.tile_a.end(), tc[w].a.begin(), tc[w].a.end());
    hp.win_split[w] = hp.win_tile.back() + tc[w].n;
    hp.tile_col.insert(hp.tile_col.end(), sp[w].col.begin(), sp[w].col.end());
    hp.tile_a.insert(hp.tile_a.end(), sp[w].a.begin(), sp[w].a.end());
    hp.win_tile.push_back(hp.win_split[w] + sp[w].n);
    hp.tc_tiles += tc[w].n;
    hp.sptc_tiles += sp[w].n;
  }
  // residual CSR over padded rows, entries of a row in table order
  const int64_t rows = (int64_t)W * 16;
  hp.res_ptr.assign(rows + 1, 0);
  for (auto& r : res)
    for (auto& e : r) hp.res_ptr[e.first + 1]++;
  for (int64_t i = 0; i < rows; ++i) hp.res_ptr[i + 1] += hp.res_ptr[i];
  hp.res_col.resize(hp.res_ptr[rows]);
  hp.res_val.resize(hp.res_ptr[rows]);
  std::vector<int32_t> fill(hp.res_ptr.begin(), hp.res_ptr.end() - 1);
  for (auto& r : res)
    for (auto& e : r) {
      const int32_t at = fill[e.first]++;
      hp.res_col[at] = e.second.first;
      hp.res_val[at] = e.second.second;
    }
  // launch order: heaviest windows first (cost ~ gathered rows)
  std::vector<int64_t> cost(W);
  for (int w = 0; w < W; ++w)
    cost[w] = (int64_t)(hp.win_tile[w + 1] - hp.win_tile[w]) * 16 +
              (hp.res_ptr[(int64_t)(w + 1) * 16] - hp.res_ptr[(int64_t)w * 16]);
  hp.win_order.resize(W);
  std::iota(hp.win_order.begin(), hp.win_order.end(), 0);
  std::stable_sort(hp.win_order.begin(), hp.win_order.end(),
                   [&](int a, int b) { return cost[a] > cost[b]; });
  int64_t nnz = (int64_t)hp.res_col.size();
  for (uint16_t v : hp.tile_a) nnz += v != 0;
  hp.nnz = nnz;
}

bool in_range(int64_t v, int64_t lo, int64_t hi) { return v >= lo && v < hi; }

// Decode packed 2:4 tiles (block_online.cpp:797-841) into dense tiles.
int add_packed_tiles(const int32_t* tile_column, int64_t n_tile_column, const uint32_t* packed_a,
                     int64_t n_packed_a, const uint32_t* packed_meta, int64_t n_packed_meta,
                     const int32_t* wto, int64_t n_wto, int32_t n_cols, int W,
                     std::vector<WinTiles>& sp, std::string& err) {
  if (n_wto == 0) return TR_OK;
  const int64_t tiles = n_tile_column / 16;
  if (n_tile_column % 16 || n_packed_a != tiles * 64 || n_packed_meta != tiles * 8) {
    err = "packed SPTC tile arrays have inconsistent sizes";
    return TR_ERR_ARG;
  }
  if (n_wto - 1 > W) { err = "s_window_tile_offset has more windows than the matrix"; return TR_ERR_ARG; }
  if (wto[0] != 0 || wto[n_wto - 1] != tiles) {
    err = "s_window_tile_offset must start at 0 and end at the tile count";
    return TR_ERR_ARG;
  }
  for (int64_t w = 0; w + 1 < n_wto; ++w) {
    if (wto[w + 1] < wto[w]) { err = "s_window_tile_offset must be non-decreasing"; return TR_ERR_ARG; }
    for (int64_t t = wto[w]; t < wto[w + 1]; ++t) {
      WinTiles& wt = sp[w];
      const size_t cbase = wt.col.size(), abase = wt.a.size();
      wt.add_empty();
      for (int k = 0; k < 16; ++k) {
        const int32_t c = tile_column[t * 16 + k];
        if (c < -1 || c >= n_cols) { err = "s_tile_column out of range"; return TR_ERR_ARG; }
        wt.col[cbase + k] = c;
      }
      for (int g = 0; g < 8; ++g) {
        const uint32_t meta = packed_meta[t * 8 + g];
        for (int ch = 0; ch < 4; ++ch)
          for (int hsel = 0; hsel < 2; ++hsel) {
            const uint32_t word = packed_a[((t * 8 + g) * 4 + ch) * 2 + hsel];
            const uint32_t nib = (meta >> (16 * hsel + 4 * ch)) & 0xFu;
            const int row = g + 8 * hsel;
            const int p[2] = {(int)(nib & 3u), (int)((nib >> 2) & 3u)};
            for (int s = 0; s < 2; ++s) {
              const uint16_t bits = (uint16_t)(word >> (16 * s));
              if ((bits & 0x7FFFu) == 0) continue;     // padding (+-0)
              const int k = ch * 4 + p[s];
              if (wt.col[cbase + k] < 0) { err = "SPTC value in a padded column"; return TR_ERR_ARG; }
              wt.a[abase + a_index(row, k)] = bits;
            }
          }
      }
    }
  }
  return TR_OK;
}

}  // namespace

int plan_from_tables(const tr_tables& t, int32_t n_rows, int32_t n_cols, int32_t window,
                     HostPlan& hp, std::string& err) {
  if (window != 16) { err = "routed plans need window == 16"; return TR_ERR_UNSUPPORTED; }
  if (n_rows < 0 || n_cols < 0) { err = "negative matrix shape"; return TR_ERR_ARG; }
  hp = HostPlan();
  hp.n_rows = n_rows;
  hp.n_cols = n_cols;
  hp.n_windows = (n_rows + 15) / 16;
  const int W = hp.n_windows;
  std::vector<WinTiles> tc(W), sp(W);
  std::vector<std::vector<std::pair<int32_t, std::pair<int32_t, uint16_t>>>> res(1);

  // ---- dense TC parts -------------------------------------------------------
  if (t.n_t_row_offset > 1) {
    const int64_t parts = t.n_t_row_offset - 1;
    if (t.n_t_window_row < parts) { err = "t_window_row shorter than the part count"; return TR_ERR_ARG; }
    const int64_t subs = t.t_row_offset[parts];
    if (t.t_row_offset[0] != 0 || subs * 8 > t.n_t_column || subs * 2 > t.n_t_binary ||
        t.n_t_block_offset < subs + 1) {
      err = "TC tables have inconsistent sizes";
      return TR_ERR_ARG;
    }
    // collect the sub-blocks of each window in table order
    std::vector<std::vector<int64_t>> win_subs(W);
    for (int64_t p = 0; p < parts; ++p) {
      const int32_t wr = t.t_window_row[p];
      if (wr < 0 || wr % 16 != 0 || wr / 16 >= W) { err = "t_window_row out of range"; return TR_ERR_ARG; }
      if (t.t_row_offset[p + 1] < t.t_row_offset[p]) { err = "t_row_offset must be non-decreasing"; return TR_ERR_ARG; }
      for (int64_t s = t.t_row_offset[p]; s < t.t_row_offset[p + 1]; ++s) win_subs[wr / 16].push_back(s);
    }
    for (int w = 0; w < W; ++w) {
      auto& L = win_subs[w];
      for (size_t i = 0; i < L.size(); i += 2) {
        WinTiles& wt = tc[w];
        const size_t cbase = wt.col.size(), abase = wt.a.size();
        wt.add_empty();
        for (int half = 0; half < 2 && i + half < L.size(); ++half) {
          const int64_t s = L[i + half];
          const int64_t voff = t.t_block_offset[s];
          const int64_t vend = t.t_block_offset[s + 1];
          if (voff < 0 || vend < voff || vend > t.n_t_value) { err = "t_block_offset out of range"; return TR_ERR_ARG; }
          for (int k = 0; k < 8; ++k) {
            const int32_t c = t.t_column[s * 8 + k];
            if (c < -1 || c >= n_cols) { err = "t_column out of range"; return TR_ERR_ARG; }
            wt.col[cbase + half * 8 + k] = c;
          }
          const uint64_t lo = (uint64_t)t.t_binary[2 * s], hi = (uint64_t)t.t_binary[2 * s + 1];
          int rank = 0;
          for (int hsel = 0; hsel < 2; ++hsel) {
            const uint64_t word = hsel ? hi : lo;
            for (int bit = 0; bit < 64; ++bit) {
              if (!((word >> bit) & 1u)) continue;
              const int row = hsel * 8 + bit / 8, k = half * 8 + bit % 8;
              if (voff + rank >= vend) { err = "TC bitmap has more bits than values"; return TR_ERR_ARG; }
              if (wt.col[cbase + k] < 0) { err = "TC bit set in a padded column"; return TR_ERR_ARG; }
              wt.a[abase + a_index(row, k)] = t.t_value[voff + rank];
              rank++;
            }
          }
        }
      }
    }
  }

  // ---- SPTC packed tiles ----------------------------------------------------
  int rc = add_packed_tiles(t.s_tile_column, t.n_s_tile_column, t.s_packed_a, t.n_s_packed_a,
                            t.s_packed_meta, t.n_s_packed_meta, t.s_window_tile_offset,
                            t.n_s_window_tile_offset, n_cols, W, sp, err);
  if (rc) return rc;

  // ---- CUDA parts (long then short) -----------------------------------------
  auto& R = res[0];
  auto add_parts = [&](const int32_t* off, int64_t n_off, const int32_t* row, int64_t n_row,
                       const int32_t* col, int64_t n_col, const uint16_t* val, int64_t n_val) -> int {
    if (n_off <= 1) return TR_OK;
    const int64_t parts = n_off - 1;
    if (n_row < parts || off[0] != 0 || off[parts] > n_col || off[parts] > n_val) {
      err = "CUDA part tables have inconsistent sizes";
      return TR_ERR_ARG;
    }
    for (int64_t p = 0; p < parts; ++p) {
      if (off[p + 1] < off[p]) { err = "c_row_offset must be non-decreasing"; return TR_ERR_ARG; }
      if (!in_range(row[p], 0, n_rows)) { err = "c_row out of range"; return TR_ERR_ARG; }
      for (int64_t e = off[p]; e < off[p + 1]; ++e) {
        if (!in_range(col[e], 0, n_cols)) { err = "c_column out of range"; return TR_ERR_ARG; }
        R.push_back({row[p], {col[e], val[e]}});
      }
    }
    return TR_OK;
  };
  rc = add_parts(t.c_row_offset, t.n_c_row_offset, t.c_row, t.n_c_row, t.c_column, t.n_c_column,
                 t.c_value, t.n_c_value);
  if (rc) return rc;
  rc = add_parts(t.cs_row_offset, t.n_cs_row_offset, t.cs_row, t.n_cs_row, t.cs_column,
                 t.n_cs_column, t.cs_value, t.n_cs_value);
  if (rc) return rc;
  finish(hp, tc, sp, res);
  return TR_OK;
}

int plan_from_groups(const int32_t* s_column, const float* s_value, const int8_t* s_pos,
                     int64_t groups, const int32_t* s_window, const int32_t* s_offsets,
                     int64_t n_offsets, int32_t window, int32_t n_rows, int32_t n_cols,
                     HostPlan& hp, std::string& err) {
  if (window != 16) { err = "routed plans need window == 16"; return TR_ERR_UNSUPPORTED; }
  hp = HostPlan();
  hp.n_rows = n_rows;
  hp.n_cols = n_cols;
  hp.n_windows = (n_rows + 15) / 16;
  const int W = hp.n_windows;
  std::vector<int32_t> gwin(groups);
  if (s_window) {
    for (int64_t g = 0; g < groups; ++g) gwin[g] = s_window[g];
  } else {
    if (n_offsets < 1 || s_offsets[0] != 0 || s_offsets[n_offsets - 1] != groups) {
      err = "s_offsets must start at 0 and end at the group count";
      return TR_ERR_ARG;
    }
    for (int64_t w = 0; w + 1 < n_offsets; ++w) {
      if (s_offsets[w + 1] < s_offsets[w]) { err = "s_offsets must be non-decreasing"; return TR_ERR_ARG; }
      for (int64_t g = s_offsets[w]; g < s_offsets[w + 1]; ++g) gwin[g] = (int32_t)w;
    }
  }
  std::vector<WinTiles> tc(W), sp(W);
  // groups of one window, four per tile, in table order
  std::vector<std::vector<int64_t>> wg(W);
  for (int64_t g = 0; g < groups; ++g) {
    if (!in_range(gwin[g], 0, W)) {
      // rows of such a group are beyond the matrix: the reference kernel
      // skips them (global_row >= mOri), so do we
      continue;
    }
    wg[gwin[g]].push_back(g);
  }
  for (int w = 0; w < W; ++w) {
    for (size_t i = 0; i < wg[w].size(); i += 4) {
      WinTiles& wt = sp[w];
      const size_t cbase = wt.col.size(), abase = wt.a.size();
      wt.add_empty();
      for (int ch = 0; ch < 4 && i + ch < wg[w].size(); ++ch) {
        const int64_t g = wg[w][i + ch];
        for (int p = 0; p < 4; ++p) {
          const int32_t c = s_column[g * 4 + p];
          if (c < -1 || c >= n_cols) { err = "s_column out of range"; return TR_ERR_ARG; }
          wt.col[cbase + ch * 4 + p] = c;
        }
        for (int lr = 0; lr < 16; ++lr) {
          if ((int64_t)w * 16 + lr >= n_rows) continue;
          for (int s = 0; s < 2; ++s) {
            const int pos = s_pos[(g * 16 + lr) * 2 + s];
            if (pos < 0) continue;
            if (pos > 3 || wt.col[cbase + ch * 4 + pos] < 0) continue;  // kernel skips (col < 0)
            wt.a[abase + a_index(lr, ch * 4 + pos)] = f2h(s_value[(g * 16 + lr) * 2 + s]);
          }
        }
      }
    }
  }
  std::vector<std::vector<std::pair<int32_t, std::pair<int32_t, uint16_t>>>> res(1);
  finish(hp, tc, sp, res);
  return TR_OK;
}

int plan_upload(const HostPlan& hp, tr_plan** out) {
  const int W = hp.n_windows;
  const int64_t T = (int64_t)hp.tile_col.size() / 16;
  auto al = [](int64_t b) { return (b + 255) / 256 * 256; };
  const int64_t sz_win_tile = al((W + 1) * 4), sz_win_split = al(std::max(W, 1) * 4),
                sz_tile_col = al(std::max<int64_t>(T, 1) * 64),
                sz_tile_a = al(std::max<int64_t>(T, 1) * 512),
                sz_res_ptr = al(((int64_t)W * 16 + 1) * 4),
                sz_res_col = al(std::max<size_t>(hp.res_col.size(), 1) * 4),
                sz_res_val = al(std::max<size_t>(hp.res_val.size(), 1) * 2),
                sz_order = al(std::max(W, 1) * 4), sz_err = 256;
  const int64_t total = sz_win_tile + sz_win_split + sz_tile_col + sz_tile_a + sz_res_ptr +
                        sz_res_col + sz_res_val + sz_order + sz_err;
  tr_plan* p = new tr_plan();
  cudaGetDevice(&p->device);
  cudaError_t e = cudaMalloc(&p->block, total);
  if (e != cudaSuccess) { delete p; return cuda_fail(e, "cudaMalloc(plan)"); }
  p->bytes = total;
  char* base = (char*)p->block;
  int64_t off = 0;
  auto put = [&](const void* src, int64_t nbytes, int64_t sz) -> char* {
    char* dst = base + off;
    off += sz;
    if (nbytes > 0) cudaMemcpy(dst, src, nbytes, cudaMemcpyHostToDevice);
    return dst;
  };
  PlanView& v = p->view;
  v.n_rows = hp.n_rows;
  v.n_cols = hp.n_cols;
  v.n_windows = W;
  v.win_tile = (int32_t*)put(hp.win_tile.data(), (W + 1) * 4, sz_win_tile);
  v.win_split = (int32_t*)put(hp.win_split.data(), W * 4, sz_win_split);
  v.tile_col = (int32_t*)put(hp.tile_col.data(), T * 64, sz_tile_col);
  v.tile_a = (uint16_t*)put(hp.tile_a.data(), T * 512, sz_tile_a);
  v.res_ptr = (int32_t*)put(hp.res_ptr.data(), ((int64_t)W * 16 + 1) * 4, sz_res_ptr);
  v.res_col = (int32_t*)put(hp.res_col.data(), hp.res_col.size() * 4, sz_res_col);
  v.res_val = (uint16_t*)put(hp.res_val.data(), hp.res_val.size() * 2, sz_res_val);
  v.win_order = (int32_t*)put(hp.win_order.data(), W * 4, sz_order);
  v.err = (int*)(base + off);
  cudaMemset(v.err, 0, sz_err);
  e = cudaDeviceSynchronize();
  if (e != cudaSuccess) { cudaFree(p->block); delete p; return cuda_fail(e, "plan upload"); }
  p->info.n_rows = hp.n_rows;
  p->info.n_cols = hp.n_cols;
  p->info.n_windows = W;
  p->info.nnz = hp.nnz;
  p->info.tc_tiles = hp.tc_tiles;
  p->info.sptc_tiles = hp.sptc_tiles;
  p->info.residual_nnz = (int64_t)hp.res_col.size();
  p->info.device_bytes = total;
  *out = p;
  return TR_OK;
}

}  // namespace trs
