// Plan construction: route tables -> the fused kernel's layout.
//
// Semantics of the tables follow the reference's kernels:
//  * dense TC sub-blocks (16 rows x 8 columns): bit (r*8 + k) of binary_lo
//    for rows 0-7 / binary_hi for rows 8-15, value index = rank of the bit
//    (popcount below it, binary_hi ranks after all of binary_lo), rows from
//    t_window_row (TR-source/SpMM/mGCNkernel_online.cu:106-204);
//  * 2:4 groups: per (group, local row) up to two (position, value) pairs
//    (TR-source/Block/block_online.cpp:663-702), or the packed tiles built
//    from them (:797-841);
//  * CUDA parts: c_row / c_row_offset / c_column / c_value, long and short
//    alike (TR-source/SpMM/spmm_utils/compute.h:27-88, :176-240).
// Every index is range-checked here so the kernels can trust the plan.
//
// Values are carried in FP32 with the CSR entry they came from (when the
// tables record it) until the plan is flattened: then an optional per-row
// scale s_r = max |v| over the row is taken in FP32, FP16(v / s_r) is stored
// and s_r is re-applied to the row in the kernel epilogue, so small GCN
// weights keep full FP16 precision.  The entry -> slot map lets a device
// kernel re-value the plan (learnable edge weights) without rebuilding it.
#include "plan.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <queue>
#include <atomic>
#include <cmath>
#include <cstring>
#include <numeric>
#include <thread>

#include "common.cuh"
#include "router.h"

namespace trs {
namespace {

inline int a_index(int n, int k) { return (n / 8) * 128 + (k / 8) * 64 + (n % 8) * 8 + (k % 8); }

// f(begin, end) over [0, n) on the host's threads (windows are independent).
template <class F>
void parallel_windows(int64_t n, F f) {
  int t = (int)std::max(1u, std::thread::hardware_concurrency());
  t = (int)std::min<int64_t>(t, std::max<int64_t>(1, n / 64));
  if (t <= 1) {
    f((int64_t)0, n);
    return;
  }
  std::vector<std::thread> pool;
  for (int k = 0; k < t; ++k) pool.emplace_back([&, k] { f(n * k / t, n * (k + 1) / t); });
  for (auto& th : pool) th.join();
}

inline uint16_t f2h(float f) {
  _Float16 h = (_Float16)f;
  uint16_t b;
  std::memcpy(&b, &h, 2);
  return b;
}
inline float h2f(uint16_t b) {
  _Float16 h;
  std::memcpy(&h, &b, 2);
  return (float)h;
}

// Per-window staging before flattening.
struct WinTiles {
  std::vector<int32_t> col;        // 16 per tile
  std::vector<float> a;            // 256 per tile (kernel operand order)
  std::vector<int32_t> edge;       // 256 per tile, -1 where no entry
  int n = 0;
  void add_empty() {
    col.insert(col.end(), 16, -1);
    a.insert(a.end(), 256, 0.f);
    edge.insert(edge.end(), 256, -1);
    n++;
  }
};

struct ResEntry {
  int32_t row, col;
  float val;
  int32_t edge;
};

struct Staging {
  std::vector<WinTiles> tc, sp, pr;   // dense TC, 2:4, promoted residual columns
  std::vector<ResEntry> res;
  explicit Staging(int W) : tc(W), sp(W), pr(W) {}
};

bool in_range(int64_t v, int64_t lo, int64_t hi) { return v >= lo && v < hi; }

// Window row of tile element i (inverse of a_index in n).
inline int elem_row(int i) { return (i / 128) * 8 + (i % 64) / 8; }

// Residual columns used by at least `min_rows` entries of a window move onto
// the tensor cores: 16 such columns per tile, each (row, column) once (a
// repeated entry stays in the residual).  Columns are taken in increasing
// order so the result does not depend on the residual's entry order.
// 2:4 tile columns holding fewer than `min_rows` entries of their window go
// back to the CUDA-core residual (a gathered feature row that serves one or
// two rows costs the tensor core more than the CUDA cores); tiles left empty
// are dropped.
void demote(Staging& st, int W, int min_rows) {
  if (min_rows <= 1) return;
  // each window's demoted entries, appended to the residual in window order
  std::vector<std::vector<ResEntry>> moved(W);
  parallel_windows(W, [&](int64_t w0, int64_t w1) {
  for (int w = (int)w0; w < (int)w1; ++w) {
    WinTiles& wt = st.sp[w];
    WinTiles kept;
    for (int t = 0; t < wt.n; ++t) {
      const size_t cb = (size_t)t * 16, ab = (size_t)t * 256;
      int cnt[16] = {0};
      for (int i = 0; i < 256; ++i)
        if (wt.a[ab + i] != 0.f || wt.edge[ab + i] >= 0) cnt[((i % 128) / 64) * 8 + (i % 8)]++;
      bool any = false;
      for (int k = 0; k < 16; ++k) {
        if (wt.col[cb + k] < 0) continue;
        if (cnt[k] >= min_rows) { any = true; continue; }
        for (int n = 0; n < 16; ++n) {              // column k's slots, rows ascending
          const int i = a_index(n, k);
          if (wt.a[ab + i] == 0.f && wt.edge[ab + i] < 0) continue;
          moved[w].push_back({w * 16 + elem_row(i), wt.col[cb + k], wt.a[ab + i], wt.edge[ab + i]});
          wt.a[ab + i] = 0.f;
          wt.edge[ab + i] = -1;
        }
        wt.col[cb + k] = -1;
      }
      if (!any) continue;
      kept.col.insert(kept.col.end(), wt.col.begin() + cb, wt.col.begin() + cb + 16);
      kept.a.insert(kept.a.end(), wt.a.begin() + ab, wt.a.begin() + ab + 256);
      kept.edge.insert(kept.edge.end(), wt.edge.begin() + ab, wt.edge.begin() + ab + 256);
      kept.n++;
    }
    wt = std::move(kept);
  }
  });
  size_t total = st.res.size();
  for (const auto& m : moved) total += m.size();
  st.res.reserve(total);
  for (auto& m : moved) {
    st.res.insert(st.res.end(), m.begin(), m.end());
    std::vector<ResEntry>().swap(m);
  }
}

void promote(Staging& st, int W, int min_rows) {
  if (min_rows <= 0) return;
  std::vector<std::vector<size_t>> by_win(W);
  for (size_t i = 0; i < st.res.size(); ++i) by_win[st.res[i].row / 16].push_back(i);
  std::vector<char> moved(st.res.size(), 0);
  std::vector<size_t> idx;
  for (int w = 0; w < W; ++w) {
    idx = by_win[w];
    std::stable_sort(idx.begin(), idx.end(),
                     [&](size_t x, size_t y) { return st.res[x].col < st.res[y].col; });
    WinTiles& wt = st.pr[w];
    std::vector<char> occ;                           // (tile, element) taken
    int slot = 16;
    for (size_t i = 0; i < idx.size();) {
      size_t j = i;
      while (j < idx.size() && st.res[idx[j]].col == st.res[idx[i]].col) ++j;
      if ((int)(j - i) >= min_rows) {
        if (slot == 16) {
          wt.add_empty();
          occ.insert(occ.end(), 256, 0);
          slot = 0;
        }
        const size_t cb = (size_t)(wt.n - 1) * 16, ab = (size_t)(wt.n - 1) * 256;
        wt.col[cb + slot] = st.res[idx[i]].col;
        for (size_t q = i; q < j; ++q) {
          const ResEntry& e = st.res[idx[q]];
          const size_t at = ab + a_index(e.row % 16, slot);
          if (occ[at]) continue;                     // repeated (row, column): stays
          occ[at] = 1;
          wt.a[at] = e.val;
          wt.edge[at] = e.edge;
          moved[idx[q]] = 1;
        }
        ++slot;
      }
      i = j;
    }
  }
  size_t keep = 0;
  for (size_t i = 0; i < st.res.size(); ++i)
    if (!moved[i]) st.res[keep++] = st.res[i];
  st.res.resize(keep);
}

void flatten(HostPlan& hp, Staging& st, const PlanOptions& opt, int64_t n_edges) {
  const int W = hp.n_windows;
  const int64_t rows = (int64_t)W * 16;
  demote(st, W, opt.demote_below);
  promote(st, W, opt.promote_min);
  // ---- per-row scales ---------------------------------------------------------
  hp.row_scale.assign(rows, 1.0f);
  hp.row_scaled = opt.row_scale;
  if (opt.row_scale) {
    std::vector<float> mx(rows, 0.f);
    for (int w = 0; w < W; ++w)
      for (WinTiles* wt : {&st.tc[w], &st.sp[w], &st.pr[w]})
        for (int t = 0; t < wt->n; ++t)
          for (int i = 0; i < 256; ++i) {
            const int64_t r = (int64_t)w * 16 + elem_row(i);
            mx[r] = std::max(mx[r], std::fabs(wt->a[(size_t)t * 256 + i]));
          }
    for (auto& e : st.res) mx[e.row] = std::max(mx[e.row], std::fabs(e.val));
    for (int64_t r = 0; r < rows; ++r) hp.row_scale[r] = mx[r] > 0.f ? mx[r] : 1.0f;
  }
  hp.row_out.resize(rows);
  for (int64_t r = 0; r < rows; ++r) hp.row_out[r] = r < hp.n_rows ? (int32_t)r : -1;
  // ---- tiles, window-major: dense TC, then 2:4, then promoted ------------------
  hp.win_tile.assign(1, 0);
  hp.win_split.resize(W);
  hp.win_prom.resize(W);
  hp.val_slot.assign(n_edges, -1);
  hp.edge_row.assign(n_edges, -1);
  // window offsets first, then every window's tiles filled in parallel (each
  // CSR entry lives in one tile slot, so the entry maps are written once)
  hp.win_tile.resize((size_t)W + 1);
  hp.win_tile[0] = 0;
  for (int w = 0; w < W; ++w) {
    hp.win_split[w] = hp.win_tile[w] + st.tc[w].n;
    hp.win_prom[w] = hp.win_split[w] + st.sp[w].n;
    hp.win_tile[w + 1] = hp.win_prom[w] + st.pr[w].n;
    hp.tc_tiles += st.tc[w].n;
    hp.sptc_tiles += st.sp[w].n;
    hp.prom_tiles += st.pr[w].n;
  }
  hp.tile_col.resize((size_t)hp.win_tile[W] * 16);
  hp.tile_a.resize((size_t)hp.win_tile[W] * 256);
  auto put_tiles = [&](int w, const WinTiles& wt, int64_t first) {
    for (int t = 0; t < wt.n; ++t) {
      const int64_t tile = first + t;
      std::copy(wt.col.begin() + t * 16, wt.col.begin() + t * 16 + 16, hp.tile_col.begin() + tile * 16);
      for (int i = 0; i < 256; ++i) {
        const int64_t r = (int64_t)w * 16 + elem_row(i);
        hp.tile_a[(size_t)tile * 256 + i] = f2h(wt.a[(size_t)t * 256 + i] / hp.row_scale[r]);
        const int32_t e = wt.edge[(size_t)t * 256 + i];
        if (e >= 0 && e < n_edges) {
          hp.val_slot[e] = (int32_t)(tile * 256 + i);
          hp.edge_row[e] = (int32_t)r;
        }
      }
    }
  };
  parallel_windows(W, [&](int64_t w0, int64_t w1) {
    for (int w = (int)w0; w < (int)w1; ++w) {
      put_tiles(w, st.tc[w], hp.win_tile[w]);
      put_tiles(w, st.sp[w], hp.win_split[w]);
      put_tiles(w, st.pr[w], hp.win_prom[w]);
    }
  });
  const int64_t T = (int64_t)hp.tile_col.size() / 16;
  // ---- residual CSR over padded rows, entries of a row in table order -------
  // (a stable counting sort by row: host threads take contiguous ranges of
  // the entries, count per row, and scatter from per-(row, thread) offsets)
  const int64_t NR = (int64_t)st.res.size();
  int nt = (int)std::max(1u, std::thread::hardware_concurrency());
  nt = (int)std::min<int64_t>(nt, std::max<int64_t>(1, NR / 65536));
  while (nt > 1 && (int64_t)nt * rows > ((int64_t)1 << 26)) --nt;
  std::vector<std::vector<int32_t>> off(nt, std::vector<int32_t>((size_t)rows, 0));
  auto on_ranges = [&](auto body) {
    std::vector<std::thread> pool;
    for (int k = 1; k < nt; ++k) pool.emplace_back(body, k);
    body(0);
    for (auto& th : pool) th.join();
  };
  on_ranges([&](int k) {
    for (int64_t i = NR * k / nt; i < NR * (k + 1) / nt; ++i) off[k][st.res[i].row]++;
  });
  hp.res_ptr.assign(rows + 1, 0);
  {
    int32_t base = 0;
    for (int64_t r = 0; r < rows; ++r) {
      hp.res_ptr[r] = base;
      for (int k = 0; k < nt; ++k) {
        const int32_t c = off[k][r];
        off[k][r] = base;
        base += c;
      }
    }
    hp.res_ptr[rows] = base;
  }
  hp.res_col.resize(hp.res_ptr[rows]);
  hp.res_val.resize(hp.res_ptr[rows]);
  hp.res_edge.assign(hp.res_ptr[rows], -1);
  on_ranges([&](int k) {
    std::vector<int32_t>& fill = off[k];
    for (int64_t i = NR * k / nt; i < NR * (k + 1) / nt; ++i) {
      const ResEntry& e = st.res[i];
      const int32_t at = fill[e.row]++;
      hp.res_col[at] = e.col;
      hp.res_val[at] = f2h(e.val / hp.row_scale[e.row]);
      if (e.edge >= 0 && e.edge < n_edges) {
        hp.res_edge[at] = e.edge;
        hp.val_slot[e.edge] = (int32_t)(T * 256 + at);
        hp.edge_row[e.edge] = e.row;
      }
    }
  });
  // ---- launch order: heaviest windows first (cost ~ gathered rows) -----------
  std::vector<int64_t> cost(W);
  for (int w = 0; w < W; ++w)
    cost[w] = (int64_t)(hp.win_tile[w + 1] - hp.win_tile[w]) * 16 +
              (hp.res_ptr[(int64_t)(w + 1) * 16] - hp.res_ptr[(int64_t)w * 16]);
  hp.win_order.resize(W);
  std::iota(hp.win_order.begin(), hp.win_order.end(), 0);
  std::stable_sort(hp.win_order.begin(), hp.win_order.end(),
                   [&](int a, int b) { return cost[a] > cost[b]; });
  int64_t nnz = (int64_t)hp.res_col.size();
  for (uint16_t v : hp.tile_a) nnz += (v & 0x7FFFu) != 0;
  hp.nnz = nnz;
}

// ---- dense TC sub-blocks ------------------------------------------------------
int add_tc(const int32_t* t_row_offset, int64_t n_t_row_offset, const int32_t* t_block_offset,
           int64_t n_t_block_offset, const int32_t* t_column, int64_t n_t_column,
           const float* t_val32, const uint16_t* t_val16, int64_t n_t_value,
           const int32_t* t_edge, const int32_t* t_window_row, int64_t n_t_window_row,
           const int64_t* t_binary, int64_t n_t_binary, int32_t n_cols, int W, Staging& st,
           std::string& err) {
  if (n_t_row_offset <= 1) return TR_OK;
  const int64_t parts = n_t_row_offset - 1;
  if (n_t_window_row < parts) { err = "t_window_row shorter than the part count"; return TR_ERR_ARG; }
  const int64_t subs = t_row_offset[parts];
  if (t_row_offset[0] != 0 || subs < 0 || subs * 8 > n_t_column || subs * 2 > n_t_binary ||
      n_t_block_offset < subs + 1) {
    err = "TC tables have inconsistent sizes";
    return TR_ERR_ARG;
  }
  std::vector<std::vector<int64_t>> win_subs(W);
  for (int64_t p = 0; p < parts; ++p) {
    const int32_t wr = t_window_row[p];
    if (wr < 0 || wr % 16 != 0 || wr / 16 >= W) { err = "t_window_row out of range"; return TR_ERR_ARG; }
    if (t_row_offset[p + 1] < t_row_offset[p]) { err = "t_row_offset must be non-decreasing"; return TR_ERR_ARG; }
    for (int64_t s = t_row_offset[p]; s < t_row_offset[p + 1]; ++s) win_subs[wr / 16].push_back(s);
  }
  for (int w = 0; w < W; ++w) {
    auto& L = win_subs[w];
    for (size_t i = 0; i < L.size(); i += 2) {
      WinTiles& wt = st.tc[w];
      const size_t cbase = wt.col.size(), abase = wt.a.size();
      wt.add_empty();
      for (int half = 0; half < 2 && i + half < L.size(); ++half) {
        const int64_t s = L[i + half];
        const int64_t voff = t_block_offset[s], vend = t_block_offset[s + 1];
        if (voff < 0 || vend < voff || vend > n_t_value) { err = "t_block_offset out of range"; return TR_ERR_ARG; }
        for (int k = 0; k < 8; ++k) {
          const int32_t c = t_column[s * 8 + k];
          if (c < -1 || c >= n_cols) { err = "t_column out of range"; return TR_ERR_ARG; }
          wt.col[cbase + half * 8 + k] = c;
        }
        const uint64_t lo = (uint64_t)t_binary[2 * s], hi = (uint64_t)t_binary[2 * s + 1];
        int rank = 0;
        for (int hsel = 0; hsel < 2; ++hsel) {
          const uint64_t word = hsel ? hi : lo;
          for (int bit = 0; bit < 64; ++bit) {
            if (!((word >> bit) & 1u)) continue;
            const int row = hsel * 8 + bit / 8, k = half * 8 + bit % 8;
            if (voff + rank >= vend) { err = "TC bitmap has more bits than values"; return TR_ERR_ARG; }
            if (wt.col[cbase + k] < 0) { err = "TC bit set in a padded column"; return TR_ERR_ARG; }
            const int64_t vi = voff + rank;
            wt.a[abase + a_index(row, k)] = t_val32 ? t_val32[vi] : h2f(t_val16[vi]);
            wt.edge[abase + a_index(row, k)] = t_edge ? t_edge[vi] : -1;
            rank++;
          }
        }
      }
    }
  }
  return TR_OK;
}

// ---- packed 2:4 tiles (block_online.cpp:797-841) --------------------------------
int add_packed_tiles(const int32_t* tile_column, int64_t n_tile_column, const uint32_t* packed_a,
                     int64_t n_packed_a, const uint32_t* packed_meta, int64_t n_packed_meta,
                     const int32_t* wto, int64_t n_wto, int32_t n_cols, int W, Staging& st,
                     std::string& err) {
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
      WinTiles& wt = st.sp[w];
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
              wt.a[abase + a_index(row, k)] = h2f(bits);
            }
          }
      }
    }
  }
  return TR_OK;
}

// ---- 2:4 groups (s_column / s_value / s_pos) -------------------------------------
// With to_residual (every 2:4 column would be demoted: no column of a
// window holds more than 16 entries) the group entries go straight to the
// CUDA-core residual, by the rule demote() applies, without being laid out
// as tiles first.
int add_groups(const int32_t* s_column, const float* s_value, const int8_t* s_pos,
               const int32_t* s_edge, int64_t groups, const std::vector<int32_t>& gwin,
               int32_t n_rows, int32_t n_cols, int W, Staging& st, std::string& err,
               bool to_residual = false) {
  std::atomic<bool> bad_col{false};
  if (to_residual) {
    // contiguous ranges of groups on the host threads, concatenated in range
    // order: the residual keeps the groups' order
    const int chunks = 64;
    std::vector<std::vector<ResEntry>> part(chunks);
    parallel_windows(chunks, [&](int64_t q0, int64_t q1) {
      for (int64_t q = q0; q < q1; ++q)
        for (int64_t g = groups * q / chunks; g < groups * (q + 1) / chunks; ++g) {
          const int w = gwin[g];
          if (!in_range(w, 0, W)) continue;                 // beyond the matrix
          int32_t c[4];
          for (int p = 0; p < 4; ++p) {
            c[p] = s_column[g * 4 + p];
            if (c[p] < -1 || c[p] >= n_cols) { bad_col = true; c[p] = -1; }
          }
          for (int lr = 0; lr < 16; ++lr) {
            if ((int64_t)w * 16 + lr >= n_rows) continue;
            const int64_t at0 = (g * 16 + lr) * 2;
            for (int s = 0; s < 2; ++s) {
              const int64_t at = at0 + s;
              const int pos = s_pos[at];
              if (pos < 0 || pos > 3 || c[pos] < 0) continue;
              if (s == 0 && s_pos[at0 + 1] == pos) continue;  // the later slot wins, as in a tile
              const float v = s_value[at];
              const int32_t e = s_edge ? s_edge[at] : -1;
              if (v != 0.f || e >= 0) part[q].push_back({w * 16 + lr, c[pos], v, e});
            }
          }
        }
    });
    if (bad_col) { err = "s_column out of range"; return TR_ERR_ARG; }
    size_t total = st.res.size();
    for (const auto& v : part) total += v.size();
    st.res.reserve(total);
    for (auto& v : part) st.res.insert(st.res.end(), v.begin(), v.end());
    return TR_OK;
  }
  std::vector<std::vector<int64_t>> wg(W);
  for (int64_t g = 0; g < groups; ++g)
    if (in_range(gwin[g], 0, W)) wg[gwin[g]].push_back(g);   // others lie beyond the matrix
  parallel_windows(W, [&](int64_t w0, int64_t w1) {
    for (int w = (int)w0; w < (int)w1; ++w) {
      WinTiles& wt = st.sp[w];
      const size_t nt = (wg[w].size() + 3) / 4;
      wt.col.reserve(wt.col.size() + nt * 16);
      wt.a.reserve(wt.a.size() + nt * 256);
      wt.edge.reserve(wt.edge.size() + nt * 256);
      for (size_t i = 0; i < wg[w].size(); i += 4) {
        const size_t cbase = wt.col.size(), abase = wt.a.size();
        wt.add_empty();
        for (int ch = 0; ch < 4 && i + ch < wg[w].size(); ++ch) {
          const int64_t g = wg[w][i + ch];
          for (int p = 0; p < 4; ++p) {
            int32_t c = s_column[g * 4 + p];
            if (c < -1 || c >= n_cols) { bad_col = true; c = -1; }
            wt.col[cbase + ch * 4 + p] = c;
          }
          for (int lr = 0; lr < 16; ++lr) {
            if ((int64_t)w * 16 + lr >= n_rows) continue;
            for (int s = 0; s < 2; ++s) {
              const int64_t at = (g * 16 + lr) * 2 + s;
              const int pos = s_pos[at];
              if (pos < 0 || pos > 3 || wt.col[cbase + ch * 4 + pos] < 0) continue;   // kernel skips
              wt.a[abase + a_index(lr, ch * 4 + pos)] = s_value[at];
              wt.edge[abase + a_index(lr, ch * 4 + pos)] = s_edge ? s_edge[at] : -1;
            }
          }
        }
      }
    }
  });
  if (bad_col) { err = "s_column out of range"; return TR_ERR_ARG; }
  return TR_OK;
}

// ---- CUDA parts -----------------------------------------------------------------
int add_parts(const int32_t* off, int64_t n_off, const int32_t* row, int64_t n_row,
              const int32_t* col, int64_t n_col, const float* v32, const uint16_t* v16,
              int64_t n_val, const int32_t* edge, int32_t n_rows, int32_t n_cols, Staging& st,
              std::string& err) {
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
      st.res.push_back({row[p], col[e], v32 ? v32[e] : h2f(v16[e]), edge ? edge[e] : -1});
    }
  }
  return TR_OK;
}

void init(HostPlan& hp, int32_t n_rows, int32_t n_cols) {
  hp = HostPlan();
  hp.n_rows = n_rows;
  hp.n_cols = n_cols;
  hp.n_windows = (n_rows + 15) / 16;
}

}  // namespace

int plan_from_tables(const tr_tables& t, int32_t n_rows, int32_t n_cols, int32_t window,
                     HostPlan& hp, std::string& err) {
  if (window != 16) { err = "routed plans need window == 16"; return TR_ERR_UNSUPPORTED; }
  if (n_rows < 0 || n_cols < 0) { err = "negative matrix shape"; return TR_ERR_ARG; }
  init(hp, n_rows, n_cols);
  Staging st(hp.n_windows);
  int rc = add_tc(t.t_row_offset, t.n_t_row_offset, t.t_block_offset, t.n_t_block_offset,
                  t.t_column, t.n_t_column, nullptr, t.t_value, t.n_t_value, nullptr,
                  t.t_window_row, t.n_t_window_row, t.t_binary, t.n_t_binary, n_cols,
                  hp.n_windows, st, err);
  if (rc) return rc;
  rc = add_packed_tiles(t.s_tile_column, t.n_s_tile_column, t.s_packed_a, t.n_s_packed_a,
                        t.s_packed_meta, t.n_s_packed_meta, t.s_window_tile_offset,
                        t.n_s_window_tile_offset, n_cols, hp.n_windows, st, err);
  if (rc) return rc;
  rc = add_parts(t.c_row_offset, t.n_c_row_offset, t.c_row, t.n_c_row, t.c_column, t.n_c_column,
                 nullptr, t.c_value, t.n_c_value, nullptr, n_rows, n_cols, st, err);
  if (rc) return rc;
  rc = add_parts(t.cs_row_offset, t.n_cs_row_offset, t.cs_row, t.n_cs_row, t.cs_column,
                 t.n_cs_column, nullptr, t.cs_value, t.n_cs_value, nullptr, n_rows, n_cols, st,
                 err);
  if (rc) return rc;
  flatten(hp, st, PlanOptions(), 0);
  return TR_OK;
}

int plan_from_route(const RouteTables& T, int32_t n_rows, int32_t n_cols, int64_t n_edges,
                    const PlanOptions& opt, HostPlan& hp, std::string& err) {
  if (T.window != 16) { err = "routed plans need window == 16"; return TR_ERR_UNSUPPORTED; }
  init(hp, n_rows, n_cols);
  Staging st(hp.n_windows);
  int rc = add_tc(T.t_row_offset.data(), (int64_t)T.t_row_offset.size(), T.t_block_offset.data(),
                  (int64_t)T.t_block_offset.size(), T.t_column.data(), (int64_t)T.t_column.size(),
                  T.t_value.data(), nullptr, (int64_t)T.t_value.size(), T.t_edge.data(),
                  T.t_window_row.data(), (int64_t)T.t_window_row.size(), T.t_binary.data(),
                  (int64_t)T.t_binary.size(), n_cols, hp.n_windows, st, err);
  if (rc) return rc;
  const int64_t groups = (int64_t)T.s_window.size();
  rc = add_groups(T.s_column.data(), T.s_value.data(), T.s_pos.data(), T.s_edge.data(), groups,
                  T.s_window, n_rows, n_cols, hp.n_windows, st, err, opt.demote_below > 16);
  if (rc) return rc;
  rc = add_parts(T.c_row_offset.data(), (int64_t)T.c_row_offset.size(), T.c_row.data(),
                 (int64_t)T.c_row.size(), T.c_column.data(), (int64_t)T.c_column.size(),
                 T.c_value.data(), nullptr, (int64_t)T.c_value.size(), T.c_edge.data(), n_rows,
                 n_cols, st, err);
  if (rc) return rc;
  rc = add_parts(T.cs_row_offset.data(), (int64_t)T.cs_row_offset.size(), T.cs_row.data(),
                 (int64_t)T.cs_row.size(), T.cs_column.data(), (int64_t)T.cs_column.size(),
                 T.cs_value.data(), nullptr, (int64_t)T.cs_value.size(), T.cs_edge.data(), n_rows,
                 n_cols, st, err);
  if (rc) return rc;
  flatten(hp, st, opt, n_edges);
  return TR_OK;
}

int plan_from_groups(const int32_t* s_column, const float* s_value, const int8_t* s_pos,
                     int64_t groups, const int32_t* s_window, const int32_t* s_offsets,
                     int64_t n_offsets, int32_t window, int32_t n_rows, int32_t n_cols,
                     HostPlan& hp, std::string& err) {
  if (window != 16) { err = "routed plans need window == 16"; return TR_ERR_UNSUPPORTED; }
  init(hp, n_rows, n_cols);
  std::vector<int32_t> gwin(groups);
  // one of the two window maps is given; with no groups s_window may be null
  if (!s_offsets) {
    if (groups > 0 && !s_window) { err = "null s_window"; return TR_ERR_ARG; }
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
  Staging st(hp.n_windows);
  int rc = add_groups(s_column, s_value, s_pos, nullptr, groups, gwin, n_rows, n_cols,
                      hp.n_windows, st, err);
  if (rc) return rc;
  flatten(hp, st, PlanOptions(), 0);
  return TR_OK;
}

int plan_upload(const HostPlan& hp, tr_plan** out) {
  const int W = hp.n_windows;
  const int64_t T = (int64_t)hp.tile_col.size() / 16;
  const int64_t rows = (int64_t)W * 16;
  const int64_t n_edges = (int64_t)hp.val_slot.size();
  auto al = [](int64_t b) { return (std::max<int64_t>(b, 1) + 255) / 256 * 256; };
  // block layout on the device: each entry as one word (FP16 value bits <<
  // 16 | tile byte offset), and val_slot naming the value's half of it
  std::vector<uint32_t> ent_pv;
  std::vector<int32_t> dev_slot;
  // block schedule: longest-processing-time first over the device's SMs
  // (each block, heaviest first, to the CTA with the fewest chunks so far)
  std::vector<int32_t> cta_ptr, cta_blk;
  if (hp.block) {
    int dev = 0, sms = 1;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms < 1) {
      cudaGetLastError();
      sms = 1;
    }
    const int32_t NB = (int32_t)hp.blk_order.size();
    const int32_t G = std::max(1, std::min(sms, NB));
    std::vector<std::vector<int32_t>> lists(G);
    std::priority_queue<std::pair<int64_t, int32_t>, std::vector<std::pair<int64_t, int32_t>>,
                        std::greater<std::pair<int64_t, int32_t>>> load;
    for (int32_t c = 0; c < G; ++c) load.push({0, c});
    for (int32_t b : hp.blk_order) {
      auto [l, c] = load.top();
      load.pop();
      lists[c].push_back(b);
      load.push({l + hp.blk_chunk[b + 1] - hp.blk_chunk[b] + 1, c});
    }
    cta_ptr.assign((size_t)G + 1, 0);
    for (int32_t c = 0; c < G; ++c) {
      cta_ptr[c + 1] = cta_ptr[c] + (int32_t)lists[c].size();
      cta_blk.insert(cta_blk.end(), lists[c].begin(), lists[c].end());
    }
  }
  if (hp.block) {
    ent_pv.resize(hp.ent_pos.size());
    for (size_t e = 0; e < ent_pv.size(); ++e)
      ent_pv[e] = (uint32_t)hp.ent_pos[e] | ((uint32_t)hp.ent_val[e] << 16);
    dev_slot.resize(hp.val_slot.size());
    for (size_t e = 0; e < dev_slot.size(); ++e)
      dev_slot[e] = hp.val_slot[e] < 0 ? -1 : 2 * hp.val_slot[e] + 1;
  }
  struct Sec { const void* src; int64_t bytes; int64_t size; };
  Sec secs[] = {
      {hp.win_tile.data(), (W + 1) * 4, 0},
      {hp.win_split.data(), (int64_t)W * 4, 0},
      {hp.win_prom.data(), (int64_t)W * 4, 0},
      {hp.tile_col.data(), T * 64, 0},
      {hp.tile_a.data(), T * 512, 0},
      {hp.res_ptr.data(), (rows + 1) * 4, 0},
      {hp.res_col.data(), (int64_t)hp.res_col.size() * 4, 0},
      {hp.res_val.data(), (int64_t)hp.res_val.size() * 2, 0},
      {hp.win_order.data(), (int64_t)W * 4, 0},
      {hp.row_scale.data(), rows * 4, 0},
      {hp.row_out.data(), rows * 4, 0},
      {hp.block ? dev_slot.data() : hp.val_slot.data(), n_edges * 4, 0},
      {hp.edge_row.data(), n_edges * 4, 0},
      {hp.res_edge.data(), (int64_t)hp.res_edge.size() * 4, 0},
      {nullptr, 0, 256},                       // error words
      {hp.blk_chunk.data(), (int64_t)hp.blk_chunk.size() * 4, 0},
      {hp.chunk_col.data(), (int64_t)hp.chunk_col.size() * 4, 0},
      {hp.chunk_ent.data(), (int64_t)hp.chunk_ent.size() * 4, 0},
      {ent_pv.data(), (int64_t)ent_pv.size() * 4, 0},
      {hp.ent_src.data(), (int64_t)hp.ent_src.size() * 4, 0},
      {hp.blk_order.data(), (int64_t)hp.blk_order.size() * 4, 0},
      {cta_ptr.data(), (int64_t)cta_ptr.size() * 4, 0},
      {cta_blk.data(), (int64_t)cta_blk.size() * 4, 0},
  };
  constexpr int kSecs = sizeof(secs) / sizeof(secs[0]);
  int64_t total = 0;
  for (auto& s : secs) {
    if (s.size == 0) s.size = al(s.bytes);
    total += s.size;
  }
  tr_plan* p = new tr_plan();
  cudaGetDevice(&p->device);
  cudaError_t e = cudaMalloc(&p->block, total);
  if (e != cudaSuccess) { delete p; return cuda_fail(e, "cudaMalloc(plan)"); }
  p->bytes = total;
  char* base = (char*)p->block;
  char* at[kSecs];
  int64_t off = 0;
  for (int i = 0; i < kSecs; ++i) {
    at[i] = base + off;
    if (secs[i].bytes > 0) e = cudaMemcpy(at[i], secs[i].src, secs[i].bytes, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) break;
    off += secs[i].size;
  }
  if (e == cudaSuccess) e = cudaMemset(at[14], 0, 256);
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e != cudaSuccess) { cudaFree(p->block); delete p; return cuda_fail(e, "plan upload"); }
  PlanView& v = p->view;
  v.n_rows = hp.n_rows;
  v.n_cols = hp.n_cols;
  v.n_windows = W;
  v.win_tile = (const int32_t*)at[0];
  v.win_split = (const int32_t*)at[1];
  v.win_prom = (const int32_t*)at[2];
  v.tile_col = (const int32_t*)at[3];
  v.tile_a = (const uint16_t*)at[4];
  v.res_ptr = (const int32_t*)at[5];
  v.res_col = (const int32_t*)at[6];
  v.res_val = (const uint16_t*)at[7];
  v.win_order = (const int32_t*)at[8];
  v.row_scale = (const float*)at[9];
  v.row_out = (const int32_t*)at[10];
  v.res_edge = (const int32_t*)at[13];
  v.err = (int*)at[14];
  v.n_blocks = hp.block ? (int32_t)hp.blk_order.size() : 0;
  v.blk_chunk = (const int32_t*)at[15];
  v.chunk_col = (const int32_t*)at[16];
  v.chunk_ent = (const int32_t*)at[17];
  v.ent_pv = (const uint32_t*)at[18];
  v.ent_src = (const int32_t*)at[19];
  v.blk_order = (const int32_t*)at[20];
  v.n_sched = hp.block ? (int32_t)cta_ptr.size() - 1 : 0;
  v.cta_ptr = (const int32_t*)at[21];
  v.cta_blk = (const int32_t*)at[22];
  p->blocked = hp.block;
  for (size_t c = 0; c + 1 < cta_ptr.size(); ++c)
    p->max_sched_blocks = std::max(p->max_sched_blocks, cta_ptr[c + 1] - cta_ptr[c]);
  // re-valuing writes FP16 values at tile_a[val_slot] below n_tile_vals; in
  // the block layout that is the value half of each entry word
  p->tile_a = hp.block ? (uint16_t*)at[18] : (uint16_t*)at[4];
  p->res_val = (uint16_t*)at[7];
  p->row_scale = (float*)at[9];
  p->val_slot = (int32_t*)at[11];
  p->edge_row = (int32_t*)at[12];
  p->n_edges = n_edges;
  p->n_tile_vals = hp.block ? 2 * (int64_t)ent_pv.size() : T * 256;
  p->row_scaled = hp.row_scaled;
  p->info.n_rows = hp.n_rows;
  p->info.n_cols = hp.n_cols;
  p->info.n_windows = W;
  p->info.nnz = hp.nnz;
  p->info.tc_tiles = hp.tc_tiles;
  p->info.sptc_tiles = hp.sptc_tiles;
  p->info.residual_nnz = (int64_t)hp.res_col.size();
  p->info.device_bytes = total;
  p->info.promoted_tiles = hp.prom_tiles;
  p->info.row_scaled = hp.row_scaled ? 1 : 0;
  p->info.reordered = hp.reordered ? 1 : 0;
  p->info.engine = hp.block ? TR_ENGINE_BLOCK : TR_ENGINE_WINDOW;
  p->info.n_blocks = v.n_blocks;
  p->info.chunks = hp.block ? (int64_t)hp.blk_chunk.back() : 0;
  // distinct (block, column) pairs, slot layers included: the B rows one
  // product gathers
  p->info.slots = 0;
  for (int32_t c : hp.chunk_col) p->info.slots += c >= 0 ? 1 : 0;
  if (hp.block) p->info.residual_nnz = 0;
  p->info.n_edges = n_edges;
  *out = p;
  return TR_OK;
}

}  // namespace trs
