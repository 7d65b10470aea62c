// 2:4 matching statistics (the reference's ablation tool for how well a
// window's columns pair up into 2:4 groups).  Three CPU variants, each a
// restatement of one reference extension:
//
//   sliding  TR-source/Block/block_matching_window_para_dr.cpp:80-290
//            (matching_utils.match_2to4): 1:2 pairs by a 32-column
//            look-ahead, 2:4 groups by a 1024-pair look-ahead, columns that
//            fail either step go to a pool that is cut into dense 16x8
//            blocks of `dense_threshold` columns, the rest into 2:4 groups
//            of at most two real columns.
//   hash     TR-source/Block/block_matching_hash.cpp:79-370
//            (matching_utils_hash.match_2to4_hash): exact-complement pairs
//            first (a mask -> column chain per window), then the 32-column
//            look-ahead; groups as above, failed pairs padded (no pool).
//   bucket   TR-source/Block/block_matching_bucket.cpp:66-420
//            (matching_utils_bucket.match_2to4_bucket): columns split by
//            whether rows 0-7 or 8-15 hold more entries, matched across
//            buckets first, 16-candidate look-aheads.
//   online   TR-source/Block/block_matching_online.cu:112-411
//            (matching_utils_online.match_2to4_online, a CUDA kernel): the
//            sliding variant's decisions over 16-row windows, with each 2:4
//            group counted as 32 slots and the pool's split between dense
//            blocks and 2:4 groups reported.  The reference orders a
//            window's columns by hash-slot arrival (not deterministic); here
//            they are in id order, on the host and in match_gpu.cu.
//
// Every variant encodes a window's column as a 16-bit row mask with the
// reference's truncation (rows past the 16th set no bit) and sorts the
// window's columns by column id, so the outcome is deterministic.  The
// counters are 64-bit (the reference's are 32-bit).
#include <algorithm>
#include <atomic>
#include <cstdint>
#include <string>
#include <thread>
#include <vector>

#include "../../include/trspmm.h"

namespace trs {
namespace {

struct MCol {
  int32_t id;
  uint16_t mask;
  int32_t nnz;
};

struct MPair {
  int32_t c1, c2;
  uint16_t g1, g2;   // AND and OR of the two masks
  int32_t nnz;
};

struct WinStats {
  int64_t groups = 0, tc_blocks = 0, blocks16 = 0, pad_groups = 0;
  int64_t fine_fb = 0, coarse_fb = 0, fake_zeros = 0;
  int64_t to_tc = 0, to_sptc = 0;      // pool columns routed to dense blocks / to 2:4 groups
};

inline int popc16(uint32_t x) { return __builtin_popcount(x & 0xFFFFu); }

// The window's distinct columns, sorted by id, with their 16-bit row masks.
void window_columns(const int32_t* indptr, const int32_t* indices, int32_t r0, int32_t r1,
                    std::vector<std::pair<int32_t, uint16_t>>& scratch, std::vector<MCol>& cols) {
  scratch.clear();
  for (int32_t r = r0; r < r1; ++r) {
    const int lr = r - r0;
    const uint16_t bit = (uint16_t)(lr < 16 ? (1u << lr) : 0u);
    for (int32_t e = indptr[r]; e < indptr[r + 1]; ++e) scratch.emplace_back(indices[e], bit);
  }
  std::sort(scratch.begin(), scratch.end(),
            [](const std::pair<int32_t, uint16_t>& a, const std::pair<int32_t, uint16_t>& b) {
              return a.first < b.first;
            });
  cols.clear();
  for (size_t i = 0; i < scratch.size();) {
    size_t j = i;
    uint16_t m = 0;
    while (j < scratch.size() && scratch[j].first == scratch[i].first) m |= scratch[j++].second;
    cols.push_back({scratch[i].first, m, popc16(m)});
    i = j;
  }
}

// Pairs column i with the best unused column among the next `look` ones:
// the first one with no common row, else the first with the fewest common
// rows when that count is <= t_max.  -1 when none qualifies.
int best_partner(const std::vector<MCol>& c, const std::vector<char>& used, int i, int look,
                 int t_max) {
  const int n = (int)c.size();
  int best = -1, best_cost = t_max + 1;
  for (int j = i + 1; j < std::min(i + 1 + look, n); ++j) {
    if (used[j]) continue;
    const int cost = popc16(c[i].mask & c[j].mask);
    if (cost == 0) return j;
    if (cost <= t_max && cost < best_cost) {
      best_cost = cost;
      best = j;
    }
  }
  return best;
}

MPair make_pair_of(const MCol& a, const MCol& b) {
  return {a.id, b.id, (uint16_t)(a.mask & b.mask), (uint16_t)(a.mask | b.mask), a.nnz + b.nnz};
}

inline bool compatible(const MPair& a, const MPair& b) {
  return ((a.g1 & b.g2) | (a.g2 & b.g1)) == 0;
}

int32_t nnz_of(const std::vector<MCol>& c, int32_t id) {
  auto it = std::lower_bound(c.begin(), c.end(), id,
                             [](const MCol& x, int32_t v) { return x.id < v; });
  return (it != c.end() && it->id == id) ? it->nnz : 0;
}

void tail_blocks(WinStats& s) {
  s.blocks16 += (s.groups + 3) / 4;
  s.pad_groups += ((s.groups + 3) / 4) * 4 - s.groups;
}

// block_matching_window_para_dr.cpp:80-243.  `slots` is what one 2:4 group
// holds: 2 * window rows in the sliding variant, always 32 in the CUDA
// variant (block_matching_online.cu:318-320, :378).
WinStats match_sliding(const std::vector<MCol>& c, int slots, int dense_threshold, int t_max) {
  WinStats s;
  const int n = (int)c.size();
  std::vector<char> used(n, 0);
  std::vector<MPair> pairs;
  std::vector<int32_t> pool;
  for (int i = 0; i < n; ++i) {
    if (used[i]) continue;
    const int j = best_partner(c, used, i, 32, t_max);
    used[i] = 1;
    if (j >= 0) {
      pairs.push_back(make_pair_of(c[i], c[j]));
      used[j] = 1;
    } else {
      pool.push_back(c[i].id);
      s.fine_fb++;
    }
  }
  const int np = (int)pairs.size();
  std::vector<char> pused(np, 0);
  for (int i = 0; i < np; ++i) {
    if (pused[i]) continue;
    pused[i] = 1;
    int j = i + 1;
    for (; j < std::min(i + 1 + 1024, np); ++j)
      if (!pused[j] && compatible(pairs[i], pairs[j])) break;
    if (j < std::min(i + 1 + 1024, np)) {
      pused[j] = 1;
      s.groups++;
      s.fake_zeros += slots - (pairs[i].nnz + pairs[j].nnz);
    } else {
      if (pairs[i].c1 >= 0) pool.push_back(pairs[i].c1);
      if (pairs[i].c2 >= 0) pool.push_back(pairs[i].c2);
      s.coarse_fb += 2;
    }
  }
  const int64_t nd = (int64_t)pool.size();
  const int64_t full = nd / dense_threshold;
  s.tc_blocks = full;
  s.to_tc = full * dense_threshold;
  s.to_sptc = nd - s.to_tc;
  int64_t idx = full * dense_threshold;
  while (idx < nd) {                      // groups of at most two real columns
    int64_t g_nnz = nnz_of(c, pool[idx++]);
    if (idx < nd) g_nnz += nnz_of(c, pool[idx++]);
    s.groups++;
    s.fake_zeros += slots - g_nnz;
  }
  tail_blocks(s);
  return s;
}

// block_matching_hash.cpp:104-283
WinStats match_hash(const std::vector<MCol>& c, int win_rows) {
  WinStats s;
  const int n = (int)c.size();
  std::vector<char> used(n, 0);
  std::vector<MPair> pairs;
  // exact complements: for each column, the unused column whose mask is the
  // complement of its own, taken from a per-mask chain walked newest first
  std::vector<int> order(n);
  for (int i = 0; i < n; ++i) order[i] = i;
  std::sort(order.begin(), order.end(), [&](int a, int b) {
    return c[a].mask != c[b].mask ? c[a].mask < c[b].mask : a > b;
  });
  auto chain_head = [&](uint16_t m) -> int {
    auto it = std::lower_bound(order.begin(), order.end(), m,
                               [&](int a, uint16_t v) { return c[a].mask < v; });
    return (it != order.end() && c[*it].mask == m) ? (int)(it - order.begin()) : -1;
  };
  for (int i = 0; i < n; ++i) {
    if (used[i]) continue;
    const uint16_t ideal = (uint16_t)(~c[i].mask);
    for (int k = chain_head(ideal); k >= 0 && k < n && c[order[k]].mask == ideal; ++k) {
      const int j = order[k];
      if (used[j] || j == i) continue;
      // the exact-complement pairs carry no entry count (their nnz is 0 in
      // the reference, which shows in fake_zeros)
      pairs.push_back({c[i].id, c[j].id, 0, (uint16_t)(c[i].mask | c[j].mask), 0});
      used[i] = used[j] = 1;
      break;
    }
  }
  for (int i = 0; i < n; ++i) {
    if (used[i]) continue;
    const int j = best_partner(c, used, i, 32, 8);
    used[i] = 1;
    if (j >= 0) {
      pairs.push_back(make_pair_of(c[i], c[j]));
      used[j] = 1;
    } else {
      pairs.push_back({c[i].id, -1, 0, c[i].mask, c[i].nnz});
      s.fine_fb++;
    }
  }
  const int np = (int)pairs.size();
  std::vector<char> pused(np, 0);
  for (int i = 0; i < np; ++i) {
    if (pused[i]) continue;
    pused[i] = 1;
    int j = i + 1;
    for (; j < std::min(i + 1 + 1024, np); ++j)
      if (!pused[j] && compatible(pairs[i], pairs[j])) break;
    s.groups++;
    if (j < std::min(i + 1 + 1024, np)) {
      pused[j] = 1;
      s.fake_zeros += (int64_t)win_rows * 2 - (pairs[i].nnz + pairs[j].nnz);
    } else {
      s.fake_zeros += (int64_t)win_rows * 2 - pairs[i].nnz;
      s.coarse_fb += 2;
    }
  }
  tail_blocks(s);
  return s;
}

// block_matching_bucket.cpp:66-358
WinStats match_bucket(const std::vector<MCol>& c) {
  constexpr int kLook = 16, kTMax = 8;
  WinStats s;
  const int n = (int)c.size();
  std::vector<char> used(n, 0);
  std::vector<MPair> pairs;
  std::vector<int> top, bottom, even;
  for (int i = 0; i < n; ++i) {
    const int lo = popc16(c[i].mask & 0x00FFu), hi = popc16(c[i].mask & 0xFF00u);
    (lo > hi ? top : hi > lo ? bottom : even).push_back(i);
  }
  // best unused candidate of `cand` for column i: the first with no common
  // row, else the fewest common rows (<= kTMax); at most kLook unused
  // candidates are examined (`skip_self`: i itself is skipped, not counted)
  auto best_in = [&](int i, const std::vector<int>& cand, bool skip_self) {
    int best = -1, best_cost = kTMax + 1, seen = 0;
    for (int j : cand) {
      if (used[j] || (skip_self && j == i)) continue;
      const int cost = popc16(c[i].mask & c[j].mask);
      if (cost == 0) return j;
      if (cost <= kTMax && cost < best_cost) {
        best_cost = cost;
        best = j;
      }
      if (++seen >= kLook) break;
    }
    return best;
  };
  auto take = [&](int i, int j) {
    pairs.push_back(make_pair_of(c[i], c[j]));
    used[i] = used[j] = 1;
  };
  for (int i : top)
    if (!used[i]) {
      const int j = best_in(i, bottom, false);
      if (j >= 0) take(i, j);
    }
  for (int i : top)
    if (!used[i]) {
      const int j = best_in(i, even, false);
      if (j >= 0) take(i, j);
    }
  for (int i : bottom)
    if (!used[i]) {
      const int j = best_in(i, even, false);
      if (j >= 0) take(i, j);
    }
  for (int i : even)
    if (!used[i]) {
      const int j = best_in(i, even, true);
      if (j >= 0) take(i, j);
    }
  for (int i = 0; i < n; ++i)
    if (!used[i]) {
      pairs.push_back({c[i].id, -1, 0, c[i].mask, c[i].nnz});
      used[i] = 1;
      s.fine_fb++;
    }
  const int np = (int)pairs.size();
  std::vector<char> pused(np, 0);
  auto group_nnz = [&](int32_t a, int32_t b) {
    return (a >= 0 ? nnz_of(c, a) : 0) + (b >= 0 ? nnz_of(c, b) : 0);
  };
  for (int i = 0; i < np; ++i) {
    if (pused[i]) continue;
    pused[i] = 1;
    int j = i + 1;
    for (; j < std::min(i + kLook, np); ++j)      // 15 candidates, as in the reference
      if (!pused[j] && compatible(pairs[i], pairs[j])) break;
    s.groups++;
    int64_t g = group_nnz(pairs[i].c1, pairs[i].c2);
    if (j < std::min(i + kLook, np)) {
      pused[j] = 1;
      g += group_nnz(pairs[j].c1, pairs[j].c2);
    } else {
      s.coarse_fb += 2;
    }
    s.fake_zeros += 32 - g;
  }
  tail_blocks(s);
  return s;
}

}  // namespace

int match_2to4(const int32_t* indptr, const int32_t* indices, int32_t n_rows, int variant,
               int32_t window_size, int32_t dense_threshold, int32_t t_max, tr_match_stats* out,
               std::string& err) {
  if (window_size < 1 || window_size > 64) {
    err = "window_size must be in [1, 64]";
    return TR_ERR_ARG;
  }
  if (variant == TR_MATCH_SLIDING && dense_threshold < 1) {
    err = "dense_threshold must be at least 1";
    return TR_ERR_ARG;
  }
  if (variant < TR_MATCH_SLIDING || variant > TR_MATCH_ONLINE) {
    err = "unknown matching variant";
    return TR_ERR_ARG;
  }
  if (variant == TR_MATCH_ONLINE && (window_size != 16 || dense_threshold < 1)) {
    err = "the online variant uses 16-row windows and dense_threshold >= 1";
    return TR_ERR_ARG;
  }
  const int64_t nnz = n_rows > 0 ? indptr[n_rows] : 0;
  int32_t n_cols = 0;
  for (int64_t e = 0; e < nnz; ++e) n_cols = std::max(n_cols, indices[e] + 1);
  if (n_rows <= 0 || n_cols <= 0) {
    err = "empty matrix (no rows or no columns)";
    return TR_ERR_ARG;
  }
  const int W = (n_rows + window_size - 1) / window_size;
  std::vector<WinStats> ws(W);
  // windows in chunks of 64 handed out to host threads (per-window results,
  // summed in window order afterwards)
  const int per_chunk = 64, nchunks = (W + per_chunk - 1) / per_chunk;
  std::atomic<int> next{0};
  auto worker = [&]() {
    std::vector<std::pair<int32_t, uint16_t>> scratch;
    std::vector<MCol> cols;
    for (int ch; (ch = next.fetch_add(1)) < nchunks;) {
      for (int w = ch * per_chunk; w < std::min(W, (ch + 1) * per_chunk); ++w) {
        const int32_t r0 = w * window_size, r1 = std::min(r0 + window_size, n_rows);
        window_columns(indptr, indices, r0, r1, scratch, cols);
        if (cols.empty()) continue;
        const int wr = r1 - r0;
        ws[w] = variant == TR_MATCH_SLIDING ? match_sliding(cols, 2 * wr, dense_threshold, t_max)
                : variant == TR_MATCH_ONLINE ? match_sliding(cols, 32, dense_threshold, t_max)
                : variant == TR_MATCH_HASH   ? match_hash(cols, wr)
                                             : match_bucket(cols);
      }
    }
  };
  const int threads =
      std::max(1, std::min((int)std::thread::hardware_concurrency(), std::max(1, nchunks)));
  if (threads == 1) {
    worker();
  } else {
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; ++t) pool.emplace_back(worker);
    for (auto& th : pool) th.join();
  }
  tr_match_stats s{};
  s.total_rows = n_rows;
  s.total_cols = n_cols;
  s.total_nnz = nnz;
  s.sparsity = 1.0 - (double)nnz / ((double)n_rows * n_cols);
  s.num_row_panels = W;
  for (const WinStats& w : ws) {
    s.num_groups += w.groups;
    s.num_tc_blocks += w.tc_blocks;
    s.num_16x16_blocks += w.blocks16;
    s.block_padding_groups += w.pad_groups;
    s.fine_fallback += w.fine_fb;
    s.coarse_fallback += w.coarse_fb;
    s.fake_zeros += w.fake_zeros;
    s.dense_to_tc_cols += w.to_tc;
    s.dense_to_sptc_cols += w.to_sptc;
  }
  *out = s;
  return TR_OK;
}

// One 16-row window of the online variant on the host (the GPU matcher
// hands back windows too large for its shared memory).  Counters in the
// order groups, tc_blocks, fine_fb, coarse_fb, fake_zeros, to_tc, to_sptc.
void match_online_window(const int32_t* indptr, const int32_t* indices, int32_t n_rows, int w,
                         int32_t dense_threshold, int32_t t_max, int64_t* out7) {
  std::vector<std::pair<int32_t, uint16_t>> scratch;
  std::vector<MCol> cols;
  const int32_t r0 = w * 16, r1 = std::min(r0 + 16, n_rows);
  window_columns(indptr, indices, r0, r1, scratch, cols);
  WinStats s;
  if (!cols.empty()) s = match_sliding(cols, 32, dense_threshold, t_max);
  const int64_t v[7] = {s.groups, s.tc_blocks, s.fine_fb, s.coarse_fb, s.fake_zeros, s.to_tc,
                        s.to_sptc};
  for (int i = 0; i < 7; ++i) out7[i] = v[i];
}

}  // namespace trs
