// Block layout of the block engine (layout described in plan.h).
//
// Each block of 128 consecutive plan rows lists the distinct columns its
// entries touch; column j becomes one K slot of a 16-slot chunk, so the
// kernel gathers row j of B once for the whole block and the tensor core
// multiplies it against all 128 rows.  A (row, column) pair that occurs more
// than once in the CSR (duplicate entries) takes a second slot of the same
// column (slot layers), so every A tile holds at most one value per
// position and the product still sums every entry.
//
// Blocks are laid out independently on host threads; the arrays are then
// concatenated in block order, so the result does not depend on the thread
// count.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <string>
#include <thread>
#include <vector>

#include "../../include/trspmm.h"
#include "plan.h"

namespace trs {
namespace {

uint16_t to_half(float f) {
  const _Float16 h = (_Float16)f;     // round to nearest even
  uint16_t bits;
  std::memcpy(&bits, &h, 2);
  return bits;
}

// One block's share of the layout.
struct BlockOut {
  std::vector<int32_t> col;      // chunks * 16 slot columns (-1 padding)
  std::vector<int32_t> ent_end;  // per chunk: end of its entries (block-local)
  std::vector<uint16_t> pos, val;
  std::vector<int32_t> src, row;  // entry of A, plan row
};

struct Key {
  int32_t col, row;   // row within the block
  int32_t e;          // entry of the Csr
};

void lay_out_block(const Csr& a, int32_t b, const std::vector<float>& scale, BlockOut& out,
                   std::vector<Key>& keys) {
  const int32_t r0 = b * kBlkRows, r1 = std::min(r0 + kBlkRows, a.n_rows);
  keys.clear();
  for (int32_t r = r0; r < r1; ++r)
    for (int32_t e = a.ptr[r]; e < a.ptr[r + 1]; ++e) keys.push_back({a.idx[e], r - r0, e});
  std::sort(keys.begin(), keys.end(), [](const Key& x, const Key& y) {
    if (x.col != y.col) return x.col < y.col;
    if (x.row != y.row) return x.row < y.row;
    return x.e < y.e;
  });
  // slot of each key: columns in ascending order, a column's layers 0, 1, ...
  // consecutive; a key's layer = how many earlier keys share its (col, row)
  const size_t n = keys.size();
  std::vector<int32_t> slot(n);
  int32_t next = 0;
  for (size_t i = 0; i < n;) {
    size_t j = i;
    int32_t layers = 1, layer = 0;
    for (; j < n && keys[j].col == keys[i].col; ++j) {
      layer = (j > i && keys[j].row == keys[j - 1].row) ? layer + 1 : 0;
      layers = std::max(layers, layer + 1);
      slot[j] = next + layer;
    }
    next += layers;
    i = j;
  }
  // whole groups of kChunkGroup chunks per block (the kernel waits for and
  // issues a group's MMAs together); padding chunks have no entries and no columns
  const int32_t n_chunks =
      (next + kChunkCols * kChunkGroup - 1) / (kChunkCols * kChunkGroup) * kChunkGroup;
  out.col.assign((size_t)n_chunks * kChunkCols, -1);
  for (size_t i = 0; i < n; ++i) out.col[slot[i]] = keys[i].col;
  // entries ordered by slot (so by chunk), a slot's entries by row
  std::vector<int32_t> order(n);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(),
                   [&](int32_t x, int32_t y) { return slot[x] < slot[y]; });
  out.ent_end.assign(n_chunks, 0);
  out.pos.resize(n);
  out.val.resize(n);
  out.src.resize(n);
  out.row.resize(n);
  for (size_t t = 0; t < n; ++t) {
    const Key& k = keys[order[t]];
    const int32_t s = slot[order[t]], kk = s % kChunkCols, m = k.row;
    out.ent_end[s / kChunkCols] = (int32_t)t + 1;
    out.pos[t] = (uint16_t)((m >> 3) * 256 + (kk >> 3) * 128 + (m & 7) * 16 + (kk & 7) * 2);
    out.val[t] = to_half(a.val[k.e] / scale[r0 + m]);
    out.src[t] = a.src[k.e];
    out.row[t] = r0 + m;
  }
  for (int32_t c = 1; c < n_chunks; ++c) out.ent_end[c] = std::max(out.ent_end[c], out.ent_end[c - 1]);
}

}  // namespace

int plan_blocks(const Csr& a, bool row_scale, int64_t n_edges, HostPlan& hp, std::string& err) {
  const int32_t R = a.n_rows;
  const int32_t NB = (R + kBlkRows - 1) / kBlkRows;
  const int64_t nnz = (int64_t)a.idx.size();
  if (nnz > INT32_MAX) { err = "more than 2^31 - 1 entries"; return TR_ERR_UNSUPPORTED; }
  hp = HostPlan();
  hp.n_rows = R;
  hp.n_cols = a.n_cols;
  hp.n_windows = NB * (kBlkRows / 16);
  hp.block = true;
  hp.nnz = nnz;
  const int64_t rows = (int64_t)NB * kBlkRows;
  hp.row_scale.assign(rows, 1.0f);
  hp.row_scaled = row_scale;
  if (row_scale) {
    for (int32_t r = 0; r < R; ++r) {
      float mx = 0.f;
      for (int32_t e = a.ptr[r]; e < a.ptr[r + 1]; ++e) mx = std::max(mx, std::fabs(a.val[e]));
      hp.row_scale[r] = mx > 0.f ? mx : 1.0f;
    }
  }
  hp.row_out.assign(rows, -1);
  for (int32_t r = 0; r < R; ++r) hp.row_out[r] = r;
  // the window sections describe empty windows (no tiles, no residual)
  const int32_t W = hp.n_windows;
  hp.win_tile.assign((size_t)W + 1, 0);
  hp.win_split.assign(W, 0);
  hp.win_prom.assign(W, 0);
  hp.res_ptr.assign((size_t)rows + 1, 0);
  hp.win_order.resize(W);
  std::iota(hp.win_order.begin(), hp.win_order.end(), 0);

  std::vector<BlockOut> outs(NB);
  int T = (int)std::max(1u, std::thread::hardware_concurrency());
  T = std::max(1, std::min(T, NB));
  {
    std::vector<std::thread> pool;
    auto body = [&](int t) {
      std::vector<Key> keys;
      for (int32_t b = t; b < NB; b += T) lay_out_block(a, b, hp.row_scale, outs[b], keys);
    };
    for (int t = 1; t < T; ++t) pool.emplace_back(body, t);
    body(0);
    for (auto& th : pool) th.join();
  }
  hp.blk_chunk.assign((size_t)NB + 1, 0);
  std::vector<int64_t> ent_at((size_t)NB + 1, 0);
  for (int32_t b = 0; b < NB; ++b) {
    hp.blk_chunk[b + 1] = hp.blk_chunk[b] + (int32_t)outs[b].ent_end.size();
    ent_at[b + 1] = ent_at[b] + (int64_t)outs[b].pos.size();
  }
  const int64_t NC = hp.blk_chunk[NB];
  hp.chunk_col.resize((size_t)NC * kChunkCols);
  hp.chunk_ent.assign((size_t)NC + 1, 0);
  hp.ent_pos.resize(nnz);
  hp.ent_val.resize(nnz);
  hp.ent_src.resize(nnz);
  hp.val_slot.assign(n_edges, -1);
  hp.edge_row.assign(n_edges, -1);
  {
    std::vector<std::thread> pool;
    auto body = [&](int t) {
      for (int32_t b = t; b < NB; b += T) {
        const BlockOut& o = outs[b];
        const int64_t c0 = hp.blk_chunk[b], e0 = ent_at[b];
        std::copy(o.col.begin(), o.col.end(), hp.chunk_col.begin() + c0 * kChunkCols);
        for (size_t c = 0; c < o.ent_end.size(); ++c)
          hp.chunk_ent[c0 + c + 1] = (int32_t)(e0 + o.ent_end[c]);
        std::copy(o.pos.begin(), o.pos.end(), hp.ent_pos.begin() + e0);
        std::copy(o.val.begin(), o.val.end(), hp.ent_val.begin() + e0);
        std::copy(o.src.begin(), o.src.end(), hp.ent_src.begin() + e0);
        for (size_t i = 0; i < o.src.size(); ++i) {
          const int32_t s = o.src[i];
          if (s >= 0 && s < n_edges) {
            hp.val_slot[s] = (int32_t)(e0 + (int64_t)i);
            hp.edge_row[s] = o.row[i];
          }
        }
      }
    };
    for (int t = 1; t < T; ++t) pool.emplace_back(body, t);
    body(0);
    for (auto& th : pool) th.join();
  }
  hp.blk_order.resize(NB);
  std::iota(hp.blk_order.begin(), hp.blk_order.end(), 0);
  std::stable_sort(hp.blk_order.begin(), hp.blk_order.end(), [&](int32_t x, int32_t y) {
    return hp.blk_chunk[x + 1] - hp.blk_chunk[x] > hp.blk_chunk[y + 1] - hp.blk_chunk[y];
  });
  return TR_OK;
}

}  // namespace trs
