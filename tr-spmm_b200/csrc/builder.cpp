// Native plan builder: CSR -> (transpose) -> (row clustering) -> route -> plan.
//
// Every step keeps, for each CSR entry it moves, the index of the entry of
// the caller's A it came from, so the finished plan knows where the value of
// each entry of A lives (learnable edge weights re-value the plan on the
// device without rebuilding it).
//
// Row orders (opts.reorder) put rows that share columns into the same 16-row
// windows, so that a gathered feature row serves several output rows: the
// reference's optional row reorder (spmm/tr_csr_fp16/tr_tca_reorder.py:44-357,
// MinHash-LSH Jaccard clustering, off by default at
// spmm/tr_csr_fp16/mdataset2_online.py:73) is TR_REORDER_TCA (tca.cpp);
// TR_REORDER_LABEL is label propagation over the bipartite row/column graph
// (deterministic sweeps, seeded visiting order), then a stable sort of rows
// by label; TR_REORDER_GIVEN takes the caller's permutation.  Only rows move;
// B is never permuted, and the kernels write every result row back to its
// original position.
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <string>
#include <thread>
#include <vector>

#include "../../include/trspmm.h"
#include "common.cuh"
#include "plan.h"
#include "router.h"
#include "tca.h"

namespace trs {

int validate_csr(const int32_t* indptr, const int32_t* indices, int32_t n_rows, int32_t n_cols,
                 std::string& err) {
  if (n_rows < 0 || n_cols < 0) { err = "negative matrix shape"; return TR_ERR_ARG; }
  if (indptr[0] != 0) { err = "indptr must start at 0"; return TR_ERR_ARG; }
  for (int32_t r = 0; r < n_rows; ++r)
    if (indptr[r + 1] < indptr[r]) { err = "indptr must be non-decreasing"; return TR_ERR_ARG; }
  const int64_t nnz = indptr[n_rows];
  if (nnz > 0 && !indices) { err = "null indices"; return TR_ERR_ARG; }
  for (int64_t e = 0; e < nnz; ++e)
    if (indices[e] < 0 || indices[e] >= n_cols) { err = "column index out of range"; return TR_ERR_ARG; }
  return TR_OK;
}

namespace {

// A^T as CSR, entries of each row of A^T in A's row order (a stable counting
// sort by column).  Host threads take contiguous ranges of A's rows, count
// their entries per column, and scatter from per-(column, thread) offsets, so
// the result is the sequential one.
void transpose(const Csr& a, Csr& t) {
  t.n_rows = a.n_cols;
  t.n_cols = a.n_rows;
  const int64_t nnz = (int64_t)a.idx.size();
  const int32_t C = a.n_cols, R = a.n_rows;
  t.ptr.assign((size_t)C + 1, 0);
  t.idx.resize(nnz);
  t.val.resize(nnz);
  t.src.resize(nnz);
  int T = (int)std::max(1u, std::thread::hardware_concurrency());
  T = (int)std::min<int64_t>(T, std::max<int64_t>(1, nnz / 65536));
  while (T > 1 && (int64_t)T * C > ((int64_t)1 << 26)) --T;      // per-thread counts fit
  std::vector<int32_t> r_at(T + 1);
  {
    int32_t r = 0;                          // row ranges of about nnz / T entries
    for (int k = 0; k <= T; ++k) {
      const int64_t want = nnz * k / T;
      while (r < R && a.ptr[r] < want) ++r;
      r_at[k] = k == T ? R : r;
    }
  }
  std::vector<std::vector<int32_t>> off(T, std::vector<int32_t>((size_t)C, 0));
  auto run = [&](auto body) {
    std::vector<std::thread> pool;
    for (int k = 1; k < T; ++k) pool.emplace_back(body, k);
    body(0);
    for (auto& th : pool) th.join();
  };
  run([&](int k) {
    for (int32_t r = r_at[k]; r < r_at[k + 1]; ++r)
      for (int32_t e = a.ptr[r]; e < a.ptr[r + 1]; ++e) off[k][a.idx[e]]++;
  });
  int32_t base = 0;
  for (int32_t c = 0; c < C; ++c) {
    t.ptr[c] = base;
    for (int k = 0; k < T; ++k) {
      const int32_t n = off[k][c];
      off[k][c] = base;
      base += n;
    }
  }
  t.ptr[C] = base;
  run([&](int k) {
    std::vector<int32_t>& fill = off[k];
    for (int32_t r = r_at[k]; r < r_at[k + 1]; ++r)
      for (int32_t e = a.ptr[r]; e < a.ptr[r + 1]; ++e) {
        const int32_t at = fill[a.idx[e]]++;
        t.idx[at] = r;
        t.val[at] = a.val[e];
        t.src[at] = a.src[e];
      }
  });
}

inline uint32_t mix32(uint32_t x) {
  x ^= x >> 16; x *= 0x7feb352dU;
  x ^= x >> 15; x *= 0x846ca68bU;
  x ^= x >> 16;
  return x;
}

// Per-label vote sums of one row: label-indexed sums (all zero between rows)
// and the labels that received votes.  Vote weights are positive, so a zero
// sum marks a label that has not been touched yet.
struct VoteAcc {
  std::vector<float> w;
  std::vector<int32_t> touched;

  void add(int32_t label, float v) {
    if (w[label] == 0.f) touched.push_back(label);
    w[label] += v;
  }
  bool empty() const { return touched.empty(); }

  // Label with the largest summed vote among those with room (size < cap),
  // the current label winning ties and otherwise the smallest label among
  // equal sums; clears the sums for the next row.  One pass in arrival
  // order: the tie rule is explicit, so no sort of the touched labels.
  int32_t pick(int32_t cur, const std::vector<int32_t>& size, int32_t cap) {
    int32_t best = cur;
    float best_w = cur >= 0 ? w[cur] : 0.f;
    for (int32_t l : touched) {
      if (l == cur || size[l] >= cap) continue;
      const float x = w[l];
      if (x > best_w || (x == best_w && best != cur && l < best)) {
        best = l;
        best_w = x;
      }
    }
    for (int32_t l : touched) w[l] = 0.f;
    touched.clear();
    return best;
  }
};

}  // namespace

// Row order that clusters rows sharing columns: perm[new] = old.
//
// Asynchronous label propagation in a seeded visiting order.  Two changes
// keep hubs of power-law graphs from flooding every community with their
// label: a neighbour's vote weighs 1 / its degree (a hub is adjacent to many
// communities, so it says little about any one), and a label takes no new
// member once it holds `cap` rows.  Sweeps stop when fewer than 0.1% of rows
// change.  A square matrix is taken as a graph on one node set (row i and
// column i are the same node, in- and out-neighbours both vote); otherwise
// rows and columns carry separate labels and vote for each other.
void cluster_rows(const Csr& a, std::vector<int32_t>& perm, int sweeps, int32_t cap) {
  const int32_t R = a.n_rows, C = a.n_cols;
  perm.resize(R);
  std::iota(perm.begin(), perm.end(), 0);
  if (R <= 16 || a.idx.empty()) return;
  std::vector<int32_t> cptr((size_t)C + 1, 0), crow(a.idx.size());
  for (int32_t c : a.idx) cptr[c + 1]++;
  for (int32_t c = 0; c < C; ++c) cptr[c + 1] += cptr[c];
  {
    std::vector<int32_t> fill(cptr.begin(), cptr.end() - 1);
    for (int32_t r = 0; r < R; ++r)
      for (int32_t e = a.ptr[r]; e < a.ptr[r + 1]; ++e) crow[fill[a.idx[e]]++] = r;
  }
  const bool square = R == C;
  std::vector<float> rinv(R), cinv(C);
  for (int32_t r = 0; r < R; ++r) {
    const int32_t d = (a.ptr[r + 1] - a.ptr[r]) + (square ? cptr[r + 1] - cptr[r] : 0);
    rinv[r] = d > 0 ? 1.f / (float)d : 0.f;
  }
  for (int32_t c = 0; c < C; ++c) {
    const int32_t d = cptr[c + 1] - cptr[c];
    cinv[c] = d > 0 ? 1.f / (float)d : 0.f;
  }
  std::vector<int32_t> rlab(R), rsize(R, 1);
  std::iota(rlab.begin(), rlab.end(), 0);
  std::vector<int32_t> clab;
  if (!square) clab.assign(C, -1);
  std::vector<int32_t> order(R);
  std::iota(order.begin(), order.end(), 0);
  std::sort(order.begin(), order.end(), [](int32_t x, int32_t y) {
    const uint32_t hx = mix32((uint32_t)x * 2654435761u), hy = mix32((uint32_t)y * 2654435761u);
    return hx != hy ? hx < hy : x < y;
  });
  const std::vector<int32_t> no_size(R, 0);
  VoteAcc acc;
  acc.w.assign(R, 0.f);
  for (int s = 0; s < sweeps; ++s) {
    if (!square) {
      for (int32_t c = 0; c < C; ++c) {
        for (int32_t e = cptr[c]; e < cptr[c + 1]; ++e) acc.add(rlab[crow[e]], rinv[crow[e]]);
        clab[c] = acc.empty() ? -1 : acc.pick(-1, no_size, INT32_MAX);
      }
    }
    int64_t changed = 0;
    for (int32_t r : order) {
      for (int32_t e = a.ptr[r]; e < a.ptr[r + 1]; ++e) {
        const int32_t c = a.idx[e];
        if (square) {
          if (c != r) acc.add(rlab[c], rinv[c]);
        } else if (clab[c] >= 0) {
          acc.add(clab[c], cinv[c]);
        }
      }
      if (square)
        for (int32_t e = cptr[r]; e < cptr[r + 1]; ++e)
          if (crow[e] != r) acc.add(rlab[crow[e]], rinv[crow[e]]);
      const int32_t cur = rlab[r];
      const int32_t l = acc.pick(cur, rsize, cap);
      if (l != cur) {
        rsize[cur]--;
        rsize[l]++;
        rlab[r] = l;
        ++changed;
      }
    }
    if (changed * 1000 < R) break;
  }
  std::stable_sort(perm.begin(), perm.end(),
                   [&](int32_t x, int32_t y) { return rlab[x] < rlab[y]; });
}

namespace {

void permute_rows(const Csr& a, const std::vector<int32_t>& perm, Csr& p) {
  p.n_rows = a.n_rows;
  p.n_cols = a.n_cols;
  p.ptr.assign((size_t)a.n_rows + 1, 0);
  for (int32_t r = 0; r < a.n_rows; ++r) p.ptr[r + 1] = p.ptr[r] + (a.ptr[perm[r] + 1] - a.ptr[perm[r]]);
  const size_t nnz = a.idx.size();
  p.idx.resize(nnz);
  p.val.resize(nnz);
  p.src.resize(nnz);
  for (int32_t r = 0; r < a.n_rows; ++r) {
    const int32_t o = perm[r];
    std::copy(a.idx.begin() + a.ptr[o], a.idx.begin() + a.ptr[o + 1], p.idx.begin() + p.ptr[r]);
    std::copy(a.val.begin() + a.ptr[o], a.val.begin() + a.ptr[o + 1], p.val.begin() + p.ptr[r]);
    std::copy(a.src.begin() + a.ptr[o], a.src.begin() + a.ptr[o + 1], p.src.begin() + p.ptr[r]);
  }
}

}  // namespace

int build_plan(const int32_t* indptr, const int32_t* indices, const float* values, int32_t n_rows,
               int32_t n_cols, const tr_route_params& params, const tr_plan_opts& opts,
               HostPlan& hp, std::string& err) {
  int rc = validate_csr(indptr, indices, n_rows, n_cols, err);
  if (rc) return rc;
  if (opts.engine != TR_ENGINE_WINDOW && opts.engine != TR_ENGINE_BLOCK) {
    err = "unknown plan engine " + std::to_string(opts.engine);
    return TR_ERR_ARG;
  }
  const bool blocks = opts.engine == TR_ENGINE_BLOCK;
  if (!blocks && params.window != 16) { err = "routed plans need window == 16"; return TR_ERR_UNSUPPORTED; }
  if (opts.promote_min < 0) { err = "promote_min must be >= 0"; return TR_ERR_ARG; }
  if (opts.demote_below < 0) { err = "demote_below must be >= 0"; return TR_ERR_ARG; }
  const int64_t nnz = indptr[n_rows];
  if (nnz > INT32_MAX) { err = "more than 2^31 - 1 entries"; return TR_ERR_UNSUPPORTED; }
  Csr a;
  a.n_rows = n_rows;
  a.n_cols = n_cols;
  a.ptr.assign(indptr, indptr + n_rows + 1);
  a.idx.assign(indices, indices + nnz);
  a.val.resize(nnz);
  for (int64_t e = 0; e < nnz; ++e) a.val[e] = values ? values[e] : 1.0f;
  a.src.resize(nnz);
  std::iota(a.src.begin(), a.src.end(), 0);
  if (opts.transpose) {
    Csr t;
    transpose(a, t);
    a = std::move(t);
  }
  if (opts.reorder < TR_REORDER_NONE || opts.reorder > TR_REORDER_GIVEN) {
    err = "unknown reorder mode " + std::to_string(opts.reorder);
    return TR_ERR_ARG;
  }
  std::vector<int32_t> perm;
  if (opts.reorder == TR_REORDER_LABEL) {
    cluster_rows(a, perm, 8, 256);
  } else if (opts.reorder == TR_REORDER_TCA) {
    TcaParams tp;
    TcaStats ts;
    rc = tca_order(a.ptr.data(), a.idx.data(), a.n_rows, tp, perm, ts, err);
    if (rc) return rc;
  } else if (opts.reorder == TR_REORDER_GIVEN) {
    if (!opts.row_order && a.n_rows > 0) { err = "TR_REORDER_GIVEN needs row_order"; return TR_ERR_ARG; }
    perm.assign(opts.row_order, opts.row_order + a.n_rows);
    std::vector<char> seen(a.n_rows, 0);
    for (int32_t r : perm) {
      if (r < 0 || r >= a.n_rows || seen[r]) { err = "row_order is not a permutation of the rows"; return TR_ERR_ARG; }
      seen[r] = 1;
    }
  }
  if (opts.reorder) {
    Csr p;
    permute_rows(a, perm, p);
    a = std::move(p);
  }
  if (blocks) {
    rc = plan_blocks(a, opts.row_scale != 0, nnz, hp, err);
    if (rc) return rc;
    if (opts.reorder)
      for (size_t r = 0; r < perm.size(); ++r) hp.row_out[r] = perm[r];
    hp.reordered = opts.reorder != 0;
    return TR_OK;
  }
  RouteTables T;
  // every 2:4 column would be demoted: form no 2:4 groups at all (the same
  // tiles and matrix; the residual keeps each row's entries in CSR order)
  tr_route_params rp = params;
  if (opts.demote_below > 16) rp.skip_sptc = 1;
  rc = build_route(a.ptr.data(), a.idx.data(), a.val.data(), a.n_rows, rp, T, err);
  if (rc) return rc;
  PlanOptions po;
  po.row_scale = opts.row_scale != 0;
  po.promote_min = opts.promote_min;
  po.demote_below = opts.demote_below;
  rc = plan_from_route(T, a.n_rows, a.n_cols, nnz, po, hp, err);
  if (rc) return rc;
  // entry indices of the routed matrix -> entries of the caller's A
  std::vector<int32_t> slot(nnz, -1), erow(nnz, -1);
  for (int64_t e = 0; e < nnz; ++e) {
    slot[a.src[e]] = hp.val_slot[e];
    erow[a.src[e]] = hp.edge_row[e];
  }
  hp.val_slot.swap(slot);
  hp.edge_row.swap(erow);
  for (int32_t& e : hp.res_edge)
    if (e >= 0) e = a.src[e];
  if (opts.reorder)
    for (size_t r = 0; r < perm.size(); ++r) hp.row_out[r] = perm[r];
  hp.reordered = opts.reorder != 0;
  return TR_OK;
}

int label_order(const int32_t* indptr, const int32_t* indices, int32_t n_rows, int32_t n_cols,
                bool transpose_first, int32_t* order, std::string& err) {
  int rc = validate_csr(indptr, indices, n_rows, n_cols, err);
  if (rc) return rc;
  const int64_t nnz = indptr[n_rows];
  if (nnz > INT32_MAX) { err = "more than 2^31 - 1 entries"; return TR_ERR_UNSUPPORTED; }
  Csr a;
  a.n_rows = n_rows;
  a.n_cols = n_cols;
  a.ptr.assign(indptr, indptr + n_rows + 1);
  a.idx.assign(indices, indices + nnz);
  a.val.assign(nnz, 1.0f);
  a.src.resize(nnz);
  std::iota(a.src.begin(), a.src.end(), 0);
  if (transpose_first) {
    Csr t;
    transpose(a, t);
    a = std::move(t);
  }
  std::vector<int32_t> perm;
  cluster_rows(a, perm, 8, 256);     // the same call as build_plan's TR_REORDER_LABEL
  std::copy(perm.begin(), perm.end(), order);
  return TR_OK;
}

}  // namespace trs
