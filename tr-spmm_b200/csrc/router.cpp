// Three-stage funnel router over 16-row windows, multi-threaded host C++.
//
// Produces the reference's 29 route tables (TR-source/Block/block_online.cpp,
// return list :844-870) from a CSR matrix.  Decisions follow the reference
// exactly in TR_ROUTE_COMPAT mode; TR_ROUTE_EXACT keeps every decision and
// additionally sends the entries the reference drops (the third and fourth
// entry of a row inside a 4-column SPTC group, block_online.cpp:688-693, and
// repeated (row, column) entries) to the CUDA-core residual.
//
// Design (differs from the reference, same results):
//  * per window, one sort of (column, edge) keys gives every column's profile
//    (count, 2-bit row vector, first edge per row) without hash maps;
//  * candidate orders (count desc, column asc) come from a counting sort
//    (count <= 16), which is the total order the reference's comparators
//    define (block_online.cpp:226-230, :285-289);
//  * the unit conflict test (block_online.cpp:85-88) can only fail when a
//    2-bit row field reaches 2, which a deduplicated column never produces,
//    so the compatibility graph of :342-351 is complete in practice; the
//    matcher then needs no O(u^2) graph: the processing order is the same
//    std::sort call on the same comparator outcomes (:360-363), and "unmatched
//    neighbour of maximum degree, ties to larger nnz, first index wins"
//    (:370-377) becomes "first unmatched unit in (nnz desc, index asc) order",
//    kept in a linked list.  The general O(u^2) path is kept for inputs with
//    odd bits set;
//  * windows are processed in parallel chunks and concatenated in window
//    order.
#include <algorithm>
#include <functional>
#include <array>
#include <atomic>
#include <chrono>
#include <cstdint>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "router.h"
#include "unit_order.h"

namespace trs {
namespace {

constexpr uint32_t kOddBits = 0xaaaaaaaau;

inline bool units_compatible(uint32_t a, uint32_t b) {
  const uint32_t c = a | b;
  return (((a & b) | ((c << 1) & c)) & kOddBits) == 0;
}

inline uint16_t f32_to_f16_bits(float f) {
  _Float16 h = (_Float16)f;   // IEEE round-to-nearest-even (as c10::Half)
  uint16_t b;
  std::memcpy(&b, &h, 2);
  return b;
}

struct ColProfile {
  int col;
  int count;
  uint32_t vec;
  int first_edge[16];   // local edge index of the first entry per local row, -1 if none
  int route;            // 0 cuda, 1 tc, 2 sptc
  int tc_slot;          // block*8 + pos when route == tc
};

struct Unit {
  int p1, p2;           // profile indices (p2 = -1: single column)
  uint32_t vec;
  int nnz;
};

// Per-chunk output; same fields as RouteTables, offsets chunk-local.
struct Chunk {
  std::vector<int32_t> t_parts, t_subcounts, t_column, t_window_row, t_atomic;
  std::vector<float> t_value;
  std::vector<int64_t> t_binary;
  std::vector<int32_t> c_counts, c_row, c_atomic, c_column;
  std::vector<float> c_value;
  std::vector<int32_t> cs_counts, cs_row, cs_atomic, cs_column;
  std::vector<float> cs_value;
  std::vector<int32_t> s_column, s_window, s_groups_per_window;
  std::vector<uint8_t> s_mask;
  std::vector<float> s_value;
  std::vector<int8_t> s_pos;
  std::vector<int32_t> s_tile_window, s_tile_group_local, s_tile_column, s_packed_a,
      s_packed_meta, s_tiles_per_window;
  std::vector<int32_t> t_edge, s_edge, c_edge, cs_edge;
  int64_t lost = 0;
};

struct Scratch {
  std::vector<uint64_t> keys;
  std::vector<ColProfile> prof;
  std::vector<int> edge_prof;      // local edge -> profile index
  std::vector<uint8_t> edge_route; // local edge -> 0 cuda / 1 tc / 2 sptc
  std::vector<int8_t> edge_row;
  std::vector<int> cand, tmp;
  std::vector<Unit> units;
  std::vector<int> order, list_next, list_prev, sorted_units, unit_nnz;
  std::vector<char> matched;
  std::vector<std::pair<int, int>> pairs;
  std::vector<int> unmatched;
  std::vector<std::array<int, 4>> groups;   // profile indices, -1 padded
  std::vector<int> rc;                      // residual columns of one row
  std::vector<float> rv;
  std::vector<int> re;                      // their CSR entry ids
};

// Candidate order of block_online.cpp:226-230 / :285-289 (count desc, column
// asc) by counting sort; profiles arrive sorted by column.
void order_by_count(const std::vector<ColProfile>& prof, std::vector<int>& idx,
                    std::vector<int>& out) {
  int buckets[17] = {0};
  for (int i : idx) buckets[prof[i].count]++;
  int start[17];
  int s = 0;
  for (int c = 16; c >= 0; --c) { start[c] = s; s += buckets[c]; }
  out.resize(idx.size());
  for (int i : idx) out[start[prof[i].count]++] = i;
}

void split_residual_row(int row, int base_atomic, int part, int shortsz,
                        const std::vector<int>& cols, const std::vector<float>& vals,
                        const std::vector<int>& edges, Chunk& ck) {
  const int n = (int)cols.size();
  auto emit = [&](int atomic, int off, int cnt, bool small) {
    auto& counts = small ? ck.cs_counts : ck.c_counts;
    auto& rows = small ? ck.cs_row : ck.c_row;
    auto& ats = small ? ck.cs_atomic : ck.c_atomic;
    auto& cc = small ? ck.cs_column : ck.c_column;
    auto& vv = small ? ck.cs_value : ck.c_value;
    auto& ee = small ? ck.cs_edge : ck.c_edge;
    counts.push_back(cnt);
    rows.push_back(row);
    ats.push_back(atomic);
    cc.insert(cc.end(), cols.begin() + off, cols.begin() + off + cnt);
    vv.insert(vv.end(), vals.begin() + off, vals.begin() + off + cnt);
    ee.insert(ee.end(), edges.begin() + off, edges.begin() + off + cnt);
  };
  if (n <= 0) return;
  if (n <= shortsz) { emit(base_atomic, 0, n, true); return; }
  if (n <= part) { emit(base_atomic, 0, n, false); return; }
  int off = 0;
  for (int i = 0; i < n / part; ++i) { emit(1, off, part, false); off += part; }
  const int rem = n % part;
  if (rem > 0) emit(1, off, rem, rem <= shortsz);
}

void route_window(const int32_t* indptr, const int32_t* indices, const float* values,
                  int n_rows, int w, const tr_route_params& p, Scratch& S, Chunk& ck) {
  const int window = p.window;
  const bool exact = p.mode == TR_ROUTE_EXACT;
  const int r0 = w * window, r1 = std::min(r0 + window, n_rows);
  const int e0 = indptr[r0], e1 = indptr[r1];
  const int ne = e1 - e0;

  // ---- column profile (block_online.cpp:589-603) -------------------------
  S.keys.resize(ne);
  for (int e = e0; e < e1; ++e)
    S.keys[e - e0] = ((uint64_t)(uint32_t)indices[e] << 32) | (uint32_t)(e - e0);
  std::sort(S.keys.begin(), S.keys.end());
  S.prof.clear();
  S.edge_prof.assign(ne, -1);
  S.edge_route.assign(ne, 0);
  std::vector<int8_t>& edge_row = S.edge_row;   // local edge -> local row
  edge_row.resize(ne);
  for (int r = r0; r < r1; ++r)
    for (int e = indptr[r]; e < indptr[r + 1]; ++e) edge_row[e - e0] = (int8_t)(r - r0);
  for (int i = 0; i < ne;) {
    const int c = (int)(S.keys[i] >> 32);
    ColProfile cp;
    cp.col = c; cp.count = 0; cp.vec = 0; cp.route = 0; cp.tc_slot = -1;
    for (int k = 0; k < 16; ++k) cp.first_edge[k] = -1;
    const int pi = (int)S.prof.size();
    int j = i;
    for (; j < ne && (int)(S.keys[j] >> 32) == c; ++j) {
      const int le = (int)(uint32_t)S.keys[j];
      const int lr = edge_row[le];
      S.edge_prof[le] = pi;
      if (cp.first_edge[lr] < 0) {        // keys ascend by edge: first hit per row
        cp.first_edge[lr] = le;
        cp.count++;
        cp.vec += 1u << (2 * lr);
      }
    }
    S.prof.push_back(cp);
    i = j;
  }
  auto& prof = S.prof;
  const int np = (int)prof.size();

  // ---- stage 1: TC funnel (block_online.cpp:215-253) ----------------------
  std::vector<std::array<int, 8>> tc_groups;
  if (!p.skip_tc) {
    S.tmp.clear();
    for (int i = 0; i < np; ++i) if (prof[i].count >= p.density) S.tmp.push_back(i);
    order_by_count(prof, S.tmp, S.cand);
    for (size_t s = 0; s < S.cand.size(); s += 8) {
      const size_t e = std::min(s + 8, S.cand.size());
      int nnz = 0;
      for (size_t i = s; i < e; ++i) nnz += prof[S.cand[i]].count;
      const float util = (float)nnz / (float)(window * 8);
      if (util < p.tc_min_util) continue;
      std::array<int, 8> g;
      g.fill(-1);
      int n = 0;
      for (size_t i = s; i < e; ++i) g[n++] = S.cand[i];
      for (int i = 1; i < n; ++i)                    // sort <= 8 columns ascending
        for (int j = i; j > 0 && prof[g[j - 1]].col > prof[g[j]].col; --j) std::swap(g[j - 1], g[j]);
      const int blk = (int)tc_groups.size();
      for (int k = 0; k < n; ++k) { prof[g[k]].route = 1; prof[g[k]].tc_slot = blk * 8 + k; }
      tc_groups.push_back(g);
    }
  }

  // ---- stage 2a: units (block_online.cpp:267-328) -------------------------
  // (skip_sptc: no candidates, so no units, pairs or groups; the columns
  // outside the TC funnel keep route 0 and go to the CUDA parts)
  S.tmp.clear();
  uint32_t any_odd = 0;
  for (int i = 0; i < np && !p.skip_sptc; ++i)
    if (prof[i].route != 1) { S.tmp.push_back(i); any_odd |= prof[i].vec & kOddBits; }
  order_by_count(prof, S.tmp, S.cand);
  S.units.clear();
  if (!any_odd) {
    // Every pair is compatible: each column pairs with the next unused one.
    for (size_t i = 0; i < S.cand.size(); i += 2) {
      const ColProfile& a = prof[S.cand[i]];
      if (i + 1 < S.cand.size()) {
        const ColProfile& b = prof[S.cand[i + 1]];
        S.units.push_back({S.cand[i], S.cand[i + 1], a.vec | b.vec, a.count + b.count});
      } else {
        S.units.push_back({S.cand[i], -1, a.vec, a.count});
      }
    }
  } else {
    std::vector<char> used(S.cand.size(), 0);
    for (size_t i = 0; i < S.cand.size(); ++i) {
      if (used[i]) continue;
      used[i] = 1;
      const ColProfile& a = prof[S.cand[i]];
      long j = -1;
      for (size_t k = i + 1; k < S.cand.size(); ++k)
        if (!used[k] && units_compatible(a.vec, prof[S.cand[k]].vec)) { j = (long)k; break; }
      if (j >= 0) {
        used[j] = 1;
        const ColProfile& b = prof[S.cand[j]];
        S.units.push_back({S.cand[i], S.cand[j], a.vec | b.vec, a.count + b.count});
      } else {
        S.units.push_back({S.cand[i], -1, a.vec, a.count});
      }
    }
  }

  // ---- stage 2b: max-degree matching (block_online.cpp:332-392) ----------
  const int nu = (int)S.units.size();
  S.pairs.clear();
  S.unmatched.clear();
  S.matched.assign(nu, 0);
  S.order.resize(nu);
  for (int i = 0; i < nu; ++i) S.order[i] = i;
  uint32_t unit_odd = 0;
  for (auto& u : S.units) unit_odd |= u.vec & kOddBits;
  if (!unit_odd) {
    // Complete compatibility graph: all degrees equal nu-1, so the
    // reference comparator reduces to nnz descending.  unit_order performs
    // the reference's std::sort step for step (the device router runs the
    // same function), so ties land where they land there.
    S.unit_nnz.resize(nu);
    for (int i = 0; i < nu; ++i) S.unit_nnz[i] = S.units[i].nnz;
    unit_order(S.order.data(), nu, S.unit_nnz.data());
    // Units by (nnz desc, index asc) in a doubly linked list of the unmatched.
    int buckets[33] = {0};
    for (auto& u : S.units) buckets[u.nnz]++;
    int start[33];
    int s = 0;
    for (int c = 32; c >= 0; --c) { start[c] = s; s += buckets[c]; }
    S.sorted_units.resize(nu);
    for (int i = 0; i < nu; ++i) S.sorted_units[start[S.units[i].nnz]++] = i;
    std::vector<int> pos(nu);
    for (int i = 0; i < nu; ++i) pos[S.sorted_units[i]] = i;
    S.list_next.resize(nu + 1);
    S.list_prev.resize(nu + 1);
    for (int i = 0; i < nu; ++i) { S.list_next[i] = i + 1; S.list_prev[i] = i - 1; }
    int head = nu > 0 ? 0 : nu;
    auto unlink = [&](int slot) {
      const int pv = S.list_prev[slot], nx = S.list_next[slot];
      if (pv >= 0) S.list_next[pv] = nx; else head = nx;
      if (nx < nu) S.list_prev[nx] = pv;
    };
    for (int idx : S.order) {
      if (S.matched[idx]) continue;
      int slot = head;
      if (slot < nu && S.sorted_units[slot] == idx) slot = S.list_next[slot];
      if (slot >= nu) continue;                       // no unmatched neighbour
      const int best = S.sorted_units[slot];
      S.matched[idx] = 1; S.matched[best] = 1;
      unlink(pos[idx]); unlink(slot);
      S.pairs.emplace_back(idx, best);
    }
  } else {
    std::vector<std::vector<int>> adj(nu);
    std::vector<int> deg(nu, 0);
    for (int i = 0; i < nu; ++i)
      for (int j = i + 1; j < nu; ++j)
        if (units_compatible(S.units[i].vec, S.units[j].vec)) {
          adj[i].push_back(j); adj[j].push_back(i); deg[i]++; deg[j]++;
        }
    std::sort(S.order.begin(), S.order.end(), [&](int a, int b) {
      if (deg[a] != deg[b]) return deg[a] > deg[b];
      return S.units[a].nnz > S.units[b].nnz;
    });
    for (int idx : S.order) {
      if (S.matched[idx]) continue;
      int best = -1, bd = -1;
      for (int nb : adj[idx]) {
        if (S.matched[nb]) continue;
        if (deg[nb] > bd || (deg[nb] == bd && S.units[nb].nnz > S.units[best].nnz)) {
          best = nb; bd = deg[nb];
        }
      }
      if (best >= 0) { S.matched[idx] = 1; S.matched[best] = 1; S.pairs.emplace_back(idx, best); }
    }
  }
  for (int i = 0; i < nu; ++i) if (!S.matched[i]) S.unmatched.push_back(i);

  // ---- stage 2c: SPTC groups + per-row metadata (block_online.cpp:629-702)
  S.groups.clear();
  auto add_group = [&](int a, int b, int c, int d) {
    std::array<int, 4> g{a, b, c, d};
    int n = 0;
    for (int x : g) if (x >= 0) g[n++] = x;
    for (int k = n; k < 4; ++k) g[k] = -1;
    for (int i = 1; i < n; ++i)                      // sort <= 4 columns ascending
      for (int j = i; j > 0 && prof[g[j - 1]].col > prof[g[j]].col; --j) std::swap(g[j - 1], g[j]);
    for (int k = 0; k < n; ++k) prof[g[k]].route = 2;
    S.groups.push_back(g);
  };
  for (auto& pr : S.pairs) {
    const Unit& a = S.units[pr.first];
    const Unit& b = S.units[pr.second];
    add_group(a.p1, a.p2, b.p1, b.p2);
  }
  for (int idx : S.unmatched) {
    const Unit& u = S.units[idx];
    if (u.nnz < p.unit_min_nnz) continue;
    add_group(u.p1, u.p2, -1, -1);
  }
  const int ng = (int)S.groups.size();
  const size_t g_base_local = ck.s_window.size();
  for (int gi = 0; gi < ng; ++gi) {
    const auto& g = S.groups[gi];
    ck.s_window.push_back(w);
    for (int k = 0; k < 4; ++k) ck.s_column.push_back(g[k] >= 0 ? prof[g[k]].col : -1);
    for (int lr = 0; lr < window; ++lr) {
      uint8_t mask = 0;
      int slots = 0;
      float v[2] = {0.f, 0.f};
      int8_t ps[2] = {-1, -1};
      int32_t ed[2] = {-1, -1};
      for (int k = 0; k < 4 && g[k] >= 0; ++k) {
        const int le = lr < 16 ? prof[g[k]].first_edge[lr] : -1;
        if (le < 0) continue;
        mask |= (uint8_t)(1u << k);
        if (slots < 2) {
          v[slots] = values[e0 + le];
          ps[slots] = (int8_t)k;
          ed[slots] = e0 + le;
          S.edge_route[le] = 2;
        } else {
          ck.lost++;                                   // dropped by the reference
        }
        slots++;
      }
      ck.s_mask.push_back(mask);
      ck.s_value.push_back(v[0]); ck.s_value.push_back(v[1]);
      ck.s_pos.push_back(ps[0]); ck.s_pos.push_back(ps[1]);
      ck.s_edge.push_back(ed[0]); ck.s_edge.push_back(ed[1]);
    }
  }
  ck.s_groups_per_window.push_back(ng);

  // ---- edge routes --------------------------------------------------------
  // compat: an edge follows its column's route (block_online.cpp:724, :467).
  // exact:  TC / SPTC keep only the first entry of each (row, column); the
  //         rest, and SPTC entries beyond two per row and group, go to CUDA.
  bool has_cuda = false;
  for (int le = 0; le < ne; ++le) {
    const ColProfile& cp = prof[S.edge_prof[le]];
    if (!exact) {
      S.edge_route[le] = (uint8_t)cp.route;
    } else if (cp.route == 1) {
      S.edge_route[le] = cp.first_edge[edge_row[le]] == le ? 1 : 0;
    } else if (cp.route == 2) {
      // set above for kept entries; everything else stays 0 (CUDA)
    } else {
      S.edge_route[le] = 0;
    }
  }
  for (int i = 0; i < np; ++i) if (prof[i].route == 0) has_cuda = true;
  if (exact && !has_cuda)
    for (int le = 0; le < ne; ++le) if (S.edge_route[le] == 0) { has_cuda = true; break; }

  // ---- TC sub-blocks (block_online.cpp:444-540) ---------------------------
  if (!tc_groups.empty()) {
    const int nsub = (int)tc_groups.size();
    const size_t val_base = ck.t_value.size();
    std::vector<uint64_t> lo(nsub, 0), hi(nsub, 0);
    std::vector<std::vector<float>> sv(nsub);
    std::vector<std::vector<int32_t>> se(nsub);
    for (int r = r0; r < r1; ++r) {
      const int lr = r - r0;
      for (int e = indptr[r]; e < indptr[r + 1]; ++e) {
        const int le = e - e0;
        if (S.edge_route[le] != 1) continue;
        const int slot = prof[S.edge_prof[le]].tc_slot;
        const int k = slot % 8, s = slot / 8;
        if (lr >= 8) hi[s] |= 1ull << ((lr - 8) * 8 + k);
        else lo[s] |= 1ull << (lr * 8 + k);
        sv[s].push_back(values[e]);
        se[s].push_back(e);
      }
    }
    (void)val_base;
    for (int s = 0; s < nsub; ++s) {
      for (int k = 0; k < 8; ++k) {
        const int pi = tc_groups[s][k];
        ck.t_column.push_back(pi >= 0 ? prof[pi].col : -1);
      }
      ck.t_binary.push_back((int64_t)lo[s]);
      ck.t_binary.push_back((int64_t)hi[s]);
      ck.t_value.insert(ck.t_value.end(), sv[s].begin(), sv[s].end());
      ck.t_edge.insert(ck.t_edge.end(), se[s].begin(), se[s].end());
    }
    auto part = [&](int first, int cnt, int atomic) {
      ck.t_parts.push_back(cnt);
      for (int s = first; s < first + cnt; ++s) ck.t_subcounts.push_back((int)sv[s].size());
      ck.t_window_row.push_back(w * 16);
      ck.t_atomic.push_back(atomic);
    };
    const int pt = p.partsize_t;
    if (nsub <= pt) {
      part(0, nsub, has_cuda ? 1 : 0);
    } else {
      for (int q = 0; q < nsub / pt; ++q) part(q * pt, pt, 1);
      if (nsub % pt) part(nsub - nsub % pt, nsub % pt, 1);
    }
  }

  // ---- CUDA residual (block_online.cpp:721-731) ---------------------------
  const int base_atomic = tc_groups.empty() ? 0 : 1;
  for (int r = r0; r < r1; ++r) {
    S.rc.clear(); S.rv.clear(); S.re.clear();
    for (int e = indptr[r]; e < indptr[r + 1]; ++e) {
      if (S.edge_route[e - e0] != 0) continue;
      S.rc.push_back(indices[e]);
      S.rv.push_back(values[e]);
      S.re.push_back(e);
    }
    split_residual_row(r, base_atomic, p.partsize_c, p.shortsize, S.rc, S.rv, S.re, ck);
  }

  // ---- mma.sp tile packing (block_online.cpp:797-841) ---------------------
  int tiles = 0;
  auto chunk_of = [&](int gl, int row, float& v0, float& v1, int& p0, int& p1) {
    // block_online.cpp:190-210; gl is chunk-local group index
    v0 = 0.f; v1 = 0.f; p0 = 0; p1 = 1;
    if (gl >= (int)(g_base_local + ng) || row >= window) return;
    const size_t b = ((size_t)gl * window + row) * 2;
    const int q0 = ck.s_pos[b], q1 = ck.s_pos[b + 1];
    const float w0 = ck.s_value[b], w1 = ck.s_value[b + 1];
    if (q0 < 0 && q1 < 0) return;
    if (q0 >= 0 && q1 >= 0) {
      if (q0 <= q1) { p0 = q0; p1 = q1; v0 = w0; v1 = w1; }
      else { p0 = q1; p1 = q0; v0 = w1; v1 = w0; }
      return;
    }
    const int rp = q0 >= 0 ? q0 : q1;
    const float rv = q0 >= 0 ? w0 : w1;
    const int dummy = rp == 0 ? 1 : 0;
    if (dummy < rp) { p0 = dummy; p1 = rp; v0 = 0.f; v1 = rv; }
    else { p0 = rp; p1 = dummy; v0 = rv; v1 = 0.f; }
  };
  const int gend = (int)(g_base_local + ng);
  for (int g0 = (int)g_base_local; g0 < gend; g0 += 4) {
    ck.s_tile_window.push_back(w);
    ck.s_tile_group_local.push_back(g0);
    for (int k = 0; k < 16; ++k) {
      const int g = g0 + (k >> 2);
      ck.s_tile_column.push_back(g < gend ? ck.s_column[(size_t)g * 4 + (k & 3)] : -1);
    }
    for (int rg = 0; rg < 8; ++rg) {
      float lo[8], hi[8];
      int pl0[4], pl1[4], ph0[4], ph1[4];
      for (int chn = 0; chn < 4; ++chn) {
        float v0, v1; int q0, q1;
        chunk_of(g0 + chn, rg, v0, v1, q0, q1);
        lo[2 * chn] = v0; lo[2 * chn + 1] = v1; pl0[chn] = q0; pl1[chn] = q1;
        chunk_of(g0 + chn, rg + 8, v0, v1, q0, q1);
        hi[2 * chn] = v0; hi[2 * chn + 1] = v1; ph0[chn] = q0; ph1[chn] = q1;
      }
      uint32_t meta = 0;
      for (int chn = 0; chn < 4; ++chn) {
        meta |= ((uint32_t)(pl0[chn] & 3) | ((uint32_t)(pl1[chn] & 3) << 2)) << (chn * 4);
        meta |= ((uint32_t)(ph0[chn] & 3) | ((uint32_t)(ph1[chn] & 3) << 2)) << (16 + chn * 4);
      }
      ck.s_packed_meta.push_back((int32_t)meta);
      for (int t = 0; t < 4; ++t) {
        ck.s_packed_a.push_back((int32_t)((uint32_t)f32_to_f16_bits(lo[2 * t]) |
                                          ((uint32_t)f32_to_f16_bits(lo[2 * t + 1]) << 16)));
        ck.s_packed_a.push_back((int32_t)((uint32_t)f32_to_f16_bits(hi[2 * t]) |
                                          ((uint32_t)f32_to_f16_bits(hi[2 * t + 1]) << 16)));
      }
    }
    tiles++;
  }
  ck.s_tiles_per_window.push_back(tiles);
}

template <typename T>
void append(std::vector<T>& dst, const std::vector<T>& src) {
  dst.insert(dst.end(), src.begin(), src.end());
}

void prefix_append(std::vector<int32_t>& dst, const std::vector<int32_t>& counts) {
  int64_t b = dst.back();
  for (int32_t c : counts) { b += c; dst.push_back((int32_t)b); }
}

// dst += the field `get` of every chunk, in chunk order: sized once, then
// copied (each chunk's field is released after its copy).
template <typename T, typename Get>
void concat(std::vector<T>& dst, std::vector<Chunk>& chunks, Get get) {
  size_t total = dst.size();
  for (auto& ck : chunks) total += get(ck).size();
  size_t at = dst.size();
  dst.resize(total);
  for (auto& ck : chunks) {
    std::vector<T>& v = get(ck);
    std::copy(v.begin(), v.end(), dst.begin() + at);
    at += v.size();
    std::vector<T>().swap(v);
  }
}

}  // namespace

int build_route(const int32_t* indptr, const int32_t* indices, const float* values,
                int32_t n_rows, const tr_route_params& p, RouteTables& out, std::string& err) {
  auto t0 = std::chrono::high_resolution_clock::now();
  if (n_rows < 0) { err = "n_rows must be >= 0"; return TR_ERR_ARG; }
  if (!(p.window > 0 && p.window <= 32 && p.wide > 0 && p.wide <= 32)) {
    err = "window and wide must be in (0, 32]";               // block_online.cpp:553
    return TR_ERR_ARG;
  }
  if (p.window > 16) {
    err = "window > 16 is not supported (the reference's 2-bit row vector overflows 32 bits)";
    return TR_ERR_UNSUPPORTED;
  }
  if (p.partsize_t <= 0 || p.partsize_c <= 0 || p.shortsize < 0) {
    err = "partsize_t / partsize_c must be positive and shortsize >= 0";
    return TR_ERR_ARG;
  }
  if (n_rows > 0 && indptr[0] != 0) { err = "row_ptr[0] must be 0"; return TR_ERR_ARG; }
  for (int32_t r = 0; r < n_rows; ++r)
    if (indptr[r + 1] < indptr[r]) { err = "row_ptr must be non-decreasing"; return TR_ERR_ARG; }
  const int64_t nnz = n_rows > 0 ? indptr[n_rows] : 0;
  for (int64_t e = 0; e < nnz; ++e)
    if (indices[e] < 0) { err = "column indices must be >= 0"; return TR_ERR_ARG; }

  const int nwin = (n_rows + p.window - 1) / p.window;
  const int per_chunk = 64;
  const int nchunks = (nwin + per_chunk - 1) / per_chunk;
  std::vector<Chunk> chunks(nchunks);
  int threads = p.threads > 0 ? p.threads : (int)std::thread::hardware_concurrency();
  threads = std::max(1, std::min(threads, std::max(1, nchunks)));
  std::atomic<int> next{0};
  auto worker = [&]() {
    Scratch S;
    for (;;) {
      const int c = next.fetch_add(1);
      if (c >= nchunks) break;
      const int w1 = std::min(nwin, (c + 1) * per_chunk);
      for (int w = c * per_chunk; w < w1; ++w)
        route_window(indptr, indices, values, n_rows, w, p, S, chunks[c]);
    }
  };
  if (threads == 1) {
    worker();
  } else {
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; ++t) pool.emplace_back(worker);
    for (auto& th : pool) th.join();
  }

  RouteTables& T = out;
  T = RouteTables();
  T.window = p.window;
  // offsets and counts in chunk order (small), then the large tables, each
  // concatenated on its own host thread (the same arrays as appending chunk
  // by chunk)
  int64_t group_base = 0;
  for (auto& ck : chunks) {
    prefix_append(T.t_row_offset, ck.t_parts);
    prefix_append(T.t_block_offset, ck.t_subcounts);
    prefix_append(T.c_row_offset, ck.c_counts);
    prefix_append(T.s_offsets, ck.s_groups_per_window);
    prefix_append(T.s_window_tile_offset, ck.s_tiles_per_window);
    for (int32_t g : ck.s_tile_group_local) T.s_tile_group.push_back((int32_t)(g + group_base));
    group_base += (int64_t)ck.s_window.size();
    T.dropped += ck.lost;
  }
  // the short residual parts follow all long ones (block_online.cpp:770-778)
  for (auto& ck : chunks) prefix_append(T.cs_row_offset, ck.cs_counts);
#define TRS_CAT(F) [&] { concat(T.F, chunks, [](Chunk& c) -> decltype(c.F)& { return c.F; }); }
  std::vector<std::function<void()>> tasks = {
      TRS_CAT(t_column),   TRS_CAT(t_value),      TRS_CAT(t_window_row), TRS_CAT(t_atomic),
      TRS_CAT(t_binary),   TRS_CAT(t_edge),       TRS_CAT(c_edge),       TRS_CAT(s_edge),
      TRS_CAT(c_row),      TRS_CAT(c_atomic),     TRS_CAT(c_column),     TRS_CAT(c_value),
      TRS_CAT(s_column),   TRS_CAT(s_mask),       TRS_CAT(s_value),      TRS_CAT(s_pos),
      TRS_CAT(s_window),   TRS_CAT(s_tile_window), TRS_CAT(s_tile_column), TRS_CAT(s_packed_a),
      TRS_CAT(s_packed_meta), TRS_CAT(cs_row),    TRS_CAT(cs_atomic),    TRS_CAT(cs_column),
      TRS_CAT(cs_value),   TRS_CAT(cs_edge)};
#undef TRS_CAT
  {
    std::atomic<size_t> next_task{0};
    auto run = [&]() {
      for (size_t i; (i = next_task.fetch_add(1)) < tasks.size();) tasks[i]();
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < threads; ++t) pool.emplace_back(run);
    run();
    for (auto& th : pool) th.join();
  }
  if (p.mode == TR_ROUTE_EXACT) T.dropped = 0;
  T.seconds = std::chrono::duration<double>(std::chrono::high_resolution_clock::now() - t0).count();
  return TR_OK;
}

}  // namespace trs
