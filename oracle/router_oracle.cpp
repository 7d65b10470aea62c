// ORACLE — test infrastructure only.  Nothing in the shipped library links,
// loads or calls this file; only tests/, the smoke check and bench.py's CPU
// baseline leg use it, and only as the checker.
//
// A plain, unoptimised CPU restatement of the reference's three-stage router
// `block_sptc_2to4_online` (TR-source/Block/block_online.cpp:545-871).  It
// produces the same 29 route tables in the same order (the 30th return of the
// reference, the wall-clock duration, is added by the Python wrapper).
// Every step cites the reference lines it restates.  Ties in the reference's
// unstable std::sort (block_online.cpp:360-363) are reproduced by calling
// std::sort with the same comparator on the same input sequence.
//
// Parity of this restatement is pinned against the reference router compiled
// from its own source (oracle/_ref, built by oracle/Makefile) and against the
// golden fixtures in tests/golden/.

#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <map>
#include <set>
#include <utility>
#include <vector>

namespace {

// One column's profile inside a row window (block_online.cpp:20-25, 589-603).
struct Profile {
  int count = 0;
  uint32_t vec = 0;                        // 2 bits per local row
  std::vector<std::pair<int, int>> hits;   // (local_row, edge id), first edge per row
};

struct Unit {                              // block_online.cpp:28-34
  int c1 = -1, c2 = -1;
  uint32_t vec = 0;
  int nnz = 0;
};

// Conflict test of block_online.cpp:85-88.
bool compatible(uint32_t a, uint32_t b) {
  const uint32_t c = a | b;
  return (((a & b) | ((c << 1) & c)) & 0xaaaaaaaau) == 0;
}

uint16_t half_bits(float f) {
  _Float16 h = (_Float16)f;               // round to nearest even, as c10::Half
  uint16_t b;
  std::memcpy(&b, &h, 2);
  return b;
}

struct CudaPart {                          // block_online.cpp:37-45
  int count, row, atomic;
  std::vector<int> cols;
  std::vector<float> vals;
};

struct Tables {
  // index order = the reference's return order (block_online.cpp:844-870)
  std::vector<int> t_row_offset{0}, t_block_offset{0}, t_column;
  std::vector<float> t_value;
  std::vector<int> t_window_row, t_atomic;
  std::vector<int64_t> t_binary;
  std::vector<int> c_row_offset{0}, c_row, c_atomic, c_column;
  std::vector<float> c_value;
  std::vector<int> cs_row_offset{0}, cs_row, cs_atomic, cs_column;
  std::vector<float> cs_value;
  std::vector<int> s_column;
  std::vector<uint8_t> s_mask;
  std::vector<float> s_value;
  std::vector<int8_t> s_pos;
  std::vector<int> s_window, s_offsets{0};
  std::vector<int> s_tile_window, s_tile_group, s_tile_column, s_packed_a, s_packed_meta;
  std::vector<int> s_window_tile_offset{0};
  int window = 16;
};

// split_cuda_row_online + append_cuda_part_online (block_online.cpp:397-439)
void split_row(int row, int base_atomic, int part, int shortsz,
               const std::vector<int>& cols, const std::vector<float>& vals,
               std::vector<CudaPart>& large, std::vector<CudaPart>& small) {
  const int n = (int)cols.size();
  auto emit = [&](int atomic, int off, int cnt, bool residue) {
    CudaPart p{cnt, row, atomic, {}, {}};
    p.cols.assign(cols.begin() + off, cols.begin() + off + cnt);
    p.vals.assign(vals.begin() + off, vals.begin() + off + cnt);
    (residue ? small : large).push_back(std::move(p));
  };
  if (n <= 0) return;
  if (n <= shortsz) { emit(base_atomic, 0, n, true); return; }
  if (n <= part) { emit(base_atomic, 0, n, false); return; }
  int off = 0;
  for (int i = 0; i < n / part; ++i) { emit(1, off, part, false); off += part; }
  const int rem = n % part;
  if (rem > 0) emit(1, off, rem, rem <= shortsz);
}

// load_sptc_row_chunk_cpu_online (block_online.cpp:190-210)
void row_chunk(const Tables& T, int g, int g_end, int row, int window,
               float& v0, float& v1, int& p0, int& p1) {
  v0 = 0.f; v1 = 0.f; p0 = 0; p1 = 1;
  if (g >= g_end || row >= window) return;
  const int b = (g * window + row) * 2;
  const int q0 = T.s_pos[b], q1 = T.s_pos[b + 1];
  const float w0 = T.s_value[b], w1 = T.s_value[b + 1];
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
}

void route(const int* rowptr, const int* col, const float* val, int rows,
           int part_t, int part_c, int shortsz, int density, int window,
           float tc_min_util, int unit_min_nnz, bool skip_tc, Tables& T) {
  T.window = window;
  const int nwin = (rows + window - 1) / window;
  const int tc_wide = 8;                                   // hard-coded, block_online.cpp:611
  struct CudaWin { std::vector<CudaPart> large, small; };
  std::vector<CudaWin> cuda(nwin);

  for (int w = 0; w < nwin; ++w) {
    const int r0 = w * window, r1 = std::min(r0 + window, rows);

    // a2: column profile (block_online.cpp:589-603)
    std::map<int, Profile> prof;
    for (int r = r0; r < r1; ++r) {
      std::set<int> seen;
      for (int e = rowptr[r]; e < rowptr[r + 1]; ++e) {
        const int c = col[e];
        if (!seen.insert(c).second) continue;
        Profile& p = prof[c];
        p.count += 1;
        p.vec += 1u << (2 * (r - r0));
        p.hits.emplace_back(r - r0, e);
      }
    }
    auto by_count = [&](int a, int b) {
      const int ca = prof[a].count, cb = prof[b].count;
      return ca != cb ? ca > cb : a < b;
    };

    // a3: TC funnel (block_online.cpp:215-253)
    std::set<int> tc_set;
    std::vector<std::vector<int>> tc_groups;
    if (!skip_tc) {
      std::vector<int> cand;
      for (auto& kv : prof) if (kv.second.count >= density) cand.push_back(kv.first);
      std::sort(cand.begin(), cand.end(), by_count);
      for (size_t s = 0; s < cand.size(); s += tc_wide) {
        const size_t e = std::min(s + (size_t)tc_wide, cand.size());
        int nnz = 0;
        std::vector<int> g;
        for (size_t i = s; i < e; ++i) { nnz += prof[cand[i]].count; g.push_back(cand[i]); }
        const float util = (float)nnz / (float)(window * tc_wide);
        if (util < tc_min_util) continue;
        std::sort(g.begin(), g.end());
        for (int c : g) tc_set.insert(c);
        tc_groups.push_back(g);
      }
    }

    // a4: unit build (block_online.cpp:267-328)
    std::vector<Unit> units;
    {
      std::vector<int> cand;
      for (auto& kv : prof) if (!tc_set.count(kv.first)) cand.push_back(kv.first);
      std::sort(cand.begin(), cand.end(), by_count);
      std::vector<char> used(cand.size(), 0);
      for (size_t i = 0; i < cand.size(); ++i) {
        if (used[i]) continue;
        used[i] = 1;
        const Profile& a = prof[cand[i]];
        long j = -1;
        for (size_t k = i + 1; k < cand.size(); ++k) {
          if (used[k]) continue;
          if (compatible(a.vec, prof[cand[k]].vec)) { j = (long)k; break; }
        }
        Unit u;
        u.c1 = cand[i];
        if (j >= 0) {
          used[j] = 1;
          const Profile& b = prof[cand[j]];
          u.c2 = cand[j]; u.vec = a.vec | b.vec; u.nnz = a.count + b.count;
        } else {
          u.vec = a.vec; u.nnz = a.count;
        }
        units.push_back(u);
      }
    }

    // a5: max-degree greedy matching (block_online.cpp:332-392)
    std::vector<std::pair<int, int>> pairs;
    std::vector<int> unmatched;
    {
      const int n = (int)units.size();
      std::vector<std::vector<int>> adj(n);
      std::vector<int> deg(n, 0);
      for (int i = 0; i < n; ++i)
        for (int j = i + 1; j < n; ++j)
          if (compatible(units[i].vec, units[j].vec)) {
            adj[i].push_back(j); adj[j].push_back(i); deg[i]++; deg[j]++;
          }
      std::vector<int> order(n);
      for (int i = 0; i < n; ++i) order[i] = i;
      std::sort(order.begin(), order.end(), [&](int a, int b) {
        if (deg[a] != deg[b]) return deg[a] > deg[b];
        return units[a].nnz > units[b].nnz;
      });
      std::vector<char> m(n, 0);
      for (int idx : order) {
        if (m[idx]) continue;
        int best = -1, best_deg = -1;
        for (int nb : adj[idx]) {
          if (m[nb]) continue;
          if (deg[nb] > best_deg || (deg[nb] == best_deg && units[nb].nnz > units[best].nnz)) {
            best = nb; best_deg = deg[nb];
          }
        }
        if (best >= 0) { m[idx] = 1; m[best] = 1; pairs.emplace_back(idx, best); }
      }
      for (int i = 0; i < n; ++i) if (!m[i]) unmatched.push_back(i);
    }

    // a6: SPTC group emission (block_online.cpp:629-702)
    std::set<int> sptc_set;
    auto emit_group = [&](std::vector<int> g) {
      std::sort(g.begin(), g.end());
      for (int c : g) sptc_set.insert(c);
      T.s_window.push_back(w);
      while (g.size() < 4) g.push_back(-1);
      for (int c : g) T.s_column.push_back(c);
    };
    for (auto& pr : pairs) {
      const Unit& a = units[pr.first];
      const Unit& b = units[pr.second];
      std::vector<int> g{a.c1};
      if (a.c2 >= 0) g.push_back(a.c2);
      if (b.c1 >= 0) g.push_back(b.c1);
      if (b.c2 >= 0) g.push_back(b.c2);
      emit_group(g);
    }
    for (int idx : unmatched) {
      const Unit& u = units[idx];
      if (u.nnz < unit_min_nnz) continue;
      std::vector<int> g{u.c1};
      if (u.c2 >= 0) g.push_back(u.c2);
      emit_group(g);
    }
    for (int g = T.s_offsets.back(); g < (int)T.s_window.size(); ++g) {
      std::vector<int> gc;
      for (int p = 0; p < 4; ++p) if (T.s_column[g * 4 + p] >= 0) gc.push_back(T.s_column[g * 4 + p]);
      for (int lr = 0; lr < window; ++lr) {
        uint8_t mask = 0;
        int slots = 0;
        float v[2] = {0.f, 0.f};
        int8_t ps[2] = {-1, -1};
        for (int p = 0; p < (int)gc.size(); ++p) {
          const auto& hits = prof[gc[p]].hits;
          auto it = std::find_if(hits.begin(), hits.end(), [&](const std::pair<int, int>& h) { return h.first == lr; });
          if (it == hits.end()) continue;
          mask |= (uint8_t)(1u << p);
          if (slots < 2) { v[slots] = val[it->second]; ps[slots] = (int8_t)p; }
          slots++;
        }
        T.s_mask.push_back(mask);
        for (int s = 0; s < 2; ++s) { T.s_value.push_back(v[s]); T.s_pos.push_back(ps[s]); }
      }
    }
    T.s_offsets.push_back((int)T.s_window.size());

    // a7: CUDA funnel flags (block_online.cpp:706-714)
    bool has_cuda = false;
    for (auto& kv : prof)
      if (!tc_set.count(kv.first) && !sptc_set.count(kv.first)) has_cuda = true;

    // a8: TC sub-block packing (block_online.cpp:444-540), serialised in
    // window order as block_online.cpp:751-760 does.
    if (!tc_groups.empty()) {
      std::map<int, int> slot;                             // column -> block*8 + pos
      for (size_t b = 0; b < tc_groups.size(); ++b)
        for (size_t p = 0; p < tc_groups[b].size(); ++p) slot[tc_groups[b][p]] = (int)(b * 8 + p);
      const int nsub = (int)tc_groups.size();
      std::vector<uint64_t> lo(nsub, 0), hi(nsub, 0);
      std::vector<std::vector<float>> sv(nsub);
      for (int r = r0; r < r1; ++r) {
        const int lr = r - r0;
        for (int e = rowptr[r]; e < rowptr[r + 1]; ++e) {
          auto f = slot.find(col[e]);
          if (f == slot.end()) continue;
          const int k = f->second % 8, s = f->second / 8;
          if (lr >= 8) hi[s] |= 1ull << ((lr - 8) * 8 + k);
          else lo[s] |= 1ull << (lr * 8 + k);
          sv[s].push_back(val[e]);
        }
      }
      for (int s = 0; s < nsub; ++s) {
        for (int p = 0; p < 8; ++p) T.t_column.push_back(p < (int)tc_groups[s].size() ? tc_groups[s][p] : -1);
        T.t_binary.push_back((int64_t)lo[s]);
        T.t_binary.push_back((int64_t)hi[s]);
        T.t_value.insert(T.t_value.end(), sv[s].begin(), sv[s].end());
      }
      auto part = [&](int first, int cnt, int atomic) {
        T.t_row_offset.push_back(T.t_row_offset.back() + cnt);
        for (int s = first; s < first + cnt; ++s)
          T.t_block_offset.push_back(T.t_block_offset.back() + (int)sv[s].size());
        T.t_window_row.push_back(w * 16);                  // block_online.cpp:497
        T.t_atomic.push_back(atomic);
      };
      if (nsub <= part_t) {
        part(0, nsub, has_cuda ? 1 : 0);
      } else {
        for (int p = 0; p < nsub / part_t; ++p) part(p * part_t, part_t, 1);
        if (nsub % part_t) part(nsub - nsub % part_t, nsub % part_t, 1);
      }
    }

    // a7: CUDA residual rows (block_online.cpp:721-731)
    const int base_atomic = tc_set.empty() ? 0 : 1;
    for (int r = r0; r < r1; ++r) {
      std::vector<int> cc;
      std::vector<float> cv;
      for (int e = rowptr[r]; e < rowptr[r + 1]; ++e) {
        if (tc_set.count(col[e]) || sptc_set.count(col[e])) continue;
        cc.push_back(col[e]); cv.push_back(val[e]);
      }
      split_row(r, base_atomic, part_c, shortsz, cc, cv, cuda[w].large, cuda[w].small);
    }
  }

  // a9: CUDA serialisation (block_online.cpp:761-778)
  for (int w = 0; w < nwin; ++w)
    for (auto& p : cuda[w].large) {
      T.c_row_offset.push_back(T.c_row_offset.back() + p.count);
      T.c_row.push_back(p.row); T.c_atomic.push_back(p.atomic);
      T.c_column.insert(T.c_column.end(), p.cols.begin(), p.cols.end());
      T.c_value.insert(T.c_value.end(), p.vals.begin(), p.vals.end());
    }
  for (int w = 0; w < nwin; ++w)
    for (auto& p : cuda[w].small) {
      T.cs_row_offset.push_back(T.cs_row_offset.back() + p.count);
      T.cs_row.push_back(p.row); T.cs_atomic.push_back(p.atomic);
      T.cs_column.insert(T.cs_column.end(), p.cols.begin(), p.cols.end());
      T.cs_value.insert(T.cs_value.end(), p.vals.begin(), p.vals.end());
    }

  // a9: mma.sp tile packing (block_online.cpp:797-841)
  for (int w = 0; w < nwin; ++w) {
    const int gb = T.s_offsets[w], ge = T.s_offsets[w + 1];
    for (int g0 = gb; g0 < ge; g0 += 4) {
      T.s_tile_window.push_back(w);
      T.s_tile_group.push_back(g0);
      for (int k = 0; k < 16; ++k) {
        const int g = g0 + (k >> 2);
        T.s_tile_column.push_back(g < ge ? T.s_column[g * 4 + (k & 3)] : -1);
      }
      for (int rg = 0; rg < 8; ++rg) {
        float lo[8], hi[8];
        int plo0[4], plo1[4], phi0[4], phi1[4];
        for (int ch = 0; ch < 4; ++ch) {
          float v0, v1; int p0, p1;
          row_chunk(T, g0 + ch, ge, rg, window, v0, v1, p0, p1);
          lo[2 * ch] = v0; lo[2 * ch + 1] = v1; plo0[ch] = p0; plo1[ch] = p1;
          row_chunk(T, g0 + ch, ge, rg + 8, window, v0, v1, p0, p1);
          hi[2 * ch] = v0; hi[2 * ch + 1] = v1; phi0[ch] = p0; phi1[ch] = p1;
        }
        uint32_t meta = 0;
        for (int ch = 0; ch < 4; ++ch) {
          meta |= ((uint32_t)(plo0[ch] & 3) | ((uint32_t)(plo1[ch] & 3) << 2)) << (ch * 4);
          meta |= ((uint32_t)(phi0[ch] & 3) | ((uint32_t)(phi1[ch] & 3) << 2)) << (16 + ch * 4);
        }
        T.s_packed_meta.push_back((int)meta);
        for (int t = 0; t < 4; ++t) {
          T.s_packed_a.push_back((int)((uint32_t)half_bits(lo[2 * t]) | ((uint32_t)half_bits(lo[2 * t + 1]) << 16)));
          T.s_packed_a.push_back((int)((uint32_t)half_bits(hi[2 * t]) | ((uint32_t)half_bits(hi[2 * t + 1]) << 16)));
        }
      }
    }
    T.s_window_tile_offset.push_back((int)T.s_tile_window.size());
  }
}

}  // namespace

extern "C" {

// Runs the restated router.  Returns an opaque handle (free with
// oracle_route_free) or nullptr on bad arguments.
void* oracle_route(const int* rowptr, const int* col, const float* val, int rows,
                   int part_t, int part_c, int shortsz, int density, int window,
                   float tc_min_util, int unit_min_nnz, int skip_tc) {
  if (rows < 0 || window <= 0 || window > 16 || part_t <= 0 || part_c <= 0) return nullptr;
  Tables* T = new Tables();
  route(rowptr, col, val, rows, part_t, part_c, shortsz, density, window,
        tc_min_util, unit_min_nnz, skip_tc != 0, *T);
  return T;
}

// Table `idx` (0..28, the reference's return order): data pointer and byte size.
int oracle_route_table(void* h, int idx, const void** data, long* nbytes) {
  const Tables& T = *static_cast<Tables*>(h);
#define TR_CASE(i, v) case i: *data = T.v.data(); *nbytes = (long)(T.v.size() * sizeof(T.v[0])); return 0;
  switch (idx) {
    TR_CASE(0, t_row_offset) TR_CASE(1, t_block_offset) TR_CASE(2, t_column) TR_CASE(3, t_value)
    TR_CASE(4, t_window_row) TR_CASE(5, t_atomic) TR_CASE(6, t_binary)
    TR_CASE(7, c_row_offset) TR_CASE(8, c_row) TR_CASE(9, c_atomic) TR_CASE(10, c_column) TR_CASE(11, c_value)
    TR_CASE(12, cs_row_offset) TR_CASE(13, cs_row) TR_CASE(14, cs_atomic) TR_CASE(15, cs_column) TR_CASE(16, cs_value)
    TR_CASE(17, s_column) TR_CASE(18, s_mask) TR_CASE(19, s_value) TR_CASE(20, s_pos) TR_CASE(21, s_window)
    TR_CASE(22, s_offsets) TR_CASE(23, s_tile_window) TR_CASE(24, s_tile_group) TR_CASE(25, s_tile_column)
    TR_CASE(26, s_packed_a) TR_CASE(27, s_packed_meta) TR_CASE(28, s_window_tile_offset)
    default: return -1;
  }
#undef TR_CASE
}

void oracle_route_free(void* h) { delete static_cast<Tables*>(h); }

}  // extern "C"
