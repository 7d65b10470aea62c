// TCA row clustering on the host (native threads), with the signature and
// Jaccard stages optionally on the GPU (tca_gpu.cu).
//
// Follows spmm/tr_csr_fp16/tr_tca_reorder.py:44-357:
//   level 1 (:84-191)  MinHash-LSH over each row's column set, every pair of
//                      rows sharing an LSH bucket queued with its exact
//                      Jaccard similarity, pairs popped most similar first and
//                      merged union-find style (smaller cluster into larger;
//                      a cluster reaching `thres` rows stops growing); a pair
//                      whose members are no longer roots re-queues their roots
//                      with the Jaccard of the roots' own rows;
//   level 2 (:193-297) the same over level-1 clusters (column set = union of
//                      the members' sets), capped at `cluster_thres` clusters;
//   order   (:299-313) level-2 groups in order of first appearance, their
//                      level-1 clusters, each cluster's rows ascending.
// Where the reference leaves an order to its libraries this file fixes it:
// candidates of a row are taken in ascending row order (the reference
// iterates a Python set), and pairs of equal similarity pop in the order they
// were queued (the reference's heap leaves ties unordered).  MinHash uses the
// hash family of tca.h instead of datasketch's SHA-1-based one, so candidate
// sets are statistically equivalent, not identical, to the reference's.
// Rows without columns are never candidates (in the reference they only meet
// each other, and are skipped when queried).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <map>
#include <mutex>
#include <numeric>
#include <queue>
#include <thread>
#include <unordered_set>

#include "../../include/trspmm.h"
#include "tca.h"

namespace trs {
namespace {

template <class F>
void parallel_for(int64_t n, int64_t grain, F f) {       // f(begin, end)
  int t = (int)std::max(1u, std::thread::hardware_concurrency());
  t = (int)std::min<int64_t>(t, std::max<int64_t>(1, n / std::max<int64_t>(1, grain)));
  if (t <= 1) {
    f((int64_t)0, n);
    return;
  }
  std::vector<std::thread> pool;
  for (int k = 0; k < t; ++k) pool.emplace_back([&, k] { f(n * k / t, n * (k + 1) / t); });
  for (auto& th : pool) th.join();
}

// Sorted, duplicate-free column list of every row.
void unique_lists(const int32_t* indptr, const int32_t* indices, int32_t n,
                  std::vector<int64_t>& ptr, std::vector<int32_t>& col) {
  const int64_t nnz = indptr[n];
  std::vector<int32_t> tmp(indices, indices + nnz);
  std::vector<int64_t> len(n);
  parallel_for(n, 1024, [&](int64_t b, int64_t e) {
    for (int64_t r = b; r < e; ++r) {
      int32_t* s = tmp.data() + indptr[r];
      int32_t* t = tmp.data() + indptr[r + 1];
      std::sort(s, t);
      len[r] = std::unique(s, t) - s;
    }
  });
  ptr.assign((size_t)n + 1, 0);
  for (int32_t r = 0; r < n; ++r) ptr[r + 1] = ptr[r] + len[r];
  col.resize(ptr[n]);
  parallel_for(n, 1024, [&](int64_t b, int64_t e) {
    for (int64_t r = b; r < e; ++r)
      std::copy(tmp.begin() + indptr[r], tmp.begin() + indptr[r] + len[r], col.begin() + ptr[r]);
  });
}

void signatures_host(const std::vector<int64_t>& ptr, const std::vector<int32_t>& col,
                     uint64_t seed, int bands, int rows, std::vector<uint32_t>& sig,
                     std::vector<uint64_t>& dig) {
  const int64_t n = (int64_t)ptr.size() - 1;
  uint64_t a[kTcaPerm], b[kTcaPerm];
  for (int i = 0; i < kTcaPerm; ++i) {
    a[i] = tca_perm_a(seed, i);
    b[i] = tca_perm_b(seed, i);
  }
  sig.resize((size_t)n * kTcaPerm);
  dig.resize((size_t)n * bands);
  parallel_for(n, 256, [&](int64_t lo, int64_t hi) {
    for (int64_t r = lo; r < hi; ++r) {
      uint32_t* v = sig.data() + r * kTcaPerm;
      std::fill(v, v + kTcaPerm, 0xFFFFFFFFu);
      for (int64_t e = ptr[r]; e < ptr[r + 1]; ++e) {
        const uint32_t key = tca_key(col[e]);
        for (int i = 0; i < kTcaPerm; ++i) v[i] = std::min(v[i], tca_hash(a[i], b[i], key));
      }
      for (int j = 0; j < bands; ++j) dig[r * bands + j] = tca_band_digest(v + j * rows, rows, j);
    }
  });
}

int32_t intersect_count(const int32_t* x, int64_t nx, const int32_t* y, int64_t ny) {
  if (nx > ny) {
    std::swap(x, y);
    std::swap(nx, ny);
  }
  int32_t c = 0;
  if (nx * 8 < ny) {                         // lopsided: binary search the long list
    for (int64_t i = 0; i < nx; ++i) c += std::binary_search(y, y + ny, x[i]) ? 1 : 0;
    return c;
  }
  for (int64_t i = 0, j = 0; i < nx && j < ny;) {     // branch-free merge
    const int32_t a = x[i], b = y[j];
    c += a == b;
    i += a <= b;
    j += b <= a;
  }
  return c;
}

// |set(pa[k]) & set(pb[k])| for pairs sorted by pa: per run of equal pa the
// thread stamps pa's columns into its own column-indexed array, then counts
// each partner's columns that carry the stamp (|pb| direct lookups, no merge).
void intersections_host(const std::vector<int64_t>& ptr, const std::vector<int32_t>& col,
                        const std::vector<int32_t>& pa, const std::vector<int32_t>& pb,
                        std::vector<int32_t>& inter) {
  inter.resize(pa.size());
  int32_t n_cols = 0;
  for (int32_t c : col) n_cols = std::max(n_cols, c + 1);
  parallel_for((int64_t)pa.size(), 4096, [&](int64_t lo, int64_t hi) {
    std::vector<int32_t> stamp(n_cols, -1);
    int32_t cur = -1;
    for (int64_t k = lo; k < hi; ++k) {
      const int32_t i = pa[k], j = pb[k];
      if (i != cur) {
        for (int64_t e = ptr[i]; e < ptr[i + 1]; ++e) stamp[col[e]] = i;
        cur = i;
      }
      int32_t c = 0;
      for (int64_t e = ptr[j]; e < ptr[j + 1]; ++e) c += stamp[col[e]] == i;
      inter[k] = c;
    }
  });
}

double jaccard(int64_t la, int64_t lb, int32_t inter) {
  if (la == 0 || lb == 0) return 0.0;
  const int64_t uni = la + lb - inter;
  return uni > 0 ? (double)inter / (double)uni : 0.0;
}

// Every pair of items (i < j, both with a non-empty set) that shares a band
// digest in some band, as sorted unique keys i * m + j.
int candidate_pairs(const std::vector<uint64_t>& dig, int bands, const std::vector<int64_t>& ptr,
                    int64_t max_pairs, std::vector<uint64_t>& keys, std::string& err) {
  const int64_t m = (int64_t)ptr.size() - 1;
  std::vector<int32_t> live;
  for (int64_t i = 0; i < m; ++i)
    if (ptr[i + 1] > ptr[i]) live.push_back((int32_t)i);
  const int t = std::max(1, std::min<int>(bands, (int)std::thread::hardware_concurrency()));
  std::vector<std::vector<uint64_t>> acc(t);
  std::vector<std::string> errs(t);
  std::vector<std::thread> pool;
  for (int k = 0; k < t; ++k)
    pool.emplace_back([&, k] {
      std::vector<std::pair<uint64_t, int32_t>> items(live.size());
      std::vector<uint64_t> band, merged;
      for (int j = k; j < bands && errs[k].empty(); j += t) {
        for (size_t x = 0; x < live.size(); ++x) items[x] = {dig[(size_t)live[x] * bands + j], live[x]};
        std::sort(items.begin(), items.end());
        band.clear();
        for (size_t s = 0; s < items.size();) {
          size_t e = s + 1;
          while (e < items.size() && items[e].first == items[s].first) ++e;
          const int64_t run = (int64_t)(e - s);
          if (run * (run - 1) / 2 + (int64_t)band.size() > max_pairs) {
            errs[k] = "TCA: more than max_pairs LSH candidate pairs (an LSH bucket of " +
                      std::to_string(run) + " rows)";
            break;
          }
          for (size_t x = s; x < e; ++x)
            for (size_t y = x + 1; y < e; ++y) band.push_back((uint64_t)items[x].second * m + items[y].second);
          s = e;
        }
        std::sort(band.begin(), band.end());
        merged.clear();
        std::set_union(acc[k].begin(), acc[k].end(), band.begin(), band.end(), std::back_inserter(merged));
        acc[k].swap(merged);
        if ((int64_t)acc[k].size() > max_pairs && errs[k].empty())
          errs[k] = "TCA: more than max_pairs LSH candidate pairs";
      }
    });
  for (auto& th : pool) th.join();
  for (auto& e : errs)
    if (!e.empty()) {
      err = e;
      return TR_ERR_UNSUPPORTED;
    }
  // union of the threads' sorted sets, merged pairwise in parallel
  for (int w = 1; w < t; w *= 2) {
    std::vector<int> left;
    for (int k = 0; k + w < t; k += 2 * w) left.push_back(k);
    parallel_for((int64_t)left.size(), 1, [&](int64_t lo, int64_t hi) {
      for (int64_t q = lo; q < hi; ++q) {
        std::vector<uint64_t>& a = acc[left[q]];
        std::vector<uint64_t>& b = acc[left[q] + w];
        std::vector<uint64_t> merged;
        merged.reserve(a.size() + b.size());
        std::set_union(a.begin(), a.end(), b.begin(), b.end(), std::back_inserter(merged));
        a.swap(merged);
        std::vector<uint64_t>().swap(b);
      }
    });
  }
  keys.swap(acc[0]);
  if ((int64_t)keys.size() > max_pairs) {
    err = "TCA: more than max_pairs LSH candidate pairs";
    return TR_ERR_UNSUPPORTED;
  }
  return TR_OK;
}

// Capped union-find clustering of m items over the queued pairs (sorted
// unique keys i * m + j with their similarities); `rejac(r1, r2)` is the
// similarity a re-queued pair of roots gets.  Returns each item's root.
// Pop order of the queued pairs: similarity descending, then queue order
// (the key index).  Records are sorted in parallel chunks and merged.
struct PopRec {
  double s;
  int64_t i;         // index of the pair among the sorted keys
  int32_t p1, p2;    // the pair (p1 < p2)
};
inline bool pop_before(const PopRec& x, const PopRec& y) { return x.s != y.s ? x.s > y.s : x.i < y.i; }

std::vector<PopRec> pop_order(const std::vector<uint64_t>& keys, const std::vector<double>& simi,
                              int64_t m) {
  const int64_t P = (int64_t)simi.size();
  std::vector<PopRec> rec(P);
  parallel_for(P, 65536, [&](int64_t lo, int64_t hi) {
    for (int64_t x = lo; x < hi; ++x)
      rec[x] = {simi[x], x, (int32_t)(keys[x] / m), (int32_t)(keys[x] % m)};
  });
  int t = (int)std::max(1u, std::thread::hardware_concurrency());
  t = (int)std::min<int64_t>(t, std::max<int64_t>(1, P / 65536));
  std::vector<int64_t> cut(t + 1);
  for (int k = 0; k <= t; ++k) cut[k] = P * k / t;
  parallel_for(t, 1, [&](int64_t lo, int64_t hi) {
    for (int64_t k = lo; k < hi; ++k) std::sort(rec.begin() + cut[k], rec.begin() + cut[k + 1], pop_before);
  });
  for (int w = 1; w < t; w *= 2) {                   // pairwise merges of sorted runs
    std::vector<std::pair<int64_t, int64_t>> jobs;
    for (int k = 0; k + w < t; k += 2 * w) jobs.push_back({k, std::min(k + 2 * w, t)});
    parallel_for((int64_t)jobs.size(), 1, [&](int64_t lo, int64_t hi) {
      for (int64_t q = lo; q < hi; ++q)
        std::inplace_merge(rec.begin() + cut[jobs[q].first], rec.begin() + cut[jobs[q].first + w],
                           rec.begin() + cut[jobs[q].second], pop_before);
    });
  }
  return rec;
}

template <class Rejac>
std::vector<int32_t> cluster(int64_t m, const std::vector<uint64_t>& keys,
                             const std::vector<double>& simi, int32_t cap, Rejac rejac) {
  const int64_t P = (int64_t)keys.size();
  const std::vector<PopRec> ord = pop_order(keys, simi, m);
  // where each item's pairs (i, .) start among the sorted keys
  std::vector<int64_t> kstart(m + 1, 0);
  for (int64_t x = 0; x < P; ++x) kstart[keys[x] / m + 1]++;
  for (int64_t i = 0; i < m; ++i) kstart[i + 1] += kstart[i];
  // rank[x] = position of key x in the pop order: an initial pair is still
  // queued while the pop position has not passed its rank
  std::vector<int64_t> rank(P);
  parallel_for(P, 65536, [&](int64_t lo, int64_t hi) {
    for (int64_t q = lo; q < hi; ++q) rank[ord[q].i] = q;
  });
  struct Re {
    double s;
    uint64_t seq;
    int32_t p1, p2;
  };
  auto worse = [](const Re& x, const Re& y) { return x.s != y.s ? x.s < y.s : x.seq > y.seq; };
  std::priority_queue<Re, std::vector<Re>, decltype(worse)> heap(worse);
  std::unordered_set<uint64_t> queued_re;       // re-queued pairs not yet popped
  uint64_t seq = (uint64_t)P;
  std::vector<int32_t> cid(m), sz(m, 1);
  std::vector<uint8_t> del(m, 0);
  std::iota(cid.begin(), cid.end(), 0);
  int64_t ncl = m, pos = 0;
  auto root = [&](int32_t i) {
    while (i != cid[i]) {
      cid[i] = cid[cid[i]];
      i = cid[i];
    }
    return i;
  };
  auto key_of = [&](int32_t a, int32_t b) {
    return a < b ? (uint64_t)a * m + b : (uint64_t)b * m + a;
  };
  auto queued = [&](uint64_t k) {
    const int64_t i = (int64_t)(k / m);
    const auto b = keys.begin() + kstart[i], e = keys.begin() + kstart[i + 1];
    const auto it = std::lower_bound(b, e, k);
    if (it != e && *it == k && rank[it - keys.begin()] >= pos) return true;
    return queued_re.count(k) > 0;
  };
  while (ncl > 0 && (pos < P || !heap.empty())) {
    int32_t p1, p2;
    if (pos < P && (heap.empty() || ord[pos].s >= heap.top().s)) {
      const PopRec& q = ord[pos++];
      p1 = q.p1;
      p2 = q.p2;
    } else {
      const Re t = heap.top();
      heap.pop();
      p1 = t.p1;
      p2 = t.p2;
      queued_re.erase(key_of(p1, p2));
    }
    if (p1 == cid[p1] && p2 == cid[p2]) {
      if (del[p1] || del[p2]) continue;
      const int32_t into = sz[p1] < sz[p2] ? p2 : p1, from = into == p1 ? p2 : p1;
      cid[from] = into;
      --ncl;
      sz[into] += sz[from];
      if (sz[into] >= cap) {
        del[into] = 1;
        --ncl;
      }
    } else {
      const int32_t r1 = root(p1), r2 = root(p2);
      if (del[r1] || del[r2]) continue;
      const uint64_t k = key_of(r1, r2);
      if (r1 != r2 && !queued(k)) {
        heap.push({rejac(r1, r2), seq++, r1, r2});
        queued_re.insert(k);
      }
    }
  }
  std::vector<int32_t> out(m);
  for (int64_t i = 0; i < m; ++i) out[i] = root((int32_t)i);
  return out;
}

// Pairs of sorted keys -> (a, b) arrays and exact Jaccard similarities.
int pair_similarities(const std::vector<int64_t>& ptr, const std::vector<int32_t>& col,
                      const std::vector<uint64_t>& keys, int device, std::vector<double>& simi,
                      std::string& err) {
  const int64_t m = (int64_t)ptr.size() - 1;
  std::vector<int32_t> pa(keys.size()), pb(keys.size()), inter;
  parallel_for((int64_t)keys.size(), 65536, [&](int64_t lo, int64_t hi) {
    for (int64_t k = lo; k < hi; ++k) {
      pa[k] = (int32_t)(keys[k] / m);
      pb[k] = (int32_t)(keys[k] % m);
    }
  });
  if (device) {
    const int rc = tca_intersections_gpu(ptr, col, pa, pb, inter, err);
    if (rc) return rc;
  } else {
    intersections_host(ptr, col, pa, pb, inter);
  }
  simi.resize(keys.size());
  parallel_for((int64_t)keys.size(), 65536, [&](int64_t lo, int64_t hi) {
    for (int64_t k = lo; k < hi; ++k)
      simi[k] = jaccard(ptr[pa[k] + 1] - ptr[pa[k]], ptr[pb[k] + 1] - ptr[pb[k]], inter[k]);
  });
  return TR_OK;
}

}  // namespace

void tca_lsh_params(double threshold, int num_perm, int& bands, int& rows) {
  static std::mutex mu;
  static std::map<std::pair<double, int>, std::pair<int, int>> memo;
  std::lock_guard<std::mutex> g(mu);
  const auto it = memo.find({threshold, num_perm});
  if (it != memo.end()) {
    bands = it->second.first;
    rows = it->second.second;
    return;
  }
  // composite Simpson rule, 4096 intervals per integral
  auto integrate = [](double lo, double hi, auto f) {
    const int n = 4096;
    const double h = (hi - lo) / n;
    double s = f(lo) + f(hi);
    for (int i = 1; i < n; ++i) s += f(lo + i * h) * (i % 2 ? 4.0 : 2.0);
    return s * h / 3.0;
  };
  double best = 0;
  bands = rows = 1;
  bool first = true;
  for (int b = 1; b <= num_perm; ++b)
    for (int r = 1; r <= num_perm / b; ++r) {
      const double fp = integrate(0.0, threshold, [&](double s) { return 1.0 - std::pow(1.0 - std::pow(s, r), b); });
      const double fn = integrate(threshold, 1.0, [&](double s) { return std::pow(1.0 - std::pow(s, r), b); });
      const double e = 0.5 * fp + 0.5 * fn;
      if (first || e < best) {
        best = e;
        bands = b;
        rows = r;
        first = false;
      }
    }
  memo[{threshold, num_perm}] = {bands, rows};
}

int tca_order(const int32_t* indptr, const int32_t* indices, int32_t n_rows, const TcaParams& p,
              std::vector<int32_t>& order, TcaStats& st, std::string& err) {
  if (n_rows < 0) { err = "negative row count"; return TR_ERR_ARG; }
  if (p.thres < 1 || p.cluster_thres < 1) { err = "TCA cluster caps must be >= 1"; return TR_ERR_ARG; }
  if (!(p.lsh_threshold > 0.0 && p.lsh_threshold < 1.0)) {
    err = "TCA lsh_threshold must be in (0, 1)";
    return TR_ERR_ARG;
  }
  if (p.max_pairs < 0) { err = "TCA max_pairs must be >= 0"; return TR_ERR_ARG; }
  st = TcaStats{};
  order.clear();
  if (n_rows == 0) return TR_OK;
  int bands = 0, rows = 0;
  tca_lsh_params(p.lsh_threshold, kTcaPerm, bands, rows);
  st.bands = bands;
  st.rows_per_band = rows;
  auto t_last = std::chrono::steady_clock::now();
  auto lap = [&](int stage) {          // adds the time since the last lap to a stage
    const auto now = std::chrono::steady_clock::now();
    st.seconds[stage] += std::chrono::duration<double>(now - t_last).count();
    t_last = now;
  };

  // ---- level 1: rows ----------------------------------------------------------
  std::vector<int64_t> ptr;
  std::vector<int32_t> col;
  unique_lists(indptr, indices, n_rows, ptr, col);
  std::vector<uint32_t> sig;
  std::vector<uint64_t> dig;
  int rc = p.device ? tca_signatures_gpu(ptr, col, p.seed, bands, rows, sig, dig, err)
                    : (signatures_host(ptr, col, p.seed, bands, rows, sig, dig), TR_OK);
  if (rc) return rc;
  lap(0);
  std::vector<uint64_t> keys;
  rc = candidate_pairs(dig, bands, ptr, p.max_pairs, keys, err);
  if (rc) return rc;
  std::vector<uint64_t>().swap(dig);
  lap(1);
  std::vector<double> simi;
  rc = pair_similarities(ptr, col, keys, p.device, simi, err);
  if (rc) return rc;
  lap(2);
  st.pairs1 = (int64_t)keys.size();
  const int64_t n = n_rows;
  std::vector<int32_t> root1 = cluster(n, keys, simi, p.thres, [&](int32_t a, int32_t b) {
    const int64_t la = ptr[a + 1] - ptr[a], lb = ptr[b + 1] - ptr[b];
    return jaccard(la, lb, intersect_count(col.data() + ptr[a], la, col.data() + ptr[b], lb));
  });
  std::vector<uint64_t>().swap(keys);
  std::vector<double>().swap(simi);
  lap(3);

  // level-1 clusters in order of first appearance, members ascending
  std::vector<int32_t> cl_of_root(n, -1), cl_start, cl_rows;
  std::vector<int32_t> cl_count;
  for (int64_t i = 0; i < n; ++i) {
    int32_t& c = cl_of_root[root1[i]];
    if (c < 0) {
      c = (int32_t)cl_count.size();
      cl_count.push_back(0);
    }
    cl_count[c]++;
  }
  const int64_t nc = (int64_t)cl_count.size();
  st.clusters1 = nc;
  cl_start.assign(nc + 1, 0);
  for (int64_t c = 0; c < nc; ++c) cl_start[c + 1] = cl_start[c] + cl_count[c];
  cl_rows.resize(n);
  {
    std::vector<int32_t> fill(cl_start.begin(), cl_start.end() - 1);
    for (int64_t i = 0; i < n; ++i) cl_rows[fill[cl_of_root[root1[i]]]++] = (int32_t)i;
  }

  // ---- level 2: clusters --------------------------------------------------------
  // column set of a cluster = union of its rows' sets; its MinHash signature
  // is the element-wise minimum of the rows' signatures (the same hashes)
  std::vector<int64_t> cptr(nc + 1, 0);
  std::vector<std::vector<int32_t>> cols_of(nc);
  std::vector<uint64_t> cdig((size_t)nc * bands);
  parallel_for(nc, 256, [&](int64_t lo, int64_t hi) {
    uint32_t v[kTcaPerm];
    for (int64_t c = lo; c < hi; ++c) {
      std::vector<int32_t>& u = cols_of[c];
      std::fill(v, v + kTcaPerm, 0xFFFFFFFFu);
      for (int32_t k = cl_start[c]; k < cl_start[c + 1]; ++k) {
        const int32_t r = cl_rows[k];
        u.insert(u.end(), col.begin() + ptr[r], col.begin() + ptr[r + 1]);
        for (int i = 0; i < kTcaPerm; ++i) v[i] = std::min(v[i], sig[(size_t)r * kTcaPerm + i]);
      }
      std::sort(u.begin(), u.end());
      u.erase(std::unique(u.begin(), u.end()), u.end());
      for (int j = 0; j < bands; ++j) cdig[c * bands + j] = tca_band_digest(v + j * rows, rows, j);
    }
  });
  std::vector<uint32_t>().swap(sig);
  for (int64_t c = 0; c < nc; ++c) cptr[c + 1] = cptr[c] + (int64_t)cols_of[c].size();
  std::vector<int32_t> ccol(cptr[nc]);
  for (int64_t c = 0; c < nc; ++c) {
    std::copy(cols_of[c].begin(), cols_of[c].end(), ccol.begin() + cptr[c]);
    std::vector<int32_t>().swap(cols_of[c]);
  }
  lap(0);
  rc = candidate_pairs(cdig, bands, cptr, p.max_pairs, keys, err);
  if (rc) return rc;
  lap(1);
  rc = pair_similarities(cptr, ccol, keys, p.device, simi, err);
  if (rc) return rc;
  lap(2);
  st.pairs2 = (int64_t)keys.size();
  std::vector<int32_t> root2 = cluster(nc, keys, simi, p.cluster_thres, [&](int32_t a, int32_t b) {
    const int64_t la = cptr[a + 1] - cptr[a], lb = cptr[b + 1] - cptr[b];
    return jaccard(la, lb, intersect_count(ccol.data() + cptr[a], la, ccol.data() + cptr[b], lb));
  });

  // ---- order: level-2 groups by first appearance, clusters ascending ----------
  std::vector<int32_t> grp_of_root(nc, -1), grp_first;
  std::vector<std::vector<int32_t>> members;
  for (int64_t c = 0; c < nc; ++c) {
    int32_t& g = grp_of_root[root2[c]];
    if (g < 0) {
      g = (int32_t)members.size();
      members.emplace_back();
    }
    members[g].push_back((int32_t)c);
  }
  st.clusters2 = (int64_t)members.size();
  order.reserve(n);
  for (const auto& g : members)
    for (int32_t c : g)
      for (int32_t k = cl_start[c]; k < cl_start[c + 1]; ++k) order.push_back(cl_rows[k]);
  lap(3);
  return TR_OK;
}

}  // namespace trs
