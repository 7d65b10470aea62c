// The whole three-stage router as sm_100a integer kernels.
//
// Restates on the device every stage of the reference router
// (TR-source/Block/block_online.cpp, block_sptc_2to4_online :545-871) the
// way the host router (router.cpp) does, table for table and bit for bit:
//
//   profile        :589-603   distinct columns of a window, their row masks
//   TC funnel      :215-253   candidates (count desc, column asc) in chunks
//                             of 8 kept by fill
//   2:4 units      :267-328   the other columns paired in candidate order
//   matching       :332-392   units in (nnz desc) order, each paired with the
//                             first unmatched unit in (nnz desc, index asc)
//                             order (the compatibility graph is complete: a
//                             column's 2-bit row vector never holds a 2)
//   2:4 groups     :629-702   pairs, then unmatched units with enough
//                             entries; per row at most two entries
//   CUDA parts     :706-733   each row's remaining entries in long parts of
//                             partsize_c and short parts of <= shortsize
//   TC packing     :444-540   16x8 bitmaps, values in CSR order
//   mma.sp packing :797-841   four groups per tile: FP16 pairs and 2-bit
//                             positions per row
//
// One CTA (256 threads) per window, two launches: the first counts every
// table's items per window, the host scans the counts into offsets, the
// second writes the tables.  The parallel stages use block-wide bitonic
// sorts, ballot scans and shared atomics; the matching (a sequential
// greedy walk) runs on one thread per window, its processing order from
// unit_order, the restatement of the reference's std::sort that the host
// router runs too.  Windows of up to kFullSmemCap entries work in shared
// memory, larger ones in a global scratch slice.
//
// Input rows must be sorted by column (t_value keeps CSR order per
// sub-block, which on sorted rows is the bit order the TC kernels read).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/trspmm.h"
#include "common.cuh"
#include "route_full_gpu.h"
#include "route_sort.cuh"
#include "unit_order.h"

namespace trs {
namespace {

constexpr int kFThreads = 256;
constexpr int kFullSmemCap = 1024;        // window entries handled in shared memory
constexpr int kFullSmemInts = 160;        // scratch words after the storage

// per-window item counts (first launch) and offsets (second launch), by table
enum : int {
  kSub = 0,    // TC sub-blocks
  kTVal,       // TC values
  kTPart,      // TC parts
  kGroup,      // 2:4 groups
  kTile,       // mma.sp tiles
  kCPart,      // long CUDA parts
  kCVal,       // their entries
  kSPart,      // short CUDA parts
  kSVal,       // their entries
  kLost,       // entries the 2:4 groups leave out (third and later per row)
  kFields
};

struct FullWork {
  uint64_t* keys;     // cap: (column << 32) | (local entry << 4) | local row, sorted
  uint64_t* aux;      // cap: candidate keys, then TC value keys
  int* pos;           // cap: per sorted key, its distinct column
  int* tmp;           // cap: scan output
  int* ucol;          // cap: distinct columns, ascending
  uint32_t* umask;    // cap: their row masks
  int* ukey0;         // cap: first sorted key of each distinct column
  int* slot;          // cap: TC slot (sub-block * 8 + k) or -1
  int* erank;         // cap: per local entry, residual rank in the window
  uint8_t* uroute;    // cap: per distinct column: 0 CUDA, 1 TC, 2 2:4
  uint8_t* eroute;    // cap: per local entry
  uint8_t* flags;     // cap
  int* u_p1;          // half: units (distinct columns, -1 for none)
  int* u_p2;
  int* u_nnz;
  int* order;         // half: the matching's processing order
  int* sorted;        // half: units by (nnz desc, index asc)
  int* spos;          // half: position of each unit in `sorted`
  int* lnext;         // half: linked list of unmatched positions
  int* lprev;
  uint8_t* matched;   // half
  int* grp;           // 4 * half: group columns (distinct-column indices)
  uint64_t* glo;      // sub: TC sub-block bitmaps, rows 0-7 / 8-15
  uint64_t* ghi;
  int* gcol;          // 8 * sub: TC sub-block columns
  int* gval;          // sub: TC values per sub-block
};

// Carves the storage of a window of capacity cap (a power of two) from
// `base`; returns the bytes used.  With base == 0 it only sizes.
__host__ __device__ inline int64_t full_layout(uint32_t cap, FullWork& w, uintptr_t base) {
  int64_t off = 0;
  auto take = [&](int64_t bytes) -> uintptr_t {
    off = (off + 15) & ~(int64_t)15;
    const uintptr_t p = base + (uintptr_t)off;
    off += bytes;
    return p;
  };
  const int64_t half = cap / 2 + 2, sub = cap / 8 + 2;
  w.keys = reinterpret_cast<uint64_t*>(take(8 * (int64_t)cap));
  w.aux = reinterpret_cast<uint64_t*>(take(8 * (int64_t)cap));
  w.pos = reinterpret_cast<int*>(take(4 * (int64_t)cap));
  w.tmp = reinterpret_cast<int*>(take(4 * (int64_t)cap));
  w.ucol = reinterpret_cast<int*>(take(4 * (int64_t)cap));
  w.umask = reinterpret_cast<uint32_t*>(take(4 * (int64_t)cap));
  w.ukey0 = reinterpret_cast<int*>(take(4 * (int64_t)cap));
  w.slot = reinterpret_cast<int*>(take(4 * (int64_t)cap));
  w.erank = reinterpret_cast<int*>(take(4 * (int64_t)cap));
  w.uroute = reinterpret_cast<uint8_t*>(take(cap));
  w.eroute = reinterpret_cast<uint8_t*>(take(cap));
  w.flags = reinterpret_cast<uint8_t*>(take(cap));
  w.u_p1 = reinterpret_cast<int*>(take(4 * half));
  w.u_p2 = reinterpret_cast<int*>(take(4 * half));
  w.u_nnz = reinterpret_cast<int*>(take(4 * half));
  w.order = reinterpret_cast<int*>(take(4 * half));
  w.sorted = reinterpret_cast<int*>(take(4 * half));
  w.spos = reinterpret_cast<int*>(take(4 * half));
  w.lnext = reinterpret_cast<int*>(take(4 * half));
  w.lprev = reinterpret_cast<int*>(take(4 * half));
  w.matched = reinterpret_cast<uint8_t*>(take(half));
  w.grp = reinterpret_cast<int*>(take(16 * half));
  w.glo = reinterpret_cast<uint64_t*>(take(8 * sub));
  w.ghi = reinterpret_cast<uint64_t*>(take(8 * sub));
  w.gcol = reinterpret_cast<int*>(take(32 * sub));
  w.gval = reinterpret_cast<int*>(take(4 * sub));
  return (off + 255) & ~(int64_t)255;
}

__host__ __device__ inline int64_t full_bytes(uint32_t cap) {
  FullWork w;
  return full_layout(cap, w, 0);
}

__device__ __forceinline__ int key_col(uint64_t k) { return (int)(k >> 32); }
__device__ __forceinline__ int key_entry(uint64_t k) { return (int)((k >> 4) & 0x0FFFFFFFu); }
__device__ __forceinline__ int key_row(uint64_t k) { return (int)(k & 15u); }

// Local entry of the first entry of distinct column u in local row lr, -1 if
// none (a column's keys ascend by entry, so by row).
__device__ int first_entry(const FullWork& w, int n, int u, int lr) {
  const int c = w.ucol[u];
  for (int i = w.ukey0[u]; i < n && key_col(w.keys[i]) == c; ++i) {
    const int r = key_row(w.keys[i]);
    if (r == lr) return key_entry(w.keys[i]);
    if (r > lr) break;
  }
  return -1;
}

// Appends a 2:4 group (columns as distinct-column indices, ascending; -1
// padded) and marks its columns as 2:4 (thread 0 only).
__device__ void add_group(FullWork& w, int& ng, int a, int b, int c, int d) {
  int g[4] = {a, b, c, d};
  int n = 0;
  for (int k = 0; k < 4; ++k)
    if (g[k] >= 0) g[n++] = g[k];
  for (int k = n; k < 4; ++k) g[k] = -1;
  for (int i = 1; i < n; ++i)                       // distinct-column order is column order
    for (int j = i; j > 0 && g[j - 1] > g[j]; --j) {
      const int t = g[j - 1];
      g[j - 1] = g[j];
      g[j] = t;
    }
  for (int k = 0; k < 4; ++k) w.grp[ng * 4 + k] = g[k];
  for (int k = 0; k < n; ++k) w.uroute[g[k]] = 2;
  ++ng;
}

__device__ __forceinline__ uint16_t f16_bits(float f) { return __half_as_ushort(__float2half_rn(f)); }

template <bool FILL>
__global__ void __launch_bounds__(kFThreads) route_full_kernel(
    const int32_t* __restrict__ indptr, const int32_t* __restrict__ indices,
    const float* __restrict__ values, int n_rows, RouteFullParams p,
    const int64_t* __restrict__ big_off, uint8_t* big, int* cnt, const int* __restrict__ off,
    FullTables o) {
  extern __shared__ __align__(16) uint8_t smem_full[];
  int* s_int = reinterpret_cast<int*>(smem_full + full_bytes(kFullSmemCap));
  const int wi = blockIdx.x, tid = threadIdx.x;
  const int window = p.window;
  const int r0 = wi * window, r1 = min(r0 + window, n_rows);
  const int e0 = indptr[r0];
  const int n = indptr[r1] - e0;
  const bool exact = p.mode == TR_ROUTE_EXACT;
  FullWork w;
  if (n <= kFullSmemCap) full_layout(kFullSmemCap, w, reinterpret_cast<uintptr_t>(smem_full));
  else full_layout(next_pow2((uint32_t)n), w, reinterpret_cast<uintptr_t>(big + big_off[wi]));
  int* warp_tot = s_int;                   // [0, 8): scan scratch
  // s_int[8..]: kept, ng, has_cuda, lost, nun, then per-row residual figures
  if (tid < 16) s_int[8 + tid] = 0;

  // ---- profile --------------------------------------------------------------
  const uint32_t np2 = next_pow2((uint32_t)max(n, 1));
  for (int i = tid; i < (int)np2; i += blockDim.x) w.keys[i] = ~0ull;
  __syncthreads();
  for (int r = r0; r < r1; ++r)
    for (int e = indptr[r] + tid; e < indptr[r + 1]; e += blockDim.x)
      w.keys[e - e0] = ((uint64_t)(uint32_t)indices[e] << 32) |
                       ((uint64_t)(uint32_t)(e - e0) << 4) | (uint32_t)(r - r0);
  bitonic_sort(w.keys, np2);
  for (int i = tid; i < n; i += blockDim.x) {
    w.flags[i] = (i == 0 || key_col(w.keys[i]) != key_col(w.keys[i - 1])) ? 1 : 0;
    w.eroute[i] = 0;
  }
  __syncthreads();
  const int nu = block_flag_scan(w.flags, n, w.pos, warp_tot);
  for (int i = tid; i < n; i += blockDim.x) w.pos[i] += w.flags[i] ? 0 : -1;
  for (int u = tid; u < nu; u += blockDim.x) {
    w.umask[u] = 0;
    w.slot[u] = -1;
    w.uroute[u] = 0;
  }
  __syncthreads();
  for (int i = tid; i < n; i += blockDim.x) {
    const int u = w.pos[i];
    if (w.flags[i]) {
      w.ucol[u] = key_col(w.keys[i]);
      w.ukey0[u] = i;
    }
    atomicOr(&w.umask[u], 1u << (uint32_t)key_row(w.keys[i]));
  }
  __syncthreads();

  // ---- stage 1: TC funnel ---------------------------------------------------
  if (!p.skip_tc) {
    for (int u = tid; u < nu; u += blockDim.x) w.flags[u] = __popc(w.umask[u]) >= p.density ? 1 : 0;
    __syncthreads();
    const int nc = block_flag_scan(w.flags, nu, w.tmp, warp_tot);
    const uint32_t cp2 = next_pow2((uint32_t)max(nc, 1));
    for (int i = tid; i < (int)cp2; i += blockDim.x) w.aux[i] = ~0ull;
    __syncthreads();
    for (int u = tid; u < nu; u += blockDim.x)
      if (w.flags[u]) w.aux[w.tmp[u]] = ((uint64_t)(16 - __popc(w.umask[u])) << 32) | (uint32_t)u;
    bitonic_sort(w.aux, cp2);
    if (tid == 0) {
      int kept = 0;
      for (int s = 0; s < nc; s += 8) {
        const int m = min(s + 8, nc) - s;
        int us[8];
        int nnz = 0;
        for (int i = 0; i < m; ++i) {
          us[i] = (int)(uint32_t)w.aux[s + i];
          nnz += __popc(w.umask[us[i]]);
        }
        if ((float)nnz / (float)(window * 8) < p.tc_min_util) continue;
        for (int i = 1; i < m; ++i)
          for (int j = i; j > 0 && us[j - 1] > us[j]; --j) {
            const int t = us[j - 1];
            us[j - 1] = us[j];
            us[j] = t;
          }
        for (int k = 0; k < 8; ++k) {
          if (k < m) {
            w.slot[us[k]] = kept * 8 + k;
            w.uroute[us[k]] = 1;
          }
          w.gcol[kept * 8 + k] = k < m ? w.ucol[us[k]] : -1;
        }
        ++kept;
      }
      s_int[8] = kept;
    }
    __syncthreads();
  }
  const int kept = s_int[8];

  // ---- stage 2a: units ------------------------------------------------------
  if (!p.skip_sptc) {
    for (int u = tid; u < nu; u += blockDim.x) w.flags[u] = w.uroute[u] != 1 ? 1 : 0;
    __syncthreads();
    const int nc = block_flag_scan(w.flags, nu, w.tmp, warp_tot);
    const uint32_t cp2 = next_pow2((uint32_t)max(nc, 1));
    for (int i = tid; i < (int)cp2; i += blockDim.x) w.aux[i] = ~0ull;
    __syncthreads();
    for (int u = tid; u < nu; u += blockDim.x)
      if (w.flags[u]) w.aux[w.tmp[u]] = ((uint64_t)(16 - __popc(w.umask[u])) << 32) | (uint32_t)u;
    bitonic_sort(w.aux, cp2);
    const int nun = (nc + 1) / 2;
    for (int i = tid; i < nun; i += blockDim.x) {
      const int a = (int)(uint32_t)w.aux[2 * i];
      const int b = 2 * i + 1 < nc ? (int)(uint32_t)w.aux[2 * i + 1] : -1;
      w.u_p1[i] = a;
      w.u_p2[i] = b;
      w.u_nnz[i] = __popc(w.umask[a]) + (b >= 0 ? __popc(w.umask[b]) : 0);
    }
    __syncthreads();

    // ---- stage 2b/2c: matching and groups (one thread) ---------------------
    if (tid == 0) {
      for (int i = 0; i < nun; ++i) w.order[i] = i;
      unit_order(w.order, nun, w.u_nnz);
      int start[34], s = 0;
      for (int c = 0; c < 34; ++c) start[c] = 0;
      for (int i = 0; i < nun; ++i) start[w.u_nnz[i]]++;
      for (int c = 33; c >= 0; --c) {
        const int b = start[c];
        start[c] = s;
        s += b;
      }
      for (int i = 0; i < nun; ++i) w.sorted[start[w.u_nnz[i]]++] = i;
      for (int i = 0; i < nun; ++i) {
        w.spos[w.sorted[i]] = i;
        w.lnext[i] = i + 1;
        w.lprev[i] = i - 1;
        w.matched[i] = 0;
      }
      int head = 0;
      auto unlink = [&](int at) {
        const int pv = w.lprev[at], nx = w.lnext[at];
        if (pv >= 0) w.lnext[pv] = nx;
        else head = nx;
        if (nx < nun) w.lprev[nx] = pv;
      };
      int ng = 0;
      for (int t = 0; t < nun; ++t) {
        const int idx = w.order[t];
        if (w.matched[idx]) continue;
        int at = head;
        if (at < nun && w.sorted[at] == idx) at = w.lnext[at];
        if (at >= nun) continue;                       // no unmatched partner
        const int best = w.sorted[at];
        w.matched[idx] = w.matched[best] = 1;
        unlink(w.spos[idx]);
        unlink(at);
        add_group(w, ng, w.u_p1[idx], w.u_p2[idx], w.u_p1[best], w.u_p2[best]);
      }
      for (int i = 0; i < nun; ++i)
        if (!w.matched[i] && w.u_nnz[i] >= p.unit_min_nnz) add_group(w, ng, w.u_p1[i], w.u_p2[i], -1, -1);
      s_int[9] = ng;
    }
    __syncthreads();
  }
  const int ng = s_int[9];

  // ---- 2:4 rows: the first two entries of each row inside a group ----------
  const int gbase = FILL ? off[wi * kFields + kGroup] : 0;
  {
    int lost = 0;
    for (int job = tid; job < ng * window; job += blockDim.x) {
      const int gi = job / window, lr = job % window;
      uint8_t mask = 0;
      int slots = 0;
      float v[2] = {0.f, 0.f};
      int8_t ps[2] = {-1, -1};
      int32_t ed[2] = {-1, -1};
      for (int k = 0; k < 4; ++k) {
        const int u = w.grp[gi * 4 + k];
        if (u < 0) break;
        const int le = first_entry(w, n, u, lr);
        if (le < 0) continue;
        mask |= (uint8_t)(1u << k);
        if (slots < 2) {
          v[slots] = values[e0 + le];
          ps[slots] = (int8_t)k;
          ed[slots] = e0 + le;
          w.eroute[le] = 2;
        } else {
          ++lost;
        }
        ++slots;
      }
      if (FILL) {
        const int64_t at = (int64_t)(gbase + gi) * window + lr;
        o.s_mask[at] = mask;
        for (int j = 0; j < 2; ++j) {
          o.s_value[2 * at + j] = v[j];
          o.s_pos[2 * at + j] = ps[j];
          o.s_edge[2 * at + j] = ed[j];
        }
      }
    }
    lost = __reduce_add_sync(0xffffffffu, lost);
    if ((tid & 31) == 0 && lost) atomicAdd(&s_int[11], lost);
  }
  __syncthreads();

  // ---- entry routes ---------------------------------------------------------
  for (int i = tid; i < n; i += blockDim.x) {
    const int le = key_entry(w.keys[i]);
    const int r = w.uroute[w.pos[i]];
    if (!exact) {
      w.eroute[le] = (uint8_t)r;
    } else if (r == 1) {
      const bool first = i == 0 || key_col(w.keys[i - 1]) != key_col(w.keys[i]) ||
                         key_row(w.keys[i - 1]) != key_row(w.keys[i]);
      w.eroute[le] = first ? 1 : 0;
    }
  }
  __syncthreads();
  {
    int any = 0;
    for (int le = tid; le < n; le += blockDim.x) any |= w.eroute[le] == 0;
    any = __any_sync(0xffffffffu, any);
    if ((tid & 31) == 0 && any) s_int[10] = 1;
  }
  __syncthreads();
  const bool has_cuda = s_int[10] != 0;

  // ---- TC sub-blocks --------------------------------------------------------
  int ntv = 0;
  if (kept > 0) {
    for (int s = tid; s < kept; s += blockDim.x) {
      w.glo[s] = w.ghi[s] = 0ull;
      w.gval[s] = 0;
    }
    __syncthreads();
    for (int i = tid; i < n; i += blockDim.x) {
      const int le = key_entry(w.keys[i]);
      const bool tc = w.eroute[le] == 1;
      w.flags[i] = tc ? 1 : 0;
      if (!tc) continue;
      const int sl = w.slot[w.pos[i]], lr = key_row(w.keys[i]), s = sl >> 3, k = sl & 7;
      if (lr >= 8) atomicOr(reinterpret_cast<unsigned long long*>(&w.ghi[s]), 1ull << ((lr - 8) * 8 + k));
      else atomicOr(reinterpret_cast<unsigned long long*>(&w.glo[s]), 1ull << (lr * 8 + k));
      atomicAdd(&w.gval[s], 1);
    }
    __syncthreads();
    ntv = block_flag_scan(w.flags, n, w.tmp, warp_tot);
    if (FILL) {
      // values per sub-block in CSR order: TC entries sorted by (sub-block, entry)
      const uint32_t tp2 = next_pow2((uint32_t)max(ntv, 1));
      for (int i = tid; i < (int)tp2; i += blockDim.x) w.aux[i] = ~0ull;
      __syncthreads();
      for (int i = tid; i < n; i += blockDim.x)
        if (w.flags[i])
          w.aux[w.tmp[i]] = ((uint64_t)(uint32_t)(w.slot[w.pos[i]] >> 3) << 32) |
                            (uint32_t)key_entry(w.keys[i]);
      bitonic_sort(w.aux, tp2);
      const int vb = off[wi * kFields + kTVal], sb = off[wi * kFields + kSub];
      for (int j = tid; j < ntv; j += blockDim.x) {
        const int le = (int)(uint32_t)w.aux[j];
        o.t_value[vb + j] = values[e0 + le];
        o.t_edge[vb + j] = e0 + le;
      }
      for (int s = tid; s < kept; s += blockDim.x) {
        o.t_binary[2 * (int64_t)(sb + s)] = (int64_t)w.glo[s];
        o.t_binary[2 * (int64_t)(sb + s) + 1] = (int64_t)w.ghi[s];
        o.t_subcnt[sb + s] = w.gval[s];
        for (int k = 0; k < 8; ++k) o.t_column[(int64_t)(sb + s) * 8 + k] = w.gcol[s * 8 + k];
      }
    }
  }
  const int pt = p.partsize_t;
  const int ntp = kept == 0 ? 0 : (kept <= pt ? 1 : kept / pt + (kept % pt ? 1 : 0));
  if (FILL && tid == 0 && kept > 0) {
    const int tp = off[wi * kFields + kTPart];
    for (int j = 0; j < ntp; ++j) {
      o.t_part_cnt[tp + j] = kept <= pt ? kept : (j < kept / pt ? pt : kept % pt);
      o.t_window_row[tp + j] = wi * 16;
      o.t_atomic[tp + j] = kept <= pt ? (has_cuda ? 1 : 0) : 1;
    }
  }

  // ---- CUDA parts -----------------------------------------------------------
  for (int le = tid; le < n; le += blockDim.x) w.flags[le] = w.eroute[le] == 0 ? 1 : 0;
  __syncthreads();
  const int nres = block_flag_scan(w.flags, n, w.erank, warp_tot);
  // per row: rank of its first residual entry, entries, long / short split
  int* s_rstart = s_int + 16;     // [16]
  int* s_long = s_int + 32;       // long entries per row, then its prefix
  int* s_lparts = s_int + 48;
  int* s_sparts = s_int + 64;
  int* s_nr = s_int + 80;
  int* s_pre = s_int + 96;        // [4][...]: prefixes (long entries, short entries, long parts, short parts)
  const int nrows = r1 - r0;
  const int part = p.partsize_c, shortsz = p.shortsize;
  if (tid < nrows) {
    const int a = indptr[r0 + tid] - e0, b = indptr[r0 + tid + 1] - e0;
    const int ra = a < n ? w.erank[a] : nres, rb = b < n ? w.erank[b] : nres;
    const int nr = rb - ra;
    int L = 0, LP = 0, SP = 0;
    if (nr > 0) {
      if (nr <= shortsz) {
        SP = 1;
      } else if (nr <= part) {
        L = nr;
        LP = 1;
      } else {
        const int rem = nr % part;
        LP = nr / part;
        L = LP * part;
        if (rem > 0) {
          if (rem <= shortsz) SP = 1;
          else { L += rem; ++LP; }
        }
      }
    }
    s_rstart[tid] = ra;
    s_nr[tid] = nr;
    s_long[tid] = L;
    s_lparts[tid] = LP;
    s_sparts[tid] = SP;
  }
  __syncthreads();
  if (tid == 0) {
    int cl = 0, cs = 0, pl = 0, ps = 0;
    for (int r = 0; r < nrows; ++r) {
      s_pre[4 * r + 0] = cl;
      s_pre[4 * r + 1] = cs;
      s_pre[4 * r + 2] = pl;
      s_pre[4 * r + 3] = ps;
      cl += s_long[r];
      cs += s_nr[r] - s_long[r];
      pl += s_lparts[r];
      ps += s_sparts[r];
    }
    s_int[12] = cl;
    s_int[13] = cs;
    s_int[14] = pl;
    s_int[15] = ps;
  }
  __syncthreads();
  if (FILL) {
    const int cv = off[wi * kFields + kCVal], sv = off[wi * kFields + kSVal];
    const int cp = off[wi * kFields + kCPart], sp = off[wi * kFields + kSPart];
    const int base_atomic = kept > 0 ? 1 : 0;
    for (int le = tid; le < n; le += blockDim.x) {
      if (!w.flags[le]) continue;
      int r = 0;
      while (r + 1 < nrows && indptr[r0 + r + 1] - e0 <= le) ++r;
      const int t = w.erank[le] - s_rstart[r];
      const int e = e0 + le;
      if (t < s_long[r]) {
        const int at = cv + s_pre[4 * r + 0] + t;
        o.c_column[at] = indices[e];
        o.c_value[at] = values[e];
        o.c_edge[at] = e;
      } else {
        const int at = sv + s_pre[4 * r + 1] + (t - s_long[r]);
        o.cs_column[at] = indices[e];
        o.cs_value[at] = values[e];
        o.cs_edge[at] = e;
      }
    }
    if (tid < nrows) {
      const int r = tid, nr = s_nr[r], LP = s_lparts[r];
      const bool multi = nr > part;
      for (int j = 0; j < LP; ++j) {
        const int at = cp + s_pre[4 * r + 2] + j;
        o.c_cnt[at] = multi ? (j < nr / part ? part : nr % part) : nr;
        o.c_row[at] = r0 + r;
        o.c_atomic[at] = multi ? 1 : base_atomic;
      }
      if (s_sparts[r]) {
        const int at = sp + s_pre[4 * r + 3];
        o.cs_cnt[at] = multi ? nr % part : nr;
        o.cs_row[at] = r0 + r;
        o.cs_atomic[at] = multi ? 1 : base_atomic;
      }
    }
  }

  // ---- 2:4 groups and mma.sp tiles ------------------------------------------
  const int ntiles = (ng + 3) / 4;
  if (FILL) {
    for (int gi = tid; gi < ng; gi += blockDim.x) {
      o.s_window[gbase + gi] = wi;
      for (int k = 0; k < 4; ++k) {
        const int u = w.grp[gi * 4 + k];
        o.s_column[(int64_t)(gbase + gi) * 4 + k] = u >= 0 ? w.ucol[u] : -1;
      }
    }
    __syncthreads();       // the rows' s_pos / s_value (written above) are read back below
    const int tb = off[wi * kFields + kTile];
    for (int job = tid; job < ntiles * 8; job += blockDim.x) {
      const int ti = job >> 3, rg = job & 7, g0 = ti * 4;
      if (rg == 0) {
        o.s_tile_window[tb + ti] = wi;
        o.s_tile_group[tb + ti] = gbase + g0;
        for (int k = 0; k < 16; ++k) {
          const int g = g0 + (k >> 2);
          const int u = g < ng ? w.grp[g * 4 + (k & 3)] : -1;
          o.s_tile_column[(int64_t)(tb + ti) * 16 + k] = u >= 0 ? w.ucol[u] : -1;
        }
      }
      // one chunk (group, row) of the packing: FP16 pair and 2-bit positions
      auto chunk = [&](int gl, int row, float& v0, float& v1, int& q0, int& q1) {
        v0 = 0.f; v1 = 0.f; q0 = 0; q1 = 1;
        if (gl >= ng || row >= window) return;
        const int64_t b = ((int64_t)(gbase + gl) * window + row) * 2;
        const int a0 = o.s_pos[b], a1 = o.s_pos[b + 1];
        const float w0 = o.s_value[b], w1 = o.s_value[b + 1];
        if (a0 < 0 && a1 < 0) return;
        if (a0 >= 0 && a1 >= 0) {
          if (a0 <= a1) { q0 = a0; q1 = a1; v0 = w0; v1 = w1; }
          else { q0 = a1; q1 = a0; v0 = w1; v1 = w0; }
          return;
        }
        const int rp = a0 >= 0 ? a0 : a1;
        const float rv = a0 >= 0 ? w0 : w1;
        const int dummy = rp == 0 ? 1 : 0;
        if (dummy < rp) { q0 = dummy; q1 = rp; v0 = 0.f; v1 = rv; }
        else { q0 = rp; q1 = dummy; v0 = rv; v1 = 0.f; }
      };
      uint32_t meta = 0;
      uint32_t words[8];
      for (int c = 0; c < 4; ++c) {
        float v0, v1;
        int q0, q1;
        chunk(g0 + c, rg, v0, v1, q0, q1);
        meta |= ((uint32_t)(q0 & 3) | ((uint32_t)(q1 & 3) << 2)) << (c * 4);
        words[2 * c] = (uint32_t)f16_bits(v0) | ((uint32_t)f16_bits(v1) << 16);
        chunk(g0 + c, rg + 8, v0, v1, q0, q1);
        meta |= ((uint32_t)(q0 & 3) | ((uint32_t)(q1 & 3) << 2)) << (16 + c * 4);
        words[2 * c + 1] = (uint32_t)f16_bits(v0) | ((uint32_t)f16_bits(v1) << 16);
      }
      const int64_t at = (int64_t)(tb + ti) * 8 + rg;
      o.s_packed_meta[at] = (int32_t)meta;
      for (int j = 0; j < 8; ++j) o.s_packed_a[at * 8 + j] = (int32_t)words[j];
    }
  } else if (tid == 0) {
    int* c = cnt + wi * kFields;
    c[kSub] = kept;
    c[kTVal] = ntv;
    c[kTPart] = ntp;
    c[kGroup] = ng;
    c[kTile] = ntiles;
    c[kCPart] = s_int[14];
    c[kCVal] = s_int[12];
    c[kSPart] = s_int[15];
    c[kSVal] = s_int[13];
    c[kLost] = s_int[11];
  }
}

__global__ void negative_index_kernel(const int32_t* __restrict__ idx, int64_t n, int* flag) {
  bool neg = false;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    neg |= idx[i] < 0;
  if (__any_sync(0xffffffffu, neg) && (threadIdx.x & 31) == 0) atomicOr(flag, 1);
}

}  // namespace

DeviceTables::~DeviceTables() {
  if (block) cudaFree(block);
}

int route_full_gpu(const int32_t* d_indptr, const int32_t* d_indices, const float* d_values,
                   int32_t n_rows, const RouteFullParams& p, DeviceTables& dev, RouteTables& host,
                   std::string& err) {
  const auto t0 = std::chrono::high_resolution_clock::now();
  host = RouteTables();
  host.window = p.window;
  if (dev.block) { cudaFree(dev.block); dev.block = nullptr; }
  for (int i = 0; i < 29; ++i) { dev.ptr[i] = nullptr; dev.count[i] = 0; dev.elem[i] = 0; }
  const int W = n_rows > 0 ? (n_rows + p.window - 1) / p.window : 0;
  std::vector<int32_t> indptr((size_t)n_rows + 1, 0);
  if (n_rows > 0) {
    TRS_CUDA(cudaMemcpy(indptr.data(), d_indptr, (size_t)(n_rows + 1) * 4, cudaMemcpyDeviceToHost));
    if (indptr[0] != 0) { err = "row_ptr[0] must be 0"; return TR_ERR_ARG; }
    for (int32_t r = 0; r < n_rows; ++r)
      if (indptr[r + 1] < indptr[r]) { err = "row_ptr must be non-decreasing"; return TR_ERR_ARG; }
    if (indptr[n_rows] > 0 && (!d_indices || !d_values)) { err = "null indices or values"; return TR_ERR_ARG; }
  }
  // scratch slices for windows beyond shared memory; stream-ordered
  // allocations (the default stream's pool) so repeated routing reuses them
  std::vector<int64_t> big_off(std::max(W, 1), 0);
  int64_t big_bytes = 0;
  for (int w = 0; w < W; ++w) {
    const int n = indptr[std::min((w + 1) * p.window, n_rows)] - indptr[w * p.window];
    if (n >= (1 << 27)) { err = "a window holds 2^27 or more entries"; return TR_ERR_UNSUPPORTED; }
    if (n > kFullSmemCap) {
      big_off[w] = big_bytes;
      big_bytes += full_bytes(next_pow2((uint32_t)n));
    }
  }
  struct AsyncBuf {
    void* p = nullptr;
    ~AsyncBuf() { if (p) cudaFreeAsync(p, 0); }
  };
  AsyncBuf scratch;
  const int64_t scratch_bytes = std::max<int64_t>(big_bytes, 256) + (int64_t)std::max(W, 1) * 8 +
                                (int64_t)std::max(W, 1) * kFields * 4 * 2 + 16;
  TRS_CUDA(cudaMallocAsync(&scratch.p, (size_t)scratch_bytes, 0));
  uint8_t* d_big = static_cast<uint8_t*>(scratch.p);
  int64_t* d_big_off = reinterpret_cast<int64_t*>(d_big + std::max<int64_t>(big_bytes, 256));
  int* d_cnt = reinterpret_cast<int*>(d_big_off + std::max(W, 1));
  int* d_off = d_cnt + (size_t)std::max(W, 1) * kFields;
  int* d_flag = d_off + (size_t)std::max(W, 1) * kFields;
  std::vector<int> cnt((size_t)W * kFields), off((size_t)W * kFields);
  int64_t total[kFields] = {0};
  const int smem = (int)full_bytes(kFullSmemCap) + kFullSmemInts * 4;
  if (W > 0) {
    TRS_CUDA(cudaMemcpyAsync(d_big_off, big_off.data(), (size_t)W * 8, cudaMemcpyHostToDevice, 0));
    TRS_CUDA(cudaMemsetAsync(d_flag, 0, 4, 0));
    const int64_t nnz = indptr[n_rows];
    if (nnz > 0)
      negative_index_kernel<<<(int)std::min<int64_t>((nnz + 255) / 256, 148 * 16), 256>>>(d_indices, nnz, d_flag);
    TRS_CUDA(cudaGetLastError());
    int rc;
    if ((rc = kernel_smem_limit((const void*)route_full_kernel<false>, smem)) ||
        (rc = kernel_smem_limit((const void*)route_full_kernel<true>, smem)))
      return rc;
    FullTables none{};
    route_full_kernel<false><<<W, kFThreads, smem>>>(d_indptr, d_indices, d_values, n_rows, p,
                                                     d_big_off, d_big, d_cnt, nullptr, none);
    TRS_CUDA(cudaGetLastError());
    int flag = 0;
    TRS_CUDA(cudaMemcpy(&flag, d_flag, 4, cudaMemcpyDeviceToHost));
    if (flag) { err = "column indices must be >= 0"; return TR_ERR_ARG; }
    TRS_CUDA(cudaMemcpy(cnt.data(), d_cnt, cnt.size() * 4, cudaMemcpyDeviceToHost));
    for (int w = 0; w < W; ++w)
      for (int f = 0; f < kFields; ++f) {
        off[(size_t)w * kFields + f] = (int)total[f];
        total[f] += cnt[(size_t)w * kFields + f];
      }
    for (int f = 0; f < kFields; ++f)
      if (total[f] * 64 > INT32_MAX) { err = "route tables too large for 32-bit offsets"; return TR_ERR_UNSUPPORTED; }
    TRS_CUDA(cudaMemcpyAsync(d_off, off.data(), off.size() * 4, cudaMemcpyHostToDevice, 0));
  }
  const int64_t nsub = total[kSub], ntv = total[kTVal], ntp = total[kTPart], ng = total[kGroup],
                ntile = total[kTile], ncp = total[kCPart], ncv = total[kCVal],
                nsp = total[kSPart], nsv = total[kSVal];
  const int64_t win = p.window;
  // one allocation for every table (16-byte aligned pieces): the 29 tables
  // in return order, the per-part / per-sub-block counts and the provenance
  FullTables t{};
  int64_t bytes = 0;
  std::vector<std::pair<void**, int64_t>> pieces;
  auto piece = [&](auto** ptr, int64_t n_items, int table) {
    using T = std::remove_pointer_t<std::remove_reference_t<decltype(*ptr)>>;
    pieces.emplace_back(reinterpret_cast<void**>(ptr), bytes);
    if (table >= 0) {
      dev.count[table] = n_items;
      dev.elem[table] = (int)sizeof(T);
    }
    bytes += ((int64_t)sizeof(T) * std::max<int64_t>(n_items, 1) + 15) / 16 * 16;
  };
  int32_t *d_t_row_offset, *d_t_block_offset, *d_c_row_offset, *d_cs_row_offset, *d_s_offsets,
      *d_s_wt_offset;
  piece(&d_t_row_offset, ntp + 1, 0); piece(&d_t_block_offset, nsub + 1, 1);
  piece(&t.t_column, nsub * 8, 2); piece(&t.t_value, ntv, 3); piece(&t.t_window_row, ntp, 4);
  piece(&t.t_atomic, ntp, 5); piece(&t.t_binary, nsub * 2, 6);
  piece(&d_c_row_offset, ncp + 1, 7); piece(&t.c_row, ncp, 8); piece(&t.c_atomic, ncp, 9);
  piece(&t.c_column, ncv, 10); piece(&t.c_value, ncv, 11);
  piece(&d_cs_row_offset, nsp + 1, 12); piece(&t.cs_row, nsp, 13); piece(&t.cs_atomic, nsp, 14);
  piece(&t.cs_column, nsv, 15); piece(&t.cs_value, nsv, 16);
  piece(&t.s_column, ng * 4, 17); piece(&t.s_mask, ng * win, 18); piece(&t.s_value, ng * win * 2, 19);
  piece(&t.s_pos, ng * win * 2, 20); piece(&t.s_window, ng, 21); piece(&d_s_offsets, (int64_t)W + 1, 22);
  piece(&t.s_tile_window, ntile, 23); piece(&t.s_tile_group, ntile, 24);
  piece(&t.s_tile_column, ntile * 16, 25); piece(&t.s_packed_a, ntile * 64, 26);
  piece(&t.s_packed_meta, ntile * 8, 27); piece(&d_s_wt_offset, (int64_t)W + 1, 28);
  piece(&t.t_part_cnt, ntp, -1); piece(&t.t_subcnt, nsub, -1); piece(&t.c_cnt, ncp, -1);
  piece(&t.cs_cnt, nsp, -1);
  piece(&t.t_edge, ntv, -1); piece(&t.s_edge, ng * win * 2, -1); piece(&t.c_edge, ncv, -1);
  piece(&t.cs_edge, nsv, -1);
  TRS_CUDA(cudaMalloc(&dev.block, (size_t)bytes));
  for (auto& pc : pieces) *pc.first = static_cast<uint8_t*>(dev.block) + pc.second;
  {
    const void* order[29] = {d_t_row_offset, d_t_block_offset, t.t_column, t.t_value,
                             t.t_window_row, t.t_atomic, t.t_binary, d_c_row_offset, t.c_row,
                             t.c_atomic, t.c_column, t.c_value, d_cs_row_offset, t.cs_row,
                             t.cs_atomic, t.cs_column, t.cs_value, t.s_column, t.s_mask,
                             t.s_value, t.s_pos, t.s_window, d_s_offsets, t.s_tile_window,
                             t.s_tile_group, t.s_tile_column, t.s_packed_a, t.s_packed_meta,
                             d_s_wt_offset};
    for (int i = 0; i < 29; ++i) dev.ptr[i] = order[i];
  }
  dev.t_edge = t.t_edge;
  dev.s_edge = t.s_edge;
  dev.c_edge = t.c_edge;
  dev.cs_edge = t.cs_edge;
  if (W > 0) {
    route_full_kernel<true><<<W, kFThreads, smem>>>(d_indptr, d_indices, d_values, n_rows, p,
                                                    d_big_off, d_big, d_cnt, d_off, t);
    TRS_CUDA(cudaGetLastError());
  }
  // the offset tables: prefix sums of the per-item counts (small; formed on
  // the host, kept there and uploaded)
  auto prefix = [&](std::vector<int32_t>& dst, const int32_t* d_counts, int64_t n_items) -> int {
    std::vector<int32_t> c((size_t)n_items);
    if (n_items > 0)
      TRS_CUDA(cudaMemcpy(c.data(), d_counts, (size_t)n_items * 4, cudaMemcpyDeviceToHost));
    dst.assign(1, 0);
    dst.reserve((size_t)n_items + 1);
    int64_t b = 0;
    for (int64_t i = 0; i < n_items; ++i) {
      b += c[(size_t)i];
      dst.push_back((int32_t)b);
    }
    return TR_OK;
  };
  int rc;
  if ((rc = prefix(host.t_row_offset, t.t_part_cnt, ntp)) ||
      (rc = prefix(host.t_block_offset, t.t_subcnt, nsub)) ||
      (rc = prefix(host.c_row_offset, t.c_cnt, ncp)) ||
      (rc = prefix(host.cs_row_offset, t.cs_cnt, nsp)))
    return rc;
  host.s_offsets.assign(1, 0);
  host.s_window_tile_offset.assign(1, 0);
  for (int w = 0; w < W; ++w) {
    host.s_offsets.push_back(host.s_offsets.back() + cnt[(size_t)w * kFields + kGroup]);
    host.s_window_tile_offset.push_back(host.s_window_tile_offset.back() +
                                        cnt[(size_t)w * kFields + kTile]);
  }
  const std::vector<int32_t>* offs[6] = {&host.t_row_offset, &host.t_block_offset,
                                         &host.c_row_offset, &host.cs_row_offset,
                                         &host.s_offsets, &host.s_window_tile_offset};
  int32_t* dsts[6] = {d_t_row_offset, d_t_block_offset, d_c_row_offset, d_cs_row_offset,
                      d_s_offsets, d_s_wt_offset};
  for (int i = 0; i < 6; ++i)
    TRS_CUDA(cudaMemcpyAsync(dsts[i], offs[i]->data(), offs[i]->size() * 4, cudaMemcpyHostToDevice, 0));
  if (p.mode != TR_ROUTE_EXACT)
    for (int w = 0; w < W; ++w) host.dropped += cnt[(size_t)w * kFields + kLost];
  TRS_CUDA(cudaDeviceSynchronize());
  host.seconds = std::chrono::duration<double>(std::chrono::high_resolution_clock::now() - t0).count();
  return TR_OK;
}

}  // namespace trs
