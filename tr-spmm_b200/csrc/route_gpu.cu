// Dense-TC funnel of the router as sm_100a integer kernels.
//
// Restates, on the device, the first stage of the reference router
// (TR-source/Block/block_online.cpp:584-620 with select_tc_columns_online
// :215-253 and build_tcu_part_online :444-540) in its exact form (a
// repeated (row, column) entry keeps only its first occurrence on the
// tensor cores, as this library's exact mode does), for rows sorted by
// column:
//
//   per 16-row window: the column profile (distinct columns and the rows
//   that use them), the candidates used by >= density rows ordered by
//   (count desc, column asc), chunks of 8 kept when their fill
//   >= tc_min_util, each chunk's columns sorted ascending, and the 16x8
//   sub-blocks: bit (row*8 + k) of binary_lo (rows 0-7) / binary_hi (rows
//   8-15), values in bit order, parts of partsize_t sub-blocks.
//
// One CTA per window.  The window's keys (column, entry, row) are sorted
// with a block-wide bitonic sort; distinct columns are found with warp
// ballots and a block prefix scan (the compaction); row masks are OR-ed per
// distinct column with shared atomics; candidates are sorted the same way.
// Windows of up to kSmemKeys entries work in shared memory; larger ones
// (hub rows) run the same code on their slice of a global scratch buffer.
// A counting launch gives sub-blocks and values per window, the host scans
// them into offsets, a filling launch writes the tables.
//
// The result equals the CPU router's t_row_offset, t_block_offset,
// t_column, t_value, t_window_row and t_binary; t_atomic is not produced
// (the reference sets it from the 2:4 matching's outcome).
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/trspmm.h"
#include "common.cuh"
#include "route_gpu.h"
#include "route_sort.cuh"

namespace trs {
namespace {

constexpr int kRThreads = 256;
constexpr int kSmemKeys = 2048;          // entries of a window handled in shared memory

// Per-window working storage for up to `cap` entries (cap a power of two).
struct WinWork {
  uint64_t* keys;      // (column << 32) | (entry << 4) | row; padding = ~0
  uint64_t* cand;      // (16 - count) << 32 | distinct-column index
  uint64_t* glo;       // per sub-block bitmaps (rows 0-7 / 8-15)
  uint64_t* ghi;
  int* pos;            // per key: distinct-column index
  int* tmp;            // scan output / per-sub-block value starts
  int* ucol;           // distinct columns, ascending
  uint32_t* umask;     // their row masks
  int* slot;           // per distinct column: tc slot (group*8 + k) or -1
  int* gcol;           // per sub-block, its 8 columns (-1 padded)
  uint8_t* flags;
};

__host__ __device__ inline int64_t storage_bytes(uint32_t cap) {
  const int64_t groups = cap / 8 + 1;
  return (int64_t)cap * 8 * 2 + groups * 8 * 2 + (int64_t)cap * 4 * 5 + (groups * 8) * 4 +
         (int64_t)cap;
}

__device__ void bind_storage(WinWork& w, uint8_t* base, uint32_t cap) {
  const uint32_t groups = cap / 8 + 1;
  w.keys = reinterpret_cast<uint64_t*>(base);
  w.cand = w.keys + cap;
  w.glo = w.cand + cap;
  w.ghi = w.glo + groups;
  w.pos = reinterpret_cast<int*>(w.ghi + groups);
  w.tmp = w.pos + cap;
  w.ucol = w.tmp + cap;
  w.umask = reinterpret_cast<uint32_t*>(w.ucol + cap);
  w.slot = reinterpret_cast<int*>(w.umask + cap);
  w.gcol = w.slot + cap;
  w.flags = reinterpret_cast<uint8_t*>(w.gcol + groups * 8);
}

// Profile, candidates and groups of one window; returns the number of
// sub-blocks kept (w.slot, w.gcol filled).  Every thread calls it.
__device__ int window_groups(const int32_t* __restrict__ indptr, const int32_t* __restrict__ indices,
                             int r0, int r1, const RouteGpuParams& p, WinWork& w, int* s_int) {
  const int e0 = indptr[r0], e1 = indptr[r1];
  const int n = e1 - e0;
  const uint32_t np2 = next_pow2((uint32_t)max(n, 1));
  for (int i = threadIdx.x; i < (int)np2; i += blockDim.x) w.keys[i] = ~0ull;
  __syncthreads();
  for (int r = r0; r < r1; ++r)
    for (int e = indptr[r] + threadIdx.x; e < indptr[r + 1]; e += blockDim.x)
      w.keys[e - e0] = ((uint64_t)(uint32_t)indices[e] << 32) |
                       ((uint64_t)(uint32_t)(e - e0) << 4) | (uint32_t)(r - r0);
  bitonic_sort(w.keys, np2);
  // distinct columns: first key of each column
  for (int i = threadIdx.x; i < n; i += blockDim.x)
    w.flags[i] = (i == 0 || (w.keys[i] >> 32) != (w.keys[i - 1] >> 32)) ? 1 : 0;
  __syncthreads();
  int* warp_tot = s_int;
  const int nu = block_flag_scan(w.flags, n, w.pos, warp_tot);
  for (int i = threadIdx.x; i < n; i += blockDim.x) w.pos[i] += w.flags[i] ? 0 : -1;
  for (int u = threadIdx.x; u < nu; u += blockDim.x) {
    w.umask[u] = 0;
    w.slot[u] = -1;
  }
  __syncthreads();
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const int u = w.pos[i];
    if (w.flags[i]) w.ucol[u] = (int)(w.keys[i] >> 32);
    atomicOr(&w.umask[u], 1u << (uint32_t)(w.keys[i] & 15u));
  }
  __syncthreads();
  if (p.skip_tc) return 0;
  // candidates: used by >= density rows, ordered by (count desc, column asc)
  for (int u = threadIdx.x; u < nu; u += blockDim.x)
    w.flags[u] = __popc(w.umask[u]) >= p.density ? 1 : 0;
  __syncthreads();
  const int nc = block_flag_scan(w.flags, nu, w.tmp, warp_tot);
  const uint32_t cp2 = next_pow2((uint32_t)max(nc, 1));
  for (int i = threadIdx.x; i < (int)cp2; i += blockDim.x) w.cand[i] = ~0ull;
  __syncthreads();
  for (int u = threadIdx.x; u < nu; u += blockDim.x)
    if (w.flags[u]) w.cand[w.tmp[u]] = ((uint64_t)(16 - __popc(w.umask[u])) << 32) | (uint32_t)u;
  bitonic_sort(w.cand, cp2);
  // chunks of 8 in candidate order; a chunk is kept when its count sum over
  // window * 8 reaches tc_min_util; thread 0 walks the (few) candidates
  if (threadIdx.x == 0) {
    int kept = 0;
    for (int s = 0; s < nc; s += 8) {
      const int e = min(s + 8, nc), m = e - s;
      int us[8];
      int nnz = 0;
      for (int i = 0; i < m; ++i) {
        us[i] = (int)(uint32_t)w.cand[s + i];
        nnz += __popc(w.umask[us[i]]);
      }
      const float util = (float)nnz / (float)(p.window * 8);
      if (util < p.tc_min_util) continue;
      for (int i = 1; i < m; ++i)
        for (int j = i; j > 0 && w.ucol[us[j - 1]] > w.ucol[us[j]]; --j) {
          const int t = us[j - 1];
          us[j - 1] = us[j];
          us[j] = t;
        }
      for (int k = 0; k < 8; ++k) {
        if (k < m) w.slot[us[k]] = kept * 8 + k;
        w.gcol[kept * 8 + k] = k < m ? w.ucol[us[k]] : -1;
      }
      ++kept;
    }
    s_int[8] = kept;
  }
  __syncthreads();
  return s_int[8];
}

// A key is on the tensor cores when its column has a slot and it is the
// first key of its (column, row) (keys of a column ascend by entry, so the
// entries of one row are adjacent).
__device__ __forceinline__ bool tc_key(const WinWork& w, int i) {
  if (w.slot[w.pos[i]] < 0) return false;
  return i == 0 || (w.keys[i - 1] >> 32) != (w.keys[i] >> 32) ||
         (w.keys[i - 1] & 15u) != (w.keys[i] & 15u);
}

constexpr int kSmemRoute = 64 * 4;        // s_int scratch after the storage

// FILL == false: sub-blocks and values per window into n_sub / n_val.
// FILL == true:  the tables at sub_off / val_off.
// NOALLOC (the entry point that allocates nothing): windows beyond shared
// memory are refused (status[0] |= 1), nothing is written when any window was refused or when
// the scanned totals exceed the caller's capacities (status[0] |= 2), and
// each sub-block's value count goes to sub_nval[sb + s] for the caller's
// t_block_offset (sub_nval = t_block_offset + 1).
template <bool FILL, bool NOALLOC = false>
__global__ void __launch_bounds__(kRThreads) tc_funnel_kernel(
    const int32_t* __restrict__ indptr, const int32_t* __restrict__ indices,
    const float* __restrict__ values, int n_rows, RouteGpuParams p,
    const int64_t* __restrict__ big_off, uint8_t* big_scratch, int* n_sub, int* n_val,
    const int* __restrict__ sub_off, const int* __restrict__ val_off, int32_t* t_column,
    int64_t* t_binary, float* t_value, int32_t* t_edge, int32_t* sub_nval, int* status = nullptr) {
  extern __shared__ __align__(16) uint8_t smem_route[];
  int* s_int = reinterpret_cast<int*>(smem_route + storage_bytes(kSmemKeys));
  const int wi = blockIdx.x;
  const int r0 = wi * 16, r1 = min(r0 + 16, n_rows);
  const int e0 = indptr[r0];
  const int n = indptr[r1] - e0;
  WinWork w;
  if (NOALLOC) {
    if (n > kSmemKeys) {
      if (threadIdx.x == 0) {
        atomicOr(status, 1);
        if (!FILL) n_sub[wi] = n_val[wi] = 0;
      }
      return;
    }
    if (FILL && status[0]) return;
  }
  if (n <= kSmemKeys) bind_storage(w, smem_route, kSmemKeys);
  else bind_storage(w, big_scratch + big_off[wi], next_pow2((uint32_t)n));
  const int kept = window_groups(indptr, indices, r0, r1, p, w, s_int);
  if (!FILL) {
    int cnt = 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) cnt += (kept > 0 && tc_key(w, i)) ? 1 : 0;
    cnt = __reduce_add_sync(0xffffffffu, cnt);
    if (threadIdx.x == 0) s_int[9] = 0;
    __syncthreads();
    if ((threadIdx.x & 31) == 0) atomicAdd(&s_int[9], cnt);
    __syncthreads();
    if (threadIdx.x == 0) {
      n_sub[wi] = kept;
      n_val[wi] = s_int[9];
    }
    return;
  }
  if (kept == 0) return;
  for (int s = threadIdx.x; s < kept; s += blockDim.x) w.glo[s] = w.ghi[s] = 0ull;
  __syncthreads();
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    if (!tc_key(w, i)) continue;
    const int sl = w.slot[w.pos[i]], lr = (int)(w.keys[i] & 15u), s = sl >> 3, k = sl & 7;
    if (lr >= 8) atomicOr(reinterpret_cast<unsigned long long*>(&w.ghi[s]), 1ull << ((lr - 8) * 8 + k));
    else atomicOr(reinterpret_cast<unsigned long long*>(&w.glo[s]), 1ull << (lr * 8 + k));
  }
  __syncthreads();
  const int sb = sub_off[wi];
  for (int s = threadIdx.x; s < kept; s += blockDim.x) {
    t_binary[2 * (int64_t)(sb + s)] = (int64_t)w.glo[s];
    t_binary[2 * (int64_t)(sb + s) + 1] = (int64_t)w.ghi[s];
    sub_nval[sb + s] = __popcll(w.glo[s]) + __popcll(w.ghi[s]);
    for (int k = 0; k < 8; ++k) t_column[(int64_t)(sb + s) * 8 + k] = w.gcol[s * 8 + k];
  }
  // values start, per sub-block, after the window's earlier sub-blocks
  if (threadIdx.x == 0) {
    int acc = 0;
    for (int s = 0; s < kept; ++s) {
      w.tmp[s] = acc;
      acc += __popcll(w.glo[s]) + __popcll(w.ghi[s]);
    }
  }
  __syncthreads();
  const int vb = val_off[wi];
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    if (!tc_key(w, i)) continue;
    const int sl = w.slot[w.pos[i]], lr = (int)(w.keys[i] & 15u), s = sl >> 3, k = sl & 7;
    const int bit = lr >= 8 ? (lr - 8) * 8 + k : lr * 8 + k;
    const int rank = lr >= 8 ? __popcll(w.glo[s]) + __popcll(w.ghi[s] & ((1ull << bit) - 1ull))
                             : __popcll(w.glo[s] & ((1ull << bit) - 1ull));
    const int e = e0 + (int)((w.keys[i] >> 4) & 0x0FFFFFFFu);
    t_value[vb + w.tmp[s] + rank] = values[e];
    if (t_edge) t_edge[vb + w.tmp[s] + rank] = e;
  }
}

template <typename T>
struct DevArr {
  T* p = nullptr;
  ~DevArr() { if (p) cudaFree(p); }
  int alloc(size_t n) {
    cudaError_t e = cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T));
    return e == cudaSuccess ? TR_OK : cuda_fail(e, "cudaMalloc (gpu router)");
  }
};

}  // namespace

int route_tc_gpu(const int32_t* d_indptr, const int32_t* d_indices, const float* d_values,
                 int32_t n_rows, const RouteGpuParams& p, TcTables& out, std::string& err) {
  out = TcTables();
  if (n_rows <= 0) return TR_OK;
  const int W = (n_rows + 15) / 16;
  std::vector<int32_t> indptr(n_rows + 1);
  TRS_CUDA(cudaMemcpy(indptr.data(), d_indptr, (n_rows + 1) * 4, cudaMemcpyDeviceToHost));
  if (indptr[n_rows] > 0 && (!d_indices || !d_values)) { err = "null indices or values"; return TR_ERR_ARG; }
  // global scratch slices for windows beyond shared memory
  std::vector<int64_t> big_off(W, 0);
  int64_t big_bytes = 0;
  for (int w = 0; w < W; ++w) {
    const int n = indptr[std::min(w * 16 + 16, n_rows)] - indptr[w * 16];
    if (n > kSmemKeys) {
      big_off[w] = big_bytes;
      big_bytes += (storage_bytes(next_pow2((uint32_t)n)) + 255) / 256 * 256;
    }
  }
  DevArr<int64_t> d_big_off;
  DevArr<uint8_t> d_big;
  DevArr<int> d_nsub, d_nval, d_soff, d_voff;
  int rc;
  if ((rc = d_big_off.alloc(W)) || (rc = d_big.alloc(big_bytes)) || (rc = d_nsub.alloc(W)) ||
      (rc = d_nval.alloc(W)) || (rc = d_soff.alloc(W)) || (rc = d_voff.alloc(W)))
    return rc;
  TRS_CUDA(cudaMemcpy(d_big_off.p, big_off.data(), W * 8, cudaMemcpyHostToDevice));
  const int smem = (int)storage_bytes(kSmemKeys) + kSmemRoute;
  if ((rc = kernel_smem_limit((const void*)tc_funnel_kernel<false>, smem)) ||
      (rc = kernel_smem_limit((const void*)tc_funnel_kernel<true>, smem)))
    return rc;
  tc_funnel_kernel<false><<<W, kRThreads, smem>>>(d_indptr, d_indices, d_values, n_rows, p,
                                                  d_big_off.p, d_big.p, d_nsub.p, d_nval.p, nullptr,
                                                  nullptr, nullptr, nullptr, nullptr, nullptr,
                                                  nullptr);
  TRS_CUDA(cudaGetLastError());
  std::vector<int> nsub(W), nval(W), soff(W), voff(W);
  TRS_CUDA(cudaMemcpy(nsub.data(), d_nsub.p, W * 4, cudaMemcpyDeviceToHost));
  TRS_CUDA(cudaMemcpy(nval.data(), d_nval.p, W * 4, cudaMemcpyDeviceToHost));
  int64_t tsub = 0, tval = 0;
  for (int w = 0; w < W; ++w) {
    soff[w] = (int)tsub;
    voff[w] = (int)tval;
    tsub += nsub[w];
    tval += nval[w];
  }
  if (tsub > INT32_MAX / 8 || tval > INT32_MAX) { err = "too many tensor-core entries"; return TR_ERR_UNSUPPORTED; }
  TRS_CUDA(cudaMemcpy(d_soff.p, soff.data(), W * 4, cudaMemcpyHostToDevice));
  TRS_CUDA(cudaMemcpy(d_voff.p, voff.data(), W * 4, cudaMemcpyHostToDevice));
  DevArr<int32_t> d_col, d_edge, d_snval;
  DevArr<int64_t> d_bin;
  DevArr<float> d_val;
  if ((rc = d_col.alloc(tsub * 8)) || (rc = d_bin.alloc(tsub * 2)) || (rc = d_val.alloc(tval)) ||
      (rc = d_edge.alloc(tval)) || (rc = d_snval.alloc(tsub)))
    return rc;
  tc_funnel_kernel<true><<<W, kRThreads, smem>>>(d_indptr, d_indices, d_values, n_rows, p,
                                                 d_big_off.p, d_big.p, nullptr, nullptr, d_soff.p,
                                                 d_voff.p, d_col.p, d_bin.p, d_val.p, d_edge.p,
                                                 d_snval.p);
  TRS_CUDA(cudaGetLastError());
  TRS_CUDA(cudaDeviceSynchronize());
  out.t_column.resize(tsub * 8);
  out.t_binary.resize(tsub * 2);
  out.t_value.resize(tval);
  out.t_edge.resize(tval);
  std::vector<int32_t> snval(tsub);
  if (tsub) {
    TRS_CUDA(cudaMemcpy(out.t_column.data(), d_col.p, tsub * 8 * 4, cudaMemcpyDeviceToHost));
    TRS_CUDA(cudaMemcpy(out.t_binary.data(), d_bin.p, tsub * 2 * 8, cudaMemcpyDeviceToHost));
    TRS_CUDA(cudaMemcpy(snval.data(), d_snval.p, tsub * 4, cudaMemcpyDeviceToHost));
  }
  if (tval) {
    TRS_CUDA(cudaMemcpy(out.t_value.data(), d_val.p, tval * 4, cudaMemcpyDeviceToHost));
    TRS_CUDA(cudaMemcpy(out.t_edge.data(), d_edge.p, tval * 4, cudaMemcpyDeviceToHost));
  }
  // value offsets per sub-block; parts of partsize_t sub-blocks per window
  out.t_block_offset.assign(1, 0);
  for (int64_t s = 0; s < tsub; ++s) out.t_block_offset.push_back(out.t_block_offset.back() + snval[s]);
  out.t_row_offset.assign(1, 0);
  const int pt = std::max(p.partsize_t, 1);
  for (int w = 0; w < W; ++w) {
    const int ns = nsub[w];
    if (ns == 0) continue;
    auto part = [&](int cnt) {
      out.t_row_offset.push_back(out.t_row_offset.back() + cnt);
      out.t_window_row.push_back(w * 16);
    };
    if (ns <= pt) {
      part(ns);
    } else {
      for (int q = 0; q < ns / pt; ++q) part(pt);
      if (ns % pt) part(ns % pt);
    }
  }
  return TR_OK;
}

// ---------------------------------------------------------------------------
// The entry point that allocates nothing (tr_route_tc_device_noalloc)
// ---------------------------------------------------------------------------
// Its scratch — per-window sub-block and value counts, their exclusive
// scans, and four status / total words — lives in one file-scope device
// array, held by every GPU that loads the library until the process exits.
// Host code never passes the array's name to a kernel (on the host the name
// is only a stand-in): the device address comes from cudaGetSymbolAddress,
// taken once per device with that device current.
constexpr int kNoAllocMaxWindows = 65536;                 // 1,048,576 rows
constexpr int kNoAllocWords = 4 * kNoAllocMaxWindows + 4; // 1 MiB + 16 bytes
static __device__ __align__(256) int g_noalloc_scratch[kNoAllocWords];

namespace {

// Exclusive scans of n_sub and n_val over W windows (one block), totals in
// status[1] / status[2]; status[0] |= 2 when a total exceeds its capacity.
__global__ void noalloc_scan_kernel(const int* n_sub, const int* n_val, int W, int* sub_off,
                                    int* val_off, int* status, long long cap_sub, long long cap_val) {
  __shared__ long long carry[2];
  __shared__ int wt[2][32];
  if (threadIdx.x == 0) carry[0] = carry[1] = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int c0 = 0; c0 < W; c0 += blockDim.x) {
    const int i = c0 + threadIdx.x;
    const int a = i < W ? n_sub[i] : 0, b = i < W ? n_val[i] : 0;
    int xa = a, xb = b;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const int ya = __shfl_up_sync(0xffffffffu, xa, off), yb = __shfl_up_sync(0xffffffffu, xb, off);
      if (lane >= off) { xa += ya; xb += yb; }
    }
    if (lane == 31) { wt[0][warp] = xa; wt[1][warp] = xb; }
    __syncthreads();
    long long ba = 0, bb = 0, ta = 0, tb = 0;
    for (int w = 0; w < nw; ++w) {
      if (w < warp) { ba += wt[0][w]; bb += wt[1][w]; }
      ta += wt[0][w];
      tb += wt[1][w];
    }
    if (i < W) {
      sub_off[i] = (int)(carry[0] + ba + xa - a);
      val_off[i] = (int)(carry[1] + bb + xb - b);
    }
    __syncthreads();
    if (threadIdx.x == 0) { carry[0] += ta; carry[1] += tb; }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    status[1] = (int)min(carry[0], (long long)INT32_MAX);
    status[2] = (int)min(carry[1], (long long)INT32_MAX);
    if (carry[0] > cap_sub || carry[1] > cap_val) atomicOr(status, 2);
  }
}

// In place: a[0] = 0, a[1..n] = inclusive prefix sums of the counts stored
// there (one block).
__global__ void noalloc_block_offsets_kernel(int32_t* a, const int* status) {
  if (status[0] != 0) return;
  const int n = status[1];
  __shared__ int wt[32];
  __shared__ int carry;
  if (threadIdx.x == 0) { carry = 0; a[0] = 0; }
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int c0 = 0; c0 < n; c0 += blockDim.x) {
    const int i = c0 + threadIdx.x;
    int x = i < n ? a[1 + i] : 0;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, x, off);
      if (lane >= off) x += y;
    }
    if (lane == 31) wt[warp] = x;
    __syncthreads();
    int before = 0, tot = 0;
    for (int w = 0; w < nw; ++w) {
      if (w < warp) before += wt[w];
      tot += wt[w];
    }
    if (i < n) a[1 + i] = carry + before + x;
    __syncthreads();
    if (threadIdx.x == 0) carry += tot;
    __syncthreads();
  }
}

// Per-device set-up: the scratch array's device address and the kernels'
// shared-memory limit, once per device.
int noalloc_setup(int** scratch) {
  static int* addr[128] = {nullptr};
  static std::mutex mu;
  int dev = 0;
  TRS_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 128) return fail(TR_ERR_UNSUPPORTED, "device ordinal beyond 127");
  std::lock_guard<std::mutex> lock(mu);
  if (!addr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(no-alloc scratch)");
    const int smem = (int)storage_bytes(kSmemKeys) + kSmemRoute;
    TRS_CUDA(cudaFuncSetAttribute(tc_funnel_kernel<false, true>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    TRS_CUDA(cudaFuncSetAttribute(tc_funnel_kernel<true, true>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    addr[dev] = static_cast<int*>(p);
  }
  *scratch = addr[dev];
  return TR_OK;
}

}  // namespace

int route_tc_gpu_noalloc(const int32_t* d_indptr, const int32_t* d_indices, const float* d_values,
                         int32_t n_rows, const RouteGpuParams& p, int32_t* t_column,
                         int64_t* t_binary, float* t_value, int32_t* t_block_offset,
                         int64_t cap_sub, int64_t cap_val, int64_t* n_sub_out,
                         int64_t* n_val_out, cudaStream_t stream) {
  if (n_rows < 0) return fail(TR_ERR_ARG, "negative row count");
  const int64_t W64 = ((int64_t)n_rows + 15) / 16;
  if (W64 > kNoAllocMaxWindows)
    return fail(TR_ERR_UNSUPPORTED, "the no-alloc router takes at most " +
                                        std::to_string((int64_t)kNoAllocMaxWindows * 16) +
                                        " rows (its scratch holds 65536 windows)");
  if (cap_sub < 0 || cap_val < 0) return fail(TR_ERR_ARG, "negative capacity");
  int* scratch = nullptr;
  int rc = noalloc_setup(&scratch);
  if (rc) return rc;
  const int W = (int)W64;
  int* n_sub = scratch;
  int* n_val = scratch + kNoAllocMaxWindows;
  int* sub_off = scratch + 2 * kNoAllocMaxWindows;
  int* val_off = scratch + 3 * kNoAllocMaxWindows;
  int* status = scratch + 4 * kNoAllocMaxWindows;
  // The status words still hold the last call's values: the only scratch
  // that must start at zero (counts and offsets are written before use).
  TRS_CUDA(cudaMemsetAsync(status, 0, 4 * sizeof(int), stream));
  if (n_rows > 0 && (!d_indices || !d_values)) {
    // null entry arrays are only valid for a matrix without entries
    int32_t nnz = 0;
    TRS_CUDA(cudaMemcpyAsync(&nnz, d_indptr + n_rows, 4, cudaMemcpyDeviceToHost, stream));
    TRS_CUDA(cudaStreamSynchronize(stream));
    if (nnz > 0) return fail(TR_ERR_ARG, "null indices or values");
  }
  int host_status[4] = {0, 0, 0, 0};
  if (W > 0) {
    const int smem = (int)storage_bytes(kSmemKeys) + kSmemRoute;
    tc_funnel_kernel<false, true><<<W, kRThreads, smem, stream>>>(
        d_indptr, d_indices, d_values, n_rows, p, nullptr, nullptr, n_sub, n_val, nullptr,
        nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, status);
    TRS_CUDA(cudaGetLastError());
    noalloc_scan_kernel<<<1, 1024, 0, stream>>>(n_sub, n_val, W, sub_off, val_off, status,
                                                cap_sub, cap_val);
    TRS_CUDA(cudaGetLastError());
    tc_funnel_kernel<true, true><<<W, kRThreads, smem, stream>>>(
        d_indptr, d_indices, d_values, n_rows, p, nullptr, nullptr, nullptr, nullptr, sub_off,
        val_off, t_column, t_binary, t_value, nullptr, t_block_offset ? t_block_offset + 1 : nullptr,
        status);
    TRS_CUDA(cudaGetLastError());
    if (t_block_offset) {
      noalloc_block_offsets_kernel<<<1, 1024, 0, stream>>>(t_block_offset, status);
      TRS_CUDA(cudaGetLastError());
    }
  } else if (t_block_offset && cap_sub >= 0) {
    TRS_CUDA(cudaMemsetAsync(t_block_offset, 0, sizeof(int32_t), stream));
  }
  TRS_CUDA(cudaMemcpyAsync(host_status, status, sizeof(host_status), cudaMemcpyDeviceToHost, stream));
  TRS_CUDA(cudaStreamSynchronize(stream));
  if (host_status[0] & 1)
    return fail(TR_ERR_UNSUPPORTED, "a 16-row window holds more than " + std::to_string(kSmemKeys) +
                                        " entries; the no-alloc router keeps windows in shared "
                                        "memory (tr_route_tc_device handles any size)");
  if (host_status[0] & 2)
    return fail(TR_ERR_ARG, "output capacity too small: need " + std::to_string(host_status[1]) +
                                " sub-blocks and " + std::to_string(host_status[2]) + " values");
  if (n_sub_out) *n_sub_out = host_status[1];
  if (n_val_out) *n_val_out = host_status[2];
  return TR_OK;
}

}  // namespace trs
