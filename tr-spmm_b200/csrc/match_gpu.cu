// Online 2:4 matching statistics on the GPU (the reference's
// matching_utils_online.match_2to4_online, TR-source/Block/block_matching_online.cu
// :112-411, rebuilt with a deterministic column order).
//
// One CTA per 16-row window.  The window's (column, row-bit) keys are sorted
// with a block bitonic sort, so the window's distinct columns come out in id
// order (the reference takes them in hash-slot arrival order, which varies
// from run to run); warp 0 merges each column's row bits into its 16-bit
// mask and then runs the matching itself with ballots: 1:2 pairs (each
// column against the next 32 unused ones, cheapest common-row count first,
// nearest first), 2:4 groups (each pair against the next 1024 unused pairs,
// first conflict-free one), and the pool of columns that fail either step
// (blocks of dense_threshold columns, then groups of at most two).  The
// decisions are those of the sliding variant; a group counts 32 slots.
// Windows with more than kMatchCap entries are flagged and counted on the
// host by the same rules (the reference drops their columns past 2048).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/trspmm.h"
#include "common.cuh"

namespace trs {

void match_online_window(const int32_t* indptr, const int32_t* indices, int32_t n_rows, int w,
                         int32_t dense_threshold, int32_t t_max, int64_t* out7);

namespace {

constexpr int kMatchCap = 2048;        // entries of a window matched on the GPU
constexpr int kMatchThreads = 256;
constexpr int kOut = 8;                // counters per window

__device__ void sort_keys(uint64_t* a, int n) {     // ascending, n a power of two
  for (int k = 2; k <= n; k <<= 1)
    for (int j = k >> 1; j > 0; j >>= 1) {
      __syncthreads();
      for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const int l = i ^ j;
        if (l > i) {
          const uint64_t x = a[i], y = a[l];
          if ((x > y) == ((i & k) == 0)) {
            a[i] = y;
            a[l] = x;
          }
        }
      }
    }
  __syncthreads();
}

// out[w*8 + 0..6] = groups, dense blocks, unpaired columns, ungrouped pair
// columns, fake zeros, pool columns in dense blocks, pool columns in groups;
// out[w*8 + 7] = 1 when the window exceeds kMatchCap entries (not counted).
__global__ void __launch_bounds__(kMatchThreads) online_match_kernel(
    const int32_t* __restrict__ indptr, const int32_t* __restrict__ indices, int n_rows,
    int dense_threshold, int t_max, long long* __restrict__ out) {
  __shared__ uint64_t keys[kMatchCap];
  __shared__ uint16_t cmask[kMatchCap];
  __shared__ uint8_t used[kMatchCap];
  __shared__ uint16_t pg1[kMatchCap / 2], pg2[kMatchCap / 2], pc1[kMatchCap / 2], pc2[kMatchCap / 2];
  __shared__ uint8_t pused[kMatchCap / 2];
  __shared__ uint16_t pool[kMatchCap];
  const int w = blockIdx.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int r0 = w * 16, r1 = min(r0 + 16, n_rows);
  const int e0 = indptr[r0], n = indptr[r1] - e0;
  long long* o = out + (size_t)w * kOut;
  if (n > kMatchCap || n == 0) {
    if (tid < kOut) o[tid] = (tid == 7 && n > kMatchCap) ? 1 : 0;
    return;
  }
  int np2 = 1;
  while (np2 < n) np2 <<= 1;
  for (int r = r0 + warp; r < r1; r += kMatchThreads / 32) {
    const uint64_t bit = 1ull << (r - r0);
    for (int e = indptr[r] + lane; e < indptr[r + 1]; e += 32)
      keys[e - e0] = ((uint64_t)(uint32_t)indices[e] << 32) | bit;
  }
  for (int i = n + tid; i < np2; i += kMatchThreads) keys[i] = ~0ull;
  sort_keys(keys, np2);
  if (warp != 0) return;

  // ---- distinct columns in id order, with their row masks -------------------
  int nc = 0;
  for (int b = 0; b < n; b += 32) {
    const int i = b + lane;
    const bool head = i < n && (i == 0 || (keys[i] >> 32) != (keys[i - 1] >> 32));
    const unsigned bal = __ballot_sync(0xffffffffu, head);
    if (head) {
      uint32_t m = 0;
      for (int j = i; j < n && (keys[j] >> 32) == (keys[i] >> 32); ++j) m |= (uint32_t)keys[j];
      const int at = nc + __popc(bal & ((1u << lane) - 1u));
      cmask[at] = (uint16_t)m;
      used[at] = 0;
    }
    nc += __popc(bal);
  }
  __syncwarp();

  // ---- 1:2 pairs ------------------------------------------------------------
  // a partner with no common row is taken whatever t_max is (as on the host)
  const int tmax = max(0, min(t_max, 16));
  int np = 0, nd = 0;
  long long fine = 0, coarse = 0, fz = 0, groups = 0;
  for (int i = 0; i < nc; ++i) {
    if (used[i]) continue;                             // uniform: shared-memory flag
    const uint32_t mi = cmask[i];
    const int j = i + 1 + lane;
    const int cost = (j < nc && !used[j]) ? __popc(mi & cmask[j]) : 99;
    int best = -1;
    for (int c = 0; c <= tmax && best < 0; ++c) {
      const unsigned bal = __ballot_sync(0xffffffffu, cost == c);
      if (bal) best = i + __ffs(bal);
    }
    if (lane == 0) {
      used[i] = 1;
      if (best >= 0) {
        used[best] = 1;
        pg1[np] = (uint16_t)(mi & cmask[best]);
        pg2[np] = (uint16_t)(mi | cmask[best]);
        pc1[np] = (uint16_t)i;
        pc2[np] = (uint16_t)best;
        pused[np] = 0;
      } else {
        pool[nd] = (uint16_t)i;
      }
    }
    if (best >= 0) ++np; else { ++nd; ++fine; }
    __syncwarp();
  }

  // ---- 2:4 groups -----------------------------------------------------------
  for (int i = 0; i < np; ++i) {
    if (pused[i]) continue;
    const uint32_t a1 = pg1[i], a2 = pg2[i];
    const int jend = min(i + 1 + 1024, np);
    int found = -1;
    for (int b = i + 1; b < jend && found < 0; b += 32) {
      const int j = b + lane;
      const bool ok = j < jend && !pused[j] && ((a1 & pg2[j]) | (a2 & pg1[j])) == 0;
      const unsigned bal = __ballot_sync(0xffffffffu, ok);
      if (bal) found = b + __ffs(bal) - 1;
    }
    if (found >= 0) {
      ++groups;
      fz += 32 - (__popc(cmask[pc1[i]]) + __popc(cmask[pc2[i]]) + __popc(cmask[pc1[found]]) +
                  __popc(cmask[pc2[found]]));
    } else {
      coarse += 2;
    }
    if (lane == 0) {
      pused[i] = 1;
      if (found >= 0) {
        pused[found] = 1;
      } else {
        pool[nd] = pc1[i];
        pool[nd + 1] = pc2[i];
      }
    }
    if (found < 0) nd += 2;
    __syncwarp();
  }

  // ---- the pool: dense blocks, then groups of at most two columns -----------
  const int blocks = nd / dense_threshold;
  const int to_tc = blocks * dense_threshold;
  for (int k = to_tc; k < nd; k += 2) {
    int g = __popc(cmask[pool[k]]);
    if (k + 1 < nd) g += __popc(cmask[pool[k + 1]]);
    ++groups;
    fz += 32 - g;
  }
  if (lane == 0) {
    o[0] = groups;
    o[1] = blocks;
    o[2] = fine;
    o[3] = coarse;
    o[4] = fz;
    o[5] = to_tc;
    o[6] = nd - to_tc;
    o[7] = 0;
  }
}

}  // namespace

int match_online_gpu(const int32_t* indptr, const int32_t* indices, int32_t n_rows,
                     int32_t dense_threshold, int32_t t_max, tr_match_stats* st,
                     std::string& err) {
  if (n_rows <= 0) {
    err = "empty matrix (no rows or no columns)";
    return TR_ERR_ARG;
  }
  if (dense_threshold < 1) {
    err = "dense_threshold must be at least 1";
    return TR_ERR_ARG;
  }
  const int64_t nnz = indptr[n_rows];
  int32_t n_cols = 0;
  for (int64_t e = 0; e < nnz; ++e) {
    if (indices[e] < 0) {
      err = "column indices must be >= 0";
      return TR_ERR_ARG;
    }
    n_cols = std::max(n_cols, indices[e] + 1);
  }
  if (n_cols <= 0) {
    err = "empty matrix (no rows or no columns)";
    return TR_ERR_ARG;
  }
  for (int32_t r = 0; r < n_rows; ++r)
    if (indptr[r + 1] < indptr[r] || indptr[r] < 0) {
      err = "row pointers must not decrease";
      return TR_ERR_ARG;
    }
  const int W = (n_rows + 15) / 16;
  // like the reference's entry point: device copies per call, synchronous
  int32_t *d_ptr = nullptr, *d_idx = nullptr;
  long long* d_out = nullptr;
  std::vector<long long> h_out((size_t)W * kOut);
  cudaError_t e = cudaMalloc(&d_ptr, (size_t)(n_rows + 1) * 4);
  if (e == cudaSuccess) e = cudaMalloc(&d_idx, (size_t)std::max<int64_t>(nnz, 1) * 4);
  if (e == cudaSuccess) e = cudaMalloc(&d_out, h_out.size() * sizeof(long long));
  if (e == cudaSuccess) e = cudaMemcpy(d_ptr, indptr, (size_t)(n_rows + 1) * 4, cudaMemcpyHostToDevice);
  if (e == cudaSuccess && nnz > 0) e = cudaMemcpy(d_idx, indices, (size_t)nnz * 4, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    online_match_kernel<<<W, kMatchThreads>>>(d_ptr, d_idx, n_rows, dense_threshold, t_max, d_out);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess)
    e = cudaMemcpy(h_out.data(), d_out, h_out.size() * sizeof(long long), cudaMemcpyDeviceToHost);
  cudaFree(d_ptr);
  cudaFree(d_idx);
  cudaFree(d_out);
  if (e != cudaSuccess) {
    err = std::string("online matching: ") + cudaGetErrorString(e);
    return TR_ERR_CUDA;
  }
  tr_match_stats s{};
  s.total_rows = n_rows;
  s.total_cols = n_cols;
  s.total_nnz = nnz;
  s.sparsity = 1.0 - (double)nnz / ((double)n_rows * n_cols);
  s.num_row_panels = W;
  for (int w = 0; w < W; ++w) {
    const long long* o = &h_out[(size_t)w * kOut];
    int64_t v[7];
    if (o[7]) match_online_window(indptr, indices, n_rows, w, dense_threshold, t_max, v);
    else for (int i = 0; i < 7; ++i) v[i] = o[i];
    s.num_groups += v[0];
    s.num_tc_blocks += v[1];
    s.fine_fallback += v[2];
    s.coarse_fallback += v[3];
    s.fake_zeros += v[4];
    s.dense_to_tc_cols += v[5];
    s.dense_to_sptc_cols += v[6];
    s.num_16x16_blocks += (v[0] + 3) / 4;
    s.block_padding_groups += (v[0] + 3) / 4 * 4 - v[0];
  }
  *st = s;
  return TR_OK;
}

}  // namespace trs
