// Block-wide sorting and compaction helpers of the device router kernels.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace trs {

__host__ __device__ inline uint32_t next_pow2(uint32_t n) {
  uint32_t p = 1;
  while (p < n) p <<= 1;
  return p;
}

// Ascending block-wide bitonic sort of a[0, n) (n a power of two).
static __device__ void bitonic_sort(uint64_t* a, uint32_t n) {
  for (uint32_t k = 2; k <= n; k <<= 1)
    for (uint32_t j = k >> 1; j > 0; j >>= 1) {
      __syncthreads();
      for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
        const uint32_t l = i ^ j;
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

// Exclusive scan of flags[0, n) into out (ballot + popc per warp, then the
// warp totals); returns the number of set flags.  Every thread calls it.
static __device__ int block_flag_scan(const uint8_t* flags, int n, int* out, int* warp_tot) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  int base = 0;
  for (int c0 = 0; c0 < n; c0 += blockDim.x) {
    const int i = c0 + threadIdx.x;
    const bool f = i < n && flags[i];
    const unsigned bal = __ballot_sync(0xffffffffu, f);
    if (lane == 0) warp_tot[warp] = __popc(bal);
    __syncthreads();
    int before = 0, total = 0;
    for (int w = 0; w < nw; ++w) {
      before += w < warp ? warp_tot[w] : 0;
      total += warp_tot[w];
    }
    if (i < n) out[i] = base + before + __popc(bal & ((1u << lane) - 1u));
    base += total;
    __syncthreads();
  }
  return base;
}

}  // namespace trs
