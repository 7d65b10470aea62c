// Device helpers shared by the block engine's kernels (block.cu, block_bwd.cu).
#pragma once
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "common.cuh"
#include "plan.h"

namespace trs {
namespace blk {

constexpr int kATile = 4096;            // 128 rows x 16 slots, FP16
constexpr int kEntReg = 2;              // entry words per lane held in registers
constexpr int kMaxBlk = 512;            // blocks per CTA (staged list)
constexpr int kMetaRing = 8;            // chunks of metadata staged ahead, per warp
// copy groups a producer leaves in flight: its range of chunk n + 2 was
// copied kMetaRing chunks back, so waiting for all but the newest
// kMetaRing - 3 groups suffices and never waits for recent gathers
constexpr int kMetaWait = kMetaRing - 3;
constexpr int kMetaInts = 18;           // a chunk's 16 columns and entry range
constexpr int kMetaStride = 32;         // ints per ring slot (16-byte aligned slots)
constexpr uint32_t kNoEntry = 0xFFFFFFFFu;   // empty register slot (offset past the tile)

__device__ __forceinline__ bool wait_bar(uint32_t bar, uint32_t parity, volatile int* abort) {
  if (mbar_try_wait(bar, parity)) return true;
  const unsigned long long t0 = global_timer_ns();
  while (!mbar_try_wait(bar, parity)) {
    if (*abort) return false;
    if (global_timer_ns() - t0 > kWaitLimitNs) {
      *abort = 1;
      return false;
    }
  }
  return true;
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(bar) : "memory");
}

// 32 lanes x 32 consecutive 32-bit TMEM columns.
__device__ __forceinline__ void tmem_ld_x32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,"
      "%15,%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]),
        "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]),
        "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void sts_u16(uint32_t addr, uint16_t v) {
  asm volatile("st.shared.u16 [%0], %1;\n" ::"r"(addr), "h"(v) : "memory");
}
__device__ __forceinline__ uint32_t lds_u32(uint32_t addr) {
  uint32_t v;
  asm volatile("ld.shared.u32 %0, [%1];\n" : "=r"(v) : "r"(addr) : "memory");
  return v;
}
// 4-byte global->shared copy (cp.async, L1-allocating form)
__device__ __forceinline__ void cp_async4(uint32_t dst, const void* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(dst), "l"(src) : "memory");
}
// The i-th element of a register ring, i known only at run time.
template <int N>
__device__ __forceinline__ int ring_at(const int (&r)[N], int i) {
  int v = 0;
#pragma unroll
  for (int t = 0; t < N; ++t) v = t == i ? r[t] : v;
  return v;
}

// 32 consecutive features of one output row, scaled.
template <bool F16OUT>
__device__ __forceinline__ void store_row32(void* C, int64_t at, const float (&v)[32], float sc) {
  if (F16OUT) {
    uint4* dst = reinterpret_cast<uint4*>(reinterpret_cast<__half*>(C) + at);
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      __half2 h[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) h[j] = __floats2half2_rn(v[8 * i + 2 * j] * sc, v[8 * i + 2 * j + 1] * sc);
      __stcs(dst + i, *reinterpret_cast<uint4*>(h));
    }
  } else {
    float4* dst = reinterpret_cast<float4*>(reinterpret_cast<float*>(C) + at);
#pragma unroll
    for (int i = 0; i < 8; ++i)
      __stcs(dst + i, make_float4(v[4 * i] * sc, v[4 * i + 1] * sc, v[4 * i + 2] * sc, v[4 * i + 3] * sc));
  }
}

template <bool F16OUT>
__device__ __forceinline__ void store_zero32(void* C, int64_t at) {
  if (F16OUT) {
    uint4* dst = reinterpret_cast<uint4*>(reinterpret_cast<__half*>(C) + at);
#pragma unroll
    for (int i = 0; i < 4; ++i) __stcs(dst + i, make_uint4(0, 0, 0, 0));
  } else {
    float4* dst = reinterpret_cast<float4*>(reinterpret_cast<float*>(C) + at);
#pragma unroll
    for (int i = 0; i < 8; ++i) __stcs(dst + i, make_float4(0.f, 0.f, 0.f, 0.f));
  }
}

// Arrive on `bar` once all of this thread's earlier cp.async copies have
// landed; the arrival is counted in the barrier's expected count.
__device__ __forceinline__ void cp_async_arrive_noinc(uint32_t bar) {
  asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];\n" ::"r"(bar) : "memory");
}

__device__ __forceinline__ uint4 lds_u128(uint32_t addr) {
  uint4 v;
  asm volatile("ld.shared.v4.u32 {%0, %1, %2, %3}, [%4];\n"
               : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w) : "r"(addr) : "memory");
  return v;
}

// Gather lanes: with 8 * NA 16-byte segments per 256 * NA-byte row, a warp
// instruction copies 32 / (8 * NA) rows, lane l taking row t * G + l / (8 * NA)
// of instruction t (G = rows per instruction).  A chunk's 16 columns are
// stored in its metadata ring slot grouped by lane group (G groups of
// 16 / G rows), so a lane reads its columns with 16-byte loads; K = 192
// (rows split across instructions) reads all 16 columns and shuffles.
template <int NA> struct RowsPerLane { static constexpr int value = NA == 3 ? 4 * NA : 16 / (32 / (8 * NA)); };
template <int NA>
__device__ __forceinline__ int col_pos(int k) {
  if constexpr (NA == 3) {
    return k;
  } else {
    constexpr int G = 32 / (8 * NA), R = 16 / G;     // lane groups, rows per lane
    return (k % G) * R + k / G;
  }
}

// Position in this CTA's chunk stream: chunk id of stream index q (q only
// grows), walking the staged block list.
struct StreamCursor {
  const int* c0;
  const int* c1;
  int nblk, i = 0, q0 = 0, qend = -1, base = 0;
  __device__ int chunk(int q) {
    if (q >= qend) {       // shared memory is read only when q leaves the block
      if (qend < 0) {
        qend = c1[0] - c0[0];
        base = c0[0];
      }
      while (i < nblk - 1 && q >= qend) {
        q0 = qend;
        ++i;
        qend = q0 + (c1[i] - c0[i]);
        base = c0[i];
      }
    }
    return base + (q - q0);
  }
};

__device__ __forceinline__ uint32_t ld_stream_u32(const uint32_t* p, uint64_t policy) {
  uint32_t v;
  asm volatile("ld.global.nc.L2::cache_hint.b32 %0, [%1], %2;\n" : "=r"(v) : "l"(p), "l"(policy));
  return v;
}

}  // namespace blk
}  // namespace trs
