// sm_100a SpMM kernels.
//
//  seg_block_kernel   CUDA-core CSR SpMM, one CTA per 16-row window: the
//                     window's entries are cut into one segment per lane
//                     group, each group streams its segment across rows with
//                     the row sum in registers (128-bit loads of B rows, FP32
//                     accumulation).  It is the routed forward's residual
//                     pass (plan rows, heaviest windows first, row scaling,
//                     output row map) and, in natural order, the plain
//                     single-route CSR kernel.
//  routed_kernel      the fused three-route forward: one CTA per 16-row
//                     window.  The dense-TC and 2:4 tiles run on tcgen05
//                     (B rows gathered into 128-byte-swizzled shared memory,
//                     D^T[feature x row] accumulated in TMEM), the residual
//                     runs on CUDA cores (row-run engine: block_accumulate),
//                     and the epilogue adds both and stores each
//                     output element once (no atomics in global memory, no
//                     separate 2:4 buffer, no merge kernel — compare
//                     TR-source/SpMM/mGCNkernel_online.cu:1529-1727).
//  generic kernels    any K (not a multiple of 8): scalar but still on the GPU.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>

#include "common.cuh"
#include "plan.h"
#include "spmm.h"

#ifndef TRS_MIXED_FMA
#define TRS_MIXED_FMA 1
#endif

namespace trs {
namespace {

constexpr int kBlockRows = 16;      // rows per window / row block
constexpr int kWarps = 8;
constexpr int kThreads = kWarps * 32;
constexpr int kChunk = 128;         // features per pass (UMMA M)
constexpr int kUnroll = 4;          // independent 16-byte B loads in flight per lane

// Staged CUDA-core engine.  The entries of a 16-row block (row pointer rp[]
// in shared memory, absolute entry indices) are processed in chunks of up to
// kStage entries: each chunk's (column, value) pairs are first copied into
// shared memory in one coalesced pass (one exposed memory latency per chunk,
// not one per batch of B loads).  Every warp then takes an even share of the
// chunk and walks it one row run at a time, so the inner loop has no row
// tracking and no divergence: groups of L lanes (L*8 >= fc) each take one
// entry and load 16 bytes of its B row per lane, kUnroll entries per lane
// group in flight, tails predicated (value 0, a valid column).  At the end of
// a run the lane groups are reduced with shuffles and one group adds the
// row's partial sum into racc[16][kChunk] (shared, FP32) with shared atomics
// (a row can be split across warps).
constexpr int kStage = 1024;

// acc[0..7] += v * b[0..7]; FP16 operands, FP32 accumulation.  The product
// of two FP16 numbers is exact in FP32, so the mixed-precision FMA
// (fma.rn.f32.f16) equals converting both operands and using fmaf.
__device__ __forceinline__ void fma8h(float (&acc)[8], uint16_t v, const uint4& b) {
  const uint32_t w[4] = {b.x, b.y, b.z, b.w};
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const uint16_t lo = (uint16_t)(w[i] & 0xFFFFu), hi = (uint16_t)(w[i] >> 16);
#if TRS_MIXED_FMA
    asm("fma.rn.f32.f16 %0, %1, %2, %0;" : "+f"(acc[2 * i]) : "h"(lo), "h"(v));
    asm("fma.rn.f32.f16 %0, %1, %2, %0;" : "+f"(acc[2 * i + 1]) : "h"(hi), "h"(v));
#else
    const float fv = __half2float(__ushort_as_half(v));
    acc[2 * i] = fmaf(__half2float(__ushort_as_half(lo)), fv, acc[2 * i]);
    acc[2 * i + 1] = fmaf(__half2float(__ushort_as_half(hi)), fv, acc[2 * i + 1]);
#endif
  }
}

// acc[0..3] += v * b[0..3]: FP16 plan value, FP32 features (16 bytes of a B
// row) and accumulation.
__device__ __forceinline__ void fma4f(float (&acc)[4], uint16_t v, const uint4& b) {
  const float fv = __half2float(__ushort_as_half(v));
  acc[0] = fmaf(__uint_as_float(b.x), fv, acc[0]);
  acc[1] = fmaf(__uint_as_float(b.y), fv, acc[1]);
  acc[2] = fmaf(__uint_as_float(b.z), fv, acc[2]);
  acc[3] = fmaf(__uint_as_float(b.w), fv, acc[3]);
}

// One entry's contribution to a lane's features, by feature type.
__device__ __forceinline__ void seg_fma(float (&acc)[8], uint16_t v, const uint4& b) { fma8h(acc, v, b); }
__device__ __forceinline__ void seg_fma(float (&acc)[4], uint16_t v, const uint4& b) { fma4f(acc, v, b); }

__device__ __forceinline__ void stage_chunk(const int32_t* __restrict__ col,
                                            const __half* __restrict__ val, int e0, int n,
                                            int2* sent) {
  const uint16_t* v16 = reinterpret_cast<const uint16_t*>(val);
  for (int i = threadIdx.x; i < n; i += kThreads)
    sent[i] = make_int2(__ldg(col + e0 + i), (int)__ldg(v16 + e0 + i));
}

__device__ __forceinline__ void accumulate_chunk(const int* rp, int e0, int n, const int2* sent,
                                                 const __half* __restrict__ B, int K, int f0,
                                                 int fc, float* racc) {
  int L = 1;
  while (L * 8 < fc) L <<= 1;
  const int G = 32 / L;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = lane / L, li = lane % L;
  const bool active = li * 8 < fc;
  const int per = (n + kWarps - 1) / kWarps;
  const int eb = warp * per;
  const int ee = min(n, eb + per);
  if (eb >= ee) return;
  const __half* Bf = B + f0 + (active ? li * 8 : 0);
  int row = 0;
  while (rp[row + 1] - e0 <= eb) ++row;            // warp-uniform
  const int c_safe = sent[eb].x;                   // a valid column for predicated tails
  for (int i = eb; i < ee;) {
    const int rend = min(ee, rp[row + 1] - e0);
    float acc[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) acc[q] = 0.f;
    for (int j0 = i + g; j0 < rend; j0 += G * kUnroll) {
      uint4 bv[kUnroll];
      uint16_t vv[kUnroll];
#pragma unroll
      for (int u = 0; u < kUnroll; ++u) {
        const int j = j0 + u * G;
        const int2 en = j < rend ? sent[j] : make_int2(c_safe, 0);
        vv[u] = (uint16_t)en.y;
        bv[u] = __ldg(reinterpret_cast<const uint4*>(Bf + (size_t)en.x * K));
      }
#pragma unroll
      for (int u = 0; u < kUnroll; ++u) fma8h(acc, vv[u], bv[u]);
    }
    for (int off = L; off < 32; off <<= 1)
#pragma unroll
      for (int q = 0; q < 8; ++q) acc[q] += __shfl_xor_sync(0xffffffffu, acc[q], off);
    if (g == 0 && active) {
      float* dst = racc + row * kChunk + li * 8;
#pragma unroll
      for (int q = 0; q < 8; ++q) atomicAdd(dst + q, acc[q]);
    }
    i = rend;
    while (row < kBlockRows - 1 && rp[row + 1] - e0 <= i) ++row;
  }
}

// All entries of the block, chunk by chunk (every thread of the CTA calls it).
__device__ __forceinline__ void block_accumulate(const int* rp, const int32_t* __restrict__ col,
                                                 const __half* __restrict__ val,
                                                 const __half* __restrict__ B, int K, int f0,
                                                 int fc, float* racc, int2* sent) {
  const int e_begin = rp[0], e_end = rp[kBlockRows];
  for (int c0 = e_begin; c0 < e_end; c0 += kStage) {
    const int n = min(kStage, e_end - c0);
    __syncthreads();                       // previous chunk fully consumed
    stage_chunk(col, val, c0, n, sent);
    __syncthreads();
    accumulate_chunk(rp, c0, n, sent, B, K, f0, fc, racc);
  }
}

// Output stores bypass L2 retention (st.global.cs): C is written once.
template <bool F16OUT>
__device__ __forceinline__ void store_row_feature(void* C, int K, int64_t row, int f, float v) {
  if (F16OUT)
    __stcs(reinterpret_cast<__half*>(C) + row * K + f, __float2half_rn(v));
  else
    __stcs(reinterpret_cast<float*>(C) + row * K + f, v);
}

// ---------------------------------------------------------------------------
// Segment-streaming engine (the routed forward's CUDA-core residual pass)
// ---------------------------------------------------------------------------
// One CTA per 16-row window, windows in the plan's launch order (heaviest
// first, so the longest CTAs start first instead of finishing last).  Each
// staged chunk of the window's entries is cut into one even-length segment
// per lane group (L lanes of 8 features), and every group streams its
// segment across row boundaries with the row's partial sum in registers.
// When a row ends: a row that lies entirely inside the group's segment is
// scaled and stored straight to C from registers; a row cut by a segment or
// chunk boundary is added into the window's rows in shared memory with
// shared atomics, in a padded layout, slot(f) = f + f/32, where the 8
// consecutive features of each of the L lanes fall in distinct banks, and is
// stored at the end of the window together with the window's empty rows.
//
// Every group runs the same number of batches of kSegU entries (entries past
// its segment are predicated), and the full-batch / no-boundary decisions
// are warp votes, so the lane groups of a warp stay converged; a batch that
// crosses no row boundary runs without per-entry checks.  Tail padding
// happens once per segment, not once per row; entry pairs come from 128-bit
// shared loads; B addresses are 32-bit element offsets from the chunk's
// feature base.
constexpr int kSegStride = kChunk + kChunk / 32;     // padded shared row (floats)
// The forward engine takes up to 256 features per pass (one 32-lane group per
// warp at K = 256: a second pass would repeat the staging, the row tracking
// and the flushes for the other half); the padded layout stays conflict-free
// for 32 lanes of 8 features.
constexpr int kSegChunk = 256;
constexpr int kSegStrideW = kSegChunk + kSegChunk / 32;
constexpr int kSegU = 4;                             // entries per lane group and batch

template <int S = kSegStrideW>
__device__ __forceinline__ int seg_slot_w(int r, int f) { return r * S + f + (f >> 5); }

// Features per 16-byte load of a B row: 8 FP16 or 4 FP32 (the FP32-feature
// route); a pass covers 32 lanes' worth (256 FP16 / 128 FP32 features).
template <class TB> struct SegFeat { static constexpr int kPer = 8; };
template <> struct SegFeat<float> { static constexpr int kPer = 4; };

// 16 bytes of B row `col` at the lane's feature base Bf.
template <bool WIDE, class TB>
__device__ __forceinline__ uint4 seg_ldg(const TB* Bf, int col, uint32_t K) {
  return __ldg(reinterpret_cast<const uint4*>(
      WIDE ? Bf + (size_t)(uint32_t)col * K : Bf + (uint32_t)col * K));
}

// Segment length for n staged entries over `groups` lane groups (even, so
// that entry pairs stay 16-byte aligned in shared memory).
__device__ __forceinline__ int seg_len(int n, int groups) {
  return (((n + groups - 1) / groups) + 1) & ~1;
}

// Whether the entries [a, b) of a row all lie in one segment (then one lane
// group accumulates and stores the whole row).
__device__ __forceinline__ bool seg_owned(int a, int b, int e_begin, int e_end, int groups) {
  if (a >= b) return false;
  const int ca = (a - e_begin) / kStage, cb = (b - 1 - e_begin) / kStage;
  if (ca != cb) return false;
  const int c0 = e_begin + ca * kStage;
  const int seg = seg_len(min(kStage, e_end - c0), groups);
  return (a - c0) / seg == (b - 1 - c0) / seg;
}

// C[row, f .. f+N-1] = s * v[0..N-1] (N = 4 or 8, f a multiple of N; 16-byte
// streaming stores for FP32, 8- or 16-byte ones for FP16).
template <bool F16OUT, int N>
__device__ __forceinline__ void store_vec(void* C, int K, int64_t row, int f, const float* v,
                                          float s) {
  if (F16OUT) {
    uint32_t w[N / 2];
#pragma unroll
    for (int i = 0; i < N / 2; ++i) {
      const __half2 h = __floats2half2_rn(v[2 * i] * s, v[2 * i + 1] * s);
      w[i] = *reinterpret_cast<const uint32_t*>(&h);
    }
    __half* p = reinterpret_cast<__half*>(C) + row * K + f;
    if (N == 8) __stcs(reinterpret_cast<uint4*>(p), make_uint4(w[0], w[1], w[2], w[3]));
    else __stcs(reinterpret_cast<uint2*>(p), make_uint2(w[0], w[1]));
  } else {
    float4* p = reinterpret_cast<float4*>(reinterpret_cast<float*>(C) + row * K + f);
#pragma unroll
    for (int i = 0; i < N / 4; ++i)
      __stcs(p + i, make_float4(v[4 * i] * s, v[4 * i + 1] * s, v[4 * i + 2] * s, v[4 * i + 3] * s));
  }
}

// With PLAN the rows are a plan's rows: result row r is scaled by
// row_scale[r] and stored to row_out[r] (skipped when negative).  Without
// WIDE, B offsets are 32-bit (requires (number of B rows) * K < 2^31).  TB is
// the feature type: __half, or float for the FP32-feature route (FP32 B,
// FP16 plan values widened to FP32, FP32 accumulation).
template <bool F16OUT, bool PLAN, bool WIDE, class TB = __half>
__global__ void __launch_bounds__(kThreads, 4) seg_block_kernel(
    const int32_t* __restrict__ indptr, const int32_t* __restrict__ indices,
    const __half* __restrict__ values, int M, const TB* __restrict__ B, int K, void* C,
    const int32_t* __restrict__ row_out, const float* __restrict__ row_scale,
    const int32_t* __restrict__ order) {
  constexpr int NPL = SegFeat<TB>::kPer, PASS = 32 * NPL;   // features per lane / per pass
  // entries per lane group and batch: FP32 features hold half the
  // accumulators, which leaves room for twice the gathers in flight
  constexpr int U = NPL == 4 ? 2 * kSegU : kSegU;
  __shared__ __align__(16) float racc[kBlockRows * kSegStrideW];
  __shared__ __align__(16) int2 sent[kStage + 2];
  __shared__ int rp[kBlockRows + 1];
  __shared__ int s_out[kBlockRows];
  __shared__ float s_scale[kBlockRows];
  __shared__ int s_own[kBlockRows];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int r0 = (order ? order[blockIdx.x] : (int)blockIdx.x) * kBlockRows;
  if (tid <= kBlockRows) rp[tid] = indptr[min(r0 + tid, M)];
  if (tid < kBlockRows) {
    const bool in = r0 + tid < M;
    s_out[tid] = !in ? -1 : (PLAN ? row_out[r0 + tid] : r0 + tid);
    s_scale[tid] = (PLAN && in) ? row_scale[r0 + tid] : 1.f;
  }
  __syncthreads();
  const int e_begin = rp[0], e_end = rp[kBlockRows];
  const uint32_t uK = (uint32_t)K;
  for (int f0 = 0; f0 < K; f0 += PASS) {
    const int fc = min(PASS, K - f0);
    int L = 1;
    while (L * NPL < fc) L <<= 1;
    const int G = 32 / L, groups = kWarps * G;
    const int li = lane % L, q = warp * G + lane / L;
    const bool active = li * NPL < fc;
    if (tid < kBlockRows) s_own[tid] = seg_owned(rp[tid], rp[tid + 1], e_begin, e_end, groups);
    {
      float4* z = reinterpret_cast<float4*>(racc);
      for (int i = tid; i < kBlockRows * kSegStrideW / 4; i += kThreads) z[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    const TB* Bf = B + f0 + (active ? li * NPL : 0);
    float* dst = racc + seg_slot_w(0, active ? li * NPL : 0);
    for (int c0 = e_begin; c0 < e_end; c0 += kStage) {
      const int n = min(kStage, e_end - c0);
      __syncthreads();                       // previous chunk consumed, racc zeroed
      stage_chunk(indices, values, c0, n, sent);
      __syncthreads();
      const int seg = seg_len(n, groups);
      // every group runs the same number of batches (control flow stays
      // warp-uniform); entries at or past hi are predicated off
      const int lo0 = q * seg;               // even: entry pairs stay 16-byte aligned
      const int lo = min(n, lo0), hi = min(n, lo0 + seg);      // chunk-relative
      int r = 0;
      while (r < kBlockRows - 1 && rp[r + 1] <= c0 + lo) ++r;
      int nb = rp[r + 1] - c0;               // chunk-relative end of row r
      float acc[NPL];
#pragma unroll
      for (int i = 0; i < NPL; ++i) acc[i] = 0.f;
      // row r is done for this group: owned rows go to C, cut rows to racc
      auto flush = [&]() {
        if (!active) return;
        if (rp[r] >= c0 + lo && rp[r + 1] <= c0 + hi) {
          if (s_out[r] >= 0) store_vec<F16OUT, NPL>(C, K, s_out[r], f0 + li * NPL, acc, s_scale[r]);
        } else {
#pragma unroll
          for (int i = 0; i < NPL; ++i) atomicAdd(dst + r * kSegStrideW + i, acc[i]);
        }
      };
#pragma unroll 1
      for (int t = lo0; t < lo0 + seg; t += U) {
        uint4 b[U];
        uint32_t v[U / 2];
        if (__all_sync(0xffffffffu, t + U <= hi)) {   // full batch: no predicates
#pragma unroll
          for (int u = 0; u < U; u += 2) {
            const int4 p = *reinterpret_cast<const int4*>(&sent[t + u]);
            b[u] = seg_ldg<WIDE>(Bf, p.x, uK);
            b[u + 1] = seg_ldg<WIDE>(Bf, p.z, uK);
            v[u / 2] = __byte_perm((uint32_t)p.y, (uint32_t)p.w, 0x5410);
          }
        } else {                             // a segment's tail
#pragma unroll
          for (int u = 0; u < U; u += 2) {
            // entries at or past hi are not used; their slot is clamped to
            // stay inside sent[] (even, so the 16-byte load stays aligned)
            const int4 p = *reinterpret_cast<const int4*>(&sent[min(t + u, kStage)]);
            b[u] = t + u < hi ? seg_ldg<WIDE>(Bf, p.x, uK) : make_uint4(0u, 0u, 0u, 0u);
            b[u + 1] = t + u + 1 < hi ? seg_ldg<WIDE>(Bf, p.z, uK) : make_uint4(0u, 0u, 0u, 0u);
            v[u / 2] = __byte_perm((uint32_t)p.y, (uint32_t)p.w, 0x5410);
          }
        }
        if (__all_sync(0xffffffffu, t + U <= nb && t + U <= hi)) {   // no boundary, full
#pragma unroll
          for (int u = 0; u < U; ++u) seg_fma(acc, (uint16_t)(v[u / 2] >> (16 * (u & 1))), b[u]);
        } else {
#pragma unroll
          for (int u = 0; u < U; ++u) {
            const int j = t + u;
            if (j < hi) {
              if (j >= nb) {                   // row r ends before entry j
                flush();
#pragma unroll
                for (int i = 0; i < NPL; ++i) acc[i] = 0.f;
                do ++r; while (rp[r + 1] - c0 <= j);
                nb = rp[r + 1] - c0;
              }
              seg_fma(acc, (uint16_t)(v[u / 2] >> (16 * (u & 1))), b[u]);
            }
          }
          __syncwarp();                      // reconverge the lane groups
        }
      }
      if (lo < hi) flush();
    }
    __syncthreads();                         // every shared atomic has landed
    // rows cut by a boundary, and empty rows: one 16-byte store per lane
    for (int r = warp; r < kBlockRows; r += kWarps)
      if (!s_own[r] && s_out[r] >= 0)
        for (int f = lane * 4; f < fc; f += 128) {
          float x[4];
#pragma unroll
          for (int i = 0; i < 4; ++i) x[i] = racc[seg_slot_w(r, f + i)];
          store_vec<F16OUT, 4>(C, K, s_out[r], f0 + f, x, s_scale[r]);
        }
    __syncthreads();                         // racc and s_own are rewritten next pass
  }
}

// Any K: one thread per (row, feature).
template <bool F16OUT>
__global__ void csr_generic_kernel(const int32_t* __restrict__ indptr,
                                   const int32_t* __restrict__ indices,
                                   const __half* __restrict__ values, int M,
                                   const __half* __restrict__ B, int K, void* C) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (int64_t)M * K) return;
  const int r = (int)(idx / K), f = (int)(idx % K);
  float acc = 0.f;
  for (int e = indptr[r]; e < indptr[r + 1]; ++e)
    acc = fmaf(__half2float(values[e]), __half2float(B[(int64_t)indices[e] * K + f]), acc);
  store_row_feature<F16OUT>(C, K, r, f, acc);
}

// Kernel-internal route-mask bit: every tile of the selected routes, none of
// the CUDA-core residual entries (they were computed by another kernel).
constexpr int kTilesOnly = 64;

// Tile ranges of window w that route_mask selects: [a0, a1) dense TC tiles,
// [b0, b1) 2:4 tiles and/or promoted residual columns (which follow the 2:4
// tiles and belong to the CUDA-core route).
__device__ __forceinline__ void route_ranges(const PlanView& pv, int w, int mask, int& a0, int& a1,
                                             int& b0, int& b1) {
  const int t0 = pv.win_tile[w], split = pv.win_split[w], prom = pv.win_prom[w],
            t1 = pv.win_tile[w + 1];
  a0 = t0;
  a1 = (mask & TR_ROUTE_TC) ? split : t0;
  b0 = (mask & TR_ROUTE_SPTC) ? split : prom;
  b1 = (mask & TR_ROUTE_CUDA) ? t1 : prom;
  if (b1 < b0) b1 = b0;
}

// ---------------------------------------------------------------------------
// Fused routed forward
// ---------------------------------------------------------------------------
// Shared memory (dynamic, 1024-aligned base):
//   aop[2][kHalf][4096] A operand: 16 gathered B rows x 128 features,
//                    MN-major, 128-byte swizzle; atoms of 8 rows x 64 features:
//                    (k, f) -> (k/8)*2048 + (f/64)*1024 + (k%8)*128 +
//                              (((f%64)/8) ^ (k%8))*16 + (f%8)*2
//   bop[2][kHalf][512]  B operand: the 16x16 A tile (K-major, no swizzle)
//   racc[16][128]    residual rows (FP32)
//   scol/sval[kStage] staged indices: the window's tile columns while the
//                    tensor-core tiles are gathered, then residual entries
//   rp[17], mbar[2], tmem base
// Tiles go through a two-deep pipeline of batches of kHalf tiles: the
// cp.async gathers of batch b+1 are in flight while batch b waits for its
// copies and its MMAs run; each half of the stage buffers has its own
// mbarrier that the MMA commit arrives on.
constexpr int kHalf = 4;
constexpr int kAOpBytes = 4096;
constexpr int kBOpBytes = 512;
constexpr int kTileColCap = kStage / 16;    // tiles whose columns fit the staging buffer
constexpr int kSmemRouted = 1024 + 2 * kHalf * (kAOpBytes + kBOpBytes) + kBlockRows * kChunk * 4 +
                            kStage * 8 + 128 + 2 * kBlockRows * 4;
constexpr uint32_t kIdesc = umma_idesc_f16(128, 16, /*a MN-major*/ true, /*b MN-major*/ false);

template <bool F16OUT, bool ACC = false>
__global__ void __launch_bounds__(kThreads, 3) routed_kernel(PlanView pv, const __half* __restrict__ B,
                                                          int K, void* C, int route_mask) {
  extern __shared__ uint8_t smem_raw[];
  // 1024-byte aligned base, derived by offsetting the __shared__ array so the
  // compiler keeps it in the shared address space (LDS/STS/ATOMS, not generic)
  uint8_t* smem = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
  uint8_t* aop = smem;
  uint8_t* bop = smem + 2 * kHalf * kAOpBytes;
  float* racc = reinterpret_cast<float*>(bop + 2 * kHalf * kBOpBytes);
  int2* sent = reinterpret_cast<int2*>(racc + kBlockRows * kChunk);
  int* scol = reinterpret_cast<int*>(sent);          // tile columns while gathering tiles
  int* rp = reinterpret_cast<int*>(sent + kStage);
  uint64_t* mbar = reinterpret_cast<uint64_t*>(rp + 18);
  // the window's output rows and row scales, read once at the start so the
  // epilogue's stores wait on shared memory only
  int* s_out = reinterpret_cast<int*>(mbar + 2) + 4;
  float* s_scale = reinterpret_cast<float*>(s_out + kBlockRows);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(mbar + 2);

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int w = pv.win_order[blockIdx.x];
  const int r0 = w * kBlockRows;
  const int M = pv.n_rows;

  // tiles of the selected routes: [ta0, ta1) dense TC, [tb0, tb1) 2:4 and/or
  // promoted residual columns (2:4 tiles precede the promoted ones)
  int ta0, ta1, tb0, tb1;
  route_ranges(pv, w, route_mask, ta0, ta1, tb0, tb1);
  const int n_tc = ta1 - ta0;
  const int nt = n_tc + (tb1 - tb0);
  const bool do_res = (route_mask & TR_ROUTE_CUDA) != 0 && !(route_mask & kTilesOnly);

  if (tid <= kBlockRows) {
    const int64_t rr = (int64_t)w * kBlockRows + tid;
    rp[tid] = do_res ? pv.res_ptr[rr] : 0;
    if (tid < kBlockRows) {
      s_out[tid] = r0 + tid < M ? pv.row_out[rr] : -1;
      s_scale[tid] = pv.row_scale[rr];
    }
  }
  uint32_t tmem = 0;
  if (nt > 0) {
    if (warp == 0) {
      tmem_alloc(smem_u32(tmem_slot), 32);
      tmem_relinquish();
    }
    if (tid == 0) {
      mbar_init(smem_u32(&mbar[0]), 1);
      mbar_init(smem_u32(&mbar[1]), 1);
      fence_mbar_init();
    }
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (nt > 0) tmem = *tmem_slot;

  const uint64_t pol_keep = l2_policy_evict_last(), pol_stream = l2_policy_evict_first();
  // commits issued / waited per mbarrier; every commit is waited for, in order
  uint32_t issued[2] = {0, 0}, waited[2] = {0, 0};
  bool failed = false;
  // Waits for all outstanding commits on barrier h (thread 0 spins, bounded;
  // the barrier broadcasts the outcome so the CTA stays uniform).
  auto drain = [&](int h) -> bool {
    bool ok = true;
    if (tid == 0)
      while (ok && waited[h] < issued[h]) {
        ok = mbar_wait_bounded(smem_u32(&mbar[h]), waited[h] & 1);
        waited[h]++;
      }
    waited[h] = issued[h];
    return !__syncthreads_or(!ok);
  };

  for (int f0 = 0; f0 < K && !failed; f0 += kChunk) {
    const int fc = min(kChunk, K - f0);
    // ---- tensor-core tiles, in rounds whose columns fit the staging buffer ----
    bool first_mma = true;
    for (int rb = 0; rb < nt && !failed; rb += kTileColCap) {
      const int nr = min(kTileColCap, nt - rb);
      __syncthreads();
      for (int i = tid; i < nr * 16; i += kThreads) {
        const int ti = rb + i / 16;
        const int t = ti < n_tc ? ta0 + ti : tb0 + (ti - n_tc);
        scol[i] = __ldg(pv.tile_col + (int64_t)t * 16 + (i & 15));
      }
      __syncthreads();
      const int nbat = (nr + kHalf - 1) / kHalf;
      auto issue = [&](int b) {
        const int h = b & 1;
        const int nb = min(kHalf, nr - b * kHalf);
        for (int s = 0; s < nb; ++s) {
          const int li = b * kHalf + s;                     // tile within the round
          const int ti = rb + li;
          const int t = ti < n_tc ? ta0 + ti : tb0 + (ti - n_tc);
          const int k = tid >> 4, j = tid & 15;             // row k, 16-byte chunk j
          const int c = scol[li * 16 + k];
          const bool ok = c >= 0 && j * 8 < fc;
          const __half* src = ok ? B + (int64_t)c * K + f0 + j * 8 : B;
          const uint32_t dst = smem_u32(aop + (h * kHalf + s) * kAOpBytes) + (k >> 3) * 2048 +
                               (j >> 3) * 1024 + (k & 7) * 128 + (((j & 7) ^ (k & 7)) << 4);
          cp_async16_hint(dst, src, ok ? 16 : 0, pol_keep);
          if (tid < 32)
            cp_async16_hint(smem_u32(bop + (h * kHalf + s) * kBOpBytes) + tid * 16,
                            pv.tile_a + (int64_t)t * 256 + tid * 8, 16, pol_stream);
        }
        cp_async_commit();
      };
      if (!drain(0) || !drain(1)) { failed = true; break; }   // stage buffers free
      issue(0);
      for (int b = 0; b < nbat; ++b) {
        if (b + 1 < nbat) {
          if (!drain((b + 1) & 1)) { failed = true; break; }   // MMAs of batch b-1 done
          issue(b + 1);
          asm volatile("cp.async.wait_group 1;\n" ::: "memory");
        } else {
          cp_async_wait_all();
        }
        fence_proxy_async_smem();
        __syncthreads();
        if (tid == 0) {
          const int h = b & 1;
          const int nb = min(kHalf, nr - b * kHalf);
          tc_fence_after();
          for (int s = 0; s < nb; ++s) {
            const uint64_t adesc =
                umma_smem_desc(smem_u32(aop + (h * kHalf + s) * kAOpBytes), 1024, 2048, 2);
            const uint64_t bdesc =
                umma_smem_desc(smem_u32(bop + (h * kHalf + s) * kBOpBytes), 128, 256, 0);
            umma_f16(tmem, adesc, bdesc, kIdesc, first_mma ? 0u : 1u);
            first_mma = false;
          }
          umma_commit(smem_u32(&mbar[h]));
        }
        first_mma = false;
        issued[b & 1]++;
      }
    }
    if (failed) break;
    // ---- CUDA-core residual --------------------------------------------------
    for (int i = tid; i < kBlockRows * kChunk; i += kThreads) racc[i] = 0.f;
    if (do_res)
      block_accumulate(rp, pv.res_col, reinterpret_cast<const __half*>(pv.res_val), B, K, f0, fc,
                       racc, sent);
    __syncthreads();
    // ---- epilogue: D^T from TMEM + residual, one store per element ------------
    float d[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) d[i] = 0.f;
    if (nt > 0) {
      if (!drain(0) || !drain(1)) { failed = true; break; }
      tc_fence_after();
      const uint32_t taddr = tmem + ((uint32_t)((warp & 3) * 32) << 16) + (uint32_t)((warp >> 2) * 8);
      tmem_ld_32x32b_x8(taddr, d);
    }
    const int f = (warp & 3) * 32 + lane;
    if (f < fc) {
      float prev[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) {             // loads before any store (same pointer)
        prev[i] = 0.f;
        const int out = s_out[(warp >> 2) * 8 + i];
        if (ACC && out >= 0) {
          const int64_t at = (int64_t)out * K + f0 + f;
          prev[i] = F16OUT ? __half2float(reinterpret_cast<const __half*>(C)[at])
                           : reinterpret_cast<const float*>(C)[at];
        }
      }
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const int r = (warp >> 2) * 8 + i;
        const int out = s_out[r];
        if (out >= 0)
          store_row_feature<F16OUT>(C, K, out, f0 + f,
                                    prev[i] + (d[i] + racc[r * kChunk + f]) * s_scale[r]);
      }
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
  }
  if (failed) {
    cp_async_wait_all();
    if (tid == 0) atomicExch(pv.err, kErrMbarTimeout);
  }
  __syncthreads();
  if (nt > 0 && warp == 0) tmem_dealloc(tmem, 32);
}

// Any K: one thread per (window row, feature), scalar loads.
__device__ __forceinline__ float feat_f32(__half x) { return __half2float(x); }
__device__ __forceinline__ float feat_f32(float x) { return x; }

template <bool F16OUT, class TB = __half>
__global__ void routed_generic_kernel(PlanView pv, const TB* __restrict__ B, int K, void* C,
                                      int route_mask) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (int64_t)pv.n_rows * K) return;
  const int row = (int)(idx / K), f = (int)(idx % K);
  const int w = row / kBlockRows, n = row % kBlockRows;
  float acc = 0.f;
  int ta0, ta1, tb0, tb1;
  route_ranges(pv, w, route_mask, ta0, ta1, tb0, tb1);
  for (int t = ta0; t < tb1; ++t) {
    if (t >= ta1 && t < tb0) continue;
    for (int k = 0; k < 16; ++k) {
      const int c = pv.tile_col[(int64_t)t * 16 + k];
      if (c < 0) continue;
      const uint16_t a = pv.tile_a[(int64_t)t * 256 + (n / 8) * 128 + (k / 8) * 64 + (n % 8) * 8 + k % 8];
      acc = fmaf(__half2float(__ushort_as_half(a)), feat_f32(B[(int64_t)c * K + f]), acc);
    }
  }
  if (route_mask & TR_ROUTE_CUDA) {
    for (int e = pv.res_ptr[row]; e < pv.res_ptr[row + 1]; ++e)
      acc = fmaf(__half2float(__ushort_as_half(pv.res_val[e])),
                 feat_f32(B[(int64_t)pv.res_col[e] * K + f]), acc);
  }
  const int out = pv.row_out[row];
  if (out >= 0) store_row_feature<F16OUT>(C, K, out, f, acc * pv.row_scale[row]);
}

// ---------------------------------------------------------------------------
// FP32-feature tile pass (CUDA cores)
// ---------------------------------------------------------------------------
// The plan's 16x16 tiles (dense TC, 2:4 and promoted columns) times FP32
// features, added to C (which the residual pass has written): one CTA per
// window, warp i takes the window's tiles i, i + 8, ...  Tiles are mostly
// empty slots (a 2:4 tile holds at most half, on power-law graphs a few
// percent), so a warp first compacts its tile's nonzeros: lane l holds 8
// values of one row (row (l/16)*8 + l%8, columns 8*((l/8)%2) .. +7), counts
// its nonzeros, and a warp prefix sum places them, lane by lane, into a
// per-warp list of (column of B, row, value).  The warp then streams the
// list like residual entries: lanes over features (one 16-byte load of 4
// FP32 features per entry and lane, 4 entries in flight), the row sum in
// registers, added into the window's shared rows at each row change.
constexpr int kTileF32Chunk = 128;
constexpr int kTileF32Stride = kTileF32Chunk + kTileF32Chunk / 32;    // padded shared row

template <bool F16OUT>
__global__ void __launch_bounds__(kThreads) tile_f32_kernel(PlanView pv, const float* __restrict__ B,
                                                           int K, void* C, int route_mask) {
  __shared__ __align__(16) float racc[kBlockRows * kTileF32Stride];
  __shared__ __align__(16) int2 ent[kWarps][256 + 4];    // (column, row | value << 16)
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int w = pv.win_order[blockIdx.x];
  int ta0, ta1, tb0, tb1;
  route_ranges(pv, w, route_mask, ta0, ta1, tb0, tb1);
  const int n_tc = ta1 - ta0, nt = n_tc + (tb1 - tb0);
  if (nt == 0) return;                       // the whole CTA: no tiles in this window
  const int my_row = (lane >> 4) * 8 + (lane & 7), my_k0 = ((lane >> 3) & 1) * 8;
  for (int f0 = 0; f0 < K; f0 += kTileF32Chunk) {
    const int fc = min(kTileF32Chunk, K - f0);
    const bool active = lane * 4 < fc;
    for (int i = tid; i < kBlockRows * kTileF32Stride; i += kThreads) racc[i] = 0.f;
    __syncthreads();
    const float* Bf = B + f0 + (active ? lane * 4 : 0);
    float* dst = racc + seg_slot_w<kTileF32Stride>(0, active ? lane * 4 : 0);
    for (int ti = warp; ti < nt; ti += kWarps) {
      const int t = ti < n_tc ? ta0 + ti : tb0 + (ti - n_tc);
      // ---- compact the tile's nonzeros into ent[warp][0 .. nz) -------------
      const uint4 q = __ldg(reinterpret_cast<const uint4*>(pv.tile_a + (int64_t)t * 256) + lane);
      const uint32_t hv[4] = {q.x, q.y, q.z, q.w};
      const int my_col = lane < 16 ? __ldg(pv.tile_col + (int64_t)t * 16 + lane) : -1;
      int cj[8];
      int cnt = 0;
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        // a slot counts when its value is nonzero and its column is a column
        // of B (an empty column slot holds zeros)
        cj[j] = __shfl_sync(0xffffffffu, my_col, my_k0 + j);
        if (((hv[j >> 1] >> (16 * (j & 1))) & 0x7FFFu) == 0) cj[j] = -1;
        cnt += cj[j] >= 0 ? 1 : 0;
      }
      int pos = cnt;                          // inclusive warp scan
#pragma unroll
      for (int off = 1; off < 32; off <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, pos, off);
        if (lane >= off) pos += y;
      }
      const int nz = __shfl_sync(0xffffffffu, pos, 31);
      pos -= cnt;
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const uint32_t h = (hv[j >> 1] >> (16 * (j & 1))) & 0xFFFFu;
        if (cj[j] >= 0) ent[warp][pos++] = make_int2(cj[j], my_row | (int)(h << 16));
      }
      __syncwarp();
      // ---- stream the entries ------------------------------------------------
      float acc[4] = {0.f, 0.f, 0.f, 0.f};
      int cur = nz > 0 ? (ent[warp][0].y & 0xFFFF) : 0;
#pragma unroll 1
      for (int e0 = 0; e0 < nz; e0 += 4) {
        int2 p[4];
        uint4 b[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          p[u] = ent[warp][min(e0 + u, nz - 1)];
          b[u] = (active && e0 + u < nz)
                     ? __ldg(reinterpret_cast<const uint4*>(Bf + (int64_t)p[u].x * K))
                     : make_uint4(0u, 0u, 0u, 0u);
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          if (e0 + u < nz) {                  // warp-uniform
            const int r = p[u].y & 0xFFFF;
            if (r != cur) {
              if (active)
#pragma unroll
                for (int i = 0; i < 4; ++i) atomicAdd(dst + cur * kTileF32Stride + i, acc[i]);
              acc[0] = acc[1] = acc[2] = acc[3] = 0.f;
              cur = r;
            }
            fma4f(acc, (uint16_t)((uint32_t)p[u].y >> 16), b[u]);
          }
        }
      }
      if (nz > 0 && active)
#pragma unroll
        for (int i = 0; i < 4; ++i) atomicAdd(dst + cur * kTileF32Stride + i, acc[i]);
      __syncwarp();                          // ent[warp] is rewritten by the next tile
    }
    __syncthreads();
    for (int r = warp; r < kBlockRows; r += kWarps) {
      const int64_t pr = (int64_t)w * kBlockRows + r;
      const int out = pv.row_out[pr];
      if (out < 0) continue;
      const float sc = pv.row_scale[pr];
      for (int f = lane; f < fc; f += 32) {
        const int64_t at = (int64_t)out * K + f0 + f;
        const float x = racc[seg_slot_w<kTileF32Stride>(r, f)] * sc;
        if (F16OUT) {
          __half* cp = reinterpret_cast<__half*>(C) + at;
          *cp = __float2half_rn(__half2float(*cp) + x);
        } else {
          reinterpret_cast<float*>(C)[at] += x;
        }
      }
    }
    __syncthreads();                         // racc is cleared for the next chunk
  }
}

// ---------------------------------------------------------------------------
// Re-valuing a plan (learnable edge weights)
// ---------------------------------------------------------------------------
// Row scales of a row-scaled plan: s_r = max |v| over the row's entries.  The
// scale words start at 0; |v| >= 0 compares like its IEEE bit pattern, so an
// integer atomicMax on the bits takes the maximum.
__global__ void row_absmax_kernel(const float* __restrict__ v, const int32_t* __restrict__ erow,
                                  int64_t n, float* scale) {
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int r = erow[e];
    if (r >= 0) atomicMax(reinterpret_cast<int*>(scale + r), __float_as_int(fabsf(v[e])));
  }
}

__global__ void scatter_values_kernel(const float* __restrict__ v, const int32_t* __restrict__ slot,
                                      const int32_t* __restrict__ erow,
                                      const float* __restrict__ scale, int64_t n,
                                      int64_t n_tile_vals, __half* tile_a, __half* res_val) {
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int s = slot[e];
    if (s < 0) continue;
    float x = v[e];
    if (scale) {
      const float sr = scale[erow[e]];
      x = sr > 0.f ? x / sr : x;
    }
    if (s < n_tile_vals) tile_a[s] = __float2half_rn(x);
    else res_val[s - n_tile_vals] = __float2half_rn(x);
  }
}

// ---------------------------------------------------------------------------
// SDDMM on A's pattern: out[e] = <x[row(e)], y[col(e)]>
// ---------------------------------------------------------------------------
// One warp per row (grid-stride); lane groups of L lanes take one entry each
// and walk the feature dimension in 16-byte chunks; the row of x is re-read
// from L1 per entry.  FP16 operands, FP32 products and sums.
__device__ __forceinline__ float dot8h(const uint4& a, const uint4& b) {
  const uint32_t x[4] = {a.x, a.y, a.z, a.w}, y[4] = {b.x, b.y, b.z, b.w};
  float acc = 0.f;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const uint16_t xl = (uint16_t)(x[i] & 0xFFFFu), xh = (uint16_t)(x[i] >> 16);
    const uint16_t yl = (uint16_t)(y[i] & 0xFFFFu), yh = (uint16_t)(y[i] >> 16);
    asm("fma.rn.f32.f16 %0, %1, %2, %0;" : "+f"(acc) : "h"(xl), "h"(yl));
    asm("fma.rn.f32.f16 %0, %1, %2, %0;" : "+f"(acc) : "h"(xh), "h"(yh));
  }
  return acc;
}

// The FP32-feature form: 4 FP32 products per 16-byte chunk.
__device__ __forceinline__ float dot4f(const uint4& a, const uint4& b) {
  float acc = __uint_as_float(a.x) * __uint_as_float(b.x);
  acc = fmaf(__uint_as_float(a.y), __uint_as_float(b.y), acc);
  acc = fmaf(__uint_as_float(a.z), __uint_as_float(b.z), acc);
  return fmaf(__uint_as_float(a.w), __uint_as_float(b.w), acc);
}
__device__ __forceinline__ float dot_chunk(const uint4& a, const uint4& b, __half) { return dot8h(a, b); }
__device__ __forceinline__ float dot_chunk(const uint4& a, const uint4& b, float) { return dot4f(a, b); }

template <class TB = __half>
__global__ void __launch_bounds__(256) sddmm_kernel(const int32_t* __restrict__ indptr,
                                                    const int32_t* __restrict__ indices, int M,
                                                    const TB* __restrict__ X,
                                                    const TB* __restrict__ Y, int K,
                                                    float* __restrict__ out,
                                                    const int32_t* __restrict__ out_id) {
  const int lane = threadIdx.x & 31;
  const int nchunk = K / SegFeat<TB>::kPer;
  int L = 1;
  while (L < nchunk && L < 32) L <<= 1;
  const int G = 32 / L, g = lane / L, li = lane % L;
  const int warps = gridDim.x * (blockDim.x >> 5);
  for (int r = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); r < M; r += warps) {
    const uint4* xr = reinterpret_cast<const uint4*>(X + (int64_t)r * K);
    const int e0 = indptr[r], e1 = indptr[r + 1];
    for (int eb = e0; eb < e1; eb += G) {
      const int e = eb + g;
      float acc = 0.f;
      if (e < e1) {
        const uint4* yr = reinterpret_cast<const uint4*>(Y + (int64_t)__ldg(indices + e) * K);
        for (int c = li; c < nchunk; c += L) acc += dot_chunk(__ldg(xr + c), __ldg(yr + c), TB());
      }
      for (int off = 1; off < L; off <<= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
      if (li == 0 && e < e1) out[out_id ? out_id[e] : e] = acc;
    }
  }
}

// K = L * CH * (8 FP16 or 4 FP32 features) with L in {8, 16, 32} lanes and
// CH 16-byte chunks per lane: groups of L lanes, one row per group, the
// lane's chunks of the row of x held in registers.  A group takes the row's
// entries U at a time: every lane loads its chunks of the U rows of y
// (coalesced: the group reads whole rows), forms U partial dot products, the
// lanes are folded down to U, and the group finishes the sums with a
// reduce-scatter over its lanes (each step halves the values a lane holds
// and the lanes that share them), after which lane i holds entry i's sum:
// U - 1 shuffles per U entries instead of log2(L) per entry, and U * CH
// loads in flight per lane.  Groups of one warp step through their rows'
// batches together (warp-uniform trip count, idle groups predicated), so
// every shuffle sees the whole warp.
template <int L, int CH = 1, class TB = __half>
__global__ void __launch_bounds__(256) sddmm_group_kernel(const int32_t* __restrict__ indptr,
                                                          const int32_t* __restrict__ indices,
                                                          int M, const TB* __restrict__ X,
                                                          const TB* __restrict__ Y,
                                                          float* __restrict__ out,
                                                          const int32_t* __restrict__ out_id) {
  constexpr int K = L * CH * SegFeat<TB>::kPer, G = 32 / L, U = (L > 16 ? 16 : L) / CH;
  const int lane = threadIdx.x & 31, grp = lane / L, li = lane % L;
  const int warps = gridDim.x * (blockDim.x >> 5);
  const int warp_id = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  for (int rb = warp_id * G; rb < M; rb += warps * G) {
    const int r = rb + grp;
    const bool has_row = r < M;
    const int e0 = has_row ? __ldg(indptr + r) : 0, e1 = has_row ? __ldg(indptr + r + 1) : 0;
    uint4 xv[CH];
#pragma unroll
    for (int h = 0; h < CH; ++h)
      xv[h] = has_row ? __ldg(reinterpret_cast<const uint4*>(X + (int64_t)r * K) + li + h * L)
                      : make_uint4(0, 0, 0, 0);
    int nb = (e1 - e0 + U - 1) / U;
#pragma unroll
    for (int off = L; off < 32; off <<= 1) nb = max(nb, __shfl_xor_sync(0xffffffffu, nb, off));
    for (int bi = 0; bi < nb; ++bi) {
      const int eb = e0 + bi * U;
      // the batch's column ids: one coalesced load (lane li < U takes entry
      // eb + li), then broadcast; every row load is issued before any use,
      // slots past the row's end reading row 0 and being dropped
      const int my_c = (li < U && eb + li < e1) ? __ldg(indices + eb + li) : 0;
      uint4 yv[U][CH];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int c = __shfl_sync(0xffffffffu, my_c, grp * L + u);
#pragma unroll
        for (int h = 0; h < CH; ++h)
          yv[u][h] = __ldg(reinterpret_cast<const uint4*>(Y + (int64_t)c * K) + li + h * L);
      }
      float v[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        if constexpr (CH == 1) {
          v[u] = eb + u < e1 ? dot_chunk(xv[0], yv[u][0], TB()) : 0.f;
        } else {
          float d = dot_chunk(xv[0], yv[u][0], TB());
#pragma unroll
          for (int h = 1; h < CH; ++h) d += dot_chunk(xv[h], yv[u][h], TB());
          v[u] = eb + u < e1 ? d : 0.f;
        }
      }
      // fold the group's lanes down to U (lane bits above log2(U))
#pragma unroll
      for (int off = L / 2; off >= U; off >>= 1)
#pragma unroll
        for (int u = 0; u < U; ++u) v[u] += __shfl_xor_sync(0xffffffffu, v[u], off);
      // reduce-scatter over U lanes (lane bits li % U): value index bits follow lane bits
#pragma unroll
      for (int c = U; c > 1; c >>= 1) {
        const int m = c >> 1;
        const bool upper = (li & m) != 0;
#pragma unroll
        for (int i = 0; i < m; ++i) {
          const float send = upper ? v[i] : v[i + m];
          const float keep = upper ? v[i + m] : v[i];
          v[i] = keep + __shfl_xor_sync(0xffffffffu, send, m);
        }
      }
      const int e = eb + (li % U);
      if (li < U && e < e1) out[out_id ? out_id[e] : e] = v[0];
    }
  }
}

// ---------------------------------------------------------------------------
// Fused adjoint + SDDMM (the backward of C = A(w) . B)
// ---------------------------------------------------------------------------
// One CTA per 16 rows of the adjoint plan (rows of A^T, i.e. rows of B),
// K <= 128.  For every residual entry (row j of A^T, column i, value a, A's
// entry e) a lane group gathers 16-byte chunks of dC[i] once and uses them
// twice: dB[j] += a * dC[i] and dval[e] = <dC[i], B[j]> (a dot product with
// row j of B, held in registers while the row lasts, reduced over the group
// with shuffles).  The separate SDDMM would gather every dC row a second
// time.

// Sums 8 per-lane values over a group of L lanes (L = 8, 16 or 32) so that
// lane (li & 7) ends up with the total of value (li & 7): for L > 8 the
// group's 8-lane quarters are folded first, then each reduce-scatter step
// halves the values a lane keeps (15 shuffles for 8 sums instead of
// 8 * log2(L) at L = 8).
template <int L>
__device__ __forceinline__ float group_reduce_scatter8(float (&d)[8], int li) {
  if (L == 32) {
#pragma unroll
    for (int u = 0; u < 8; ++u) d[u] += __shfl_xor_sync(0xffffffffu, d[u], 16);
  }
  if (L >= 16) {
#pragma unroll
    for (int u = 0; u < 8; ++u) d[u] += __shfl_xor_sync(0xffffffffu, d[u], 8);
  }
#pragma unroll
  for (int c = 8; c > 1; c >>= 1) {
    const int m = c >> 1;
    const bool upper = (li & m) != 0;
#pragma unroll
    for (int i = 0; i < m; ++i) {
      const float send = upper ? d[i] : d[i + m];
      const float keep = upper ? d[i + m] : d[i];
      d[i] = keep + __shfl_xor_sync(0xffffffffu, send, m);
    }
  }
  return d[0];
}

// The fused adjoint + SDDMM on the segment-streaming engine (same segments,
// warp-uniform batches and owned-row stores as seg_block_kernel; rows cut by
// a segment boundary are added with shared atomics, or, on plans set
// deterministic, without atomics in segment order, so the result is bitwise
// repeatable).  Batches are 8 entries per lane group: each gathered
// 16-byte chunk of dC[i] feeds dB[j] += a * dC[i] and the partial dot with
// row j of B (held in registers, reloaded when the row changes), and the
// group's 8 partial dots are reduce-scattered so that lane u (< 8) writes
// dval for the batch's entry u.  K <= 256 in one pass (lane groups of 8,
// 16 or 32 lanes).  Four CTAs per SM (64 registers, a few bytes of spill)
// beat three without spill.
template <bool F16OUT, int L, bool WIDE, class TB = __half, bool DET = false>
__global__ void __launch_bounds__(kThreads, 4) seg_adjoint_sddmm_kernel(
    const int32_t* __restrict__ indptr, const int32_t* __restrict__ indices,
    const __half* __restrict__ values, const int32_t* __restrict__ edges, int M,
    const TB* __restrict__ G, int K, void* C, const int32_t* __restrict__ row_out,
    const float* __restrict__ row_scale, const TB* __restrict__ H, float* __restrict__ dval,
    const int32_t* __restrict__ order) {
  constexpr int U = 8;
  constexpr int NPL = SegFeat<TB>::kPer;                   // features per lane
  constexpr int Gn = 32 / L, groups = kWarps * Gn;
  constexpr int S = L * NPL > kChunk ? kSegStrideW : kSegStride;   // padded shared row (floats)
  constexpr int W = L * NPL;                                // features a lane group covers
  __shared__ __align__(16) float racc[kBlockRows * S];
  __shared__ __align__(16) int4 sent[kStage + 1];
  __shared__ int rp[kBlockRows + 1];
  __shared__ int s_out[kBlockRows];
  __shared__ float s_scale[kBlockRows];
  __shared__ int s_own[kBlockRows];
  // DET: per lane group and chunk, its partial sums of the rows it shares
  // with other groups: slot 0 its first row (begun before the segment),
  // slot 1 its last (running past it); dynamic shared memory, 2 * groups * W
  // floats.  Otherwise those partials go to racc by shared atomics.
  extern __shared__ __align__(16) float part[];
  __shared__ int s_cqa[kBlockRows], s_cqb[kBlockRows], s_cs0[kBlockRows];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int r0 = (order ? order[blockIdx.x] : (int)blockIdx.x) * kBlockRows;
  if (tid <= kBlockRows) rp[tid] = indptr[min(r0 + tid, M)];
  if (tid < kBlockRows) {
    const bool in = r0 + tid < M;
    s_out[tid] = in ? row_out[r0 + tid] : -1;
    s_scale[tid] = in ? row_scale[r0 + tid] : 0.f;
  }
  __syncthreads();
  const int e_begin = rp[0], e_end = rp[kBlockRows];
  const uint32_t uK = (uint32_t)K;
  const int li = lane % L, q = warp * Gn + lane / L;
  const bool active = li * NPL < K;
  if (tid < kBlockRows) s_own[tid] = seg_owned(rp[tid], rp[tid + 1], e_begin, e_end, groups);
  {
    float4* z = reinterpret_cast<float4*>(racc);
    for (int i = tid; i < kBlockRows * S / 4; i += kThreads) z[i] = make_float4(0.f, 0.f, 0.f, 0.f);
  }
  const TB* Gf = G + (active ? li * NPL : 0);
  float* dst = racc + seg_slot_w<S>(0, active ? li * NPL : 0);
  const uint16_t* v16 = reinterpret_cast<const uint16_t*>(values);
  for (int c0 = e_begin; c0 < e_end; c0 += kStage) {
    const int n = min(kStage, e_end - c0);
    __syncthreads();                         // previous chunk consumed, racc zeroed
    for (int i = tid; i < n; i += kThreads)
      sent[i] = make_int4(__ldg(indices + c0 + i), (int)__ldg(v16 + c0 + i),
                          edges ? __ldg(edges + c0 + i) : c0 + i, 0);
    __syncthreads();
    const int seg = seg_len(n, groups);
    const int lo0 = q * seg;
    const int lo = min(n, lo0), hi = min(n, lo0 + seg);        // chunk-relative
    int r = 0;
    while (r < kBlockRows - 1 && rp[r + 1] <= c0 + lo) ++r;
    const int r_first = r;
    int nb = rp[r + 1] - c0;
    // row j of B for the dot products of row r's entries
    auto load_h = [&]() {
      const int o = s_out[r];
      return (active && o >= 0) ? __ldg(reinterpret_cast<const uint4*>(H + (int64_t)o * K + li * NPL))
                                : make_uint4(0u, 0u, 0u, 0u);
    };
    uint4 hv = load_h();
    float acc[NPL];
#pragma unroll
    for (int i = 0; i < NPL; ++i) acc[i] = 0.f;
    auto flush = [&]() {
      if (!active) return;
      if (rp[r] >= c0 + lo && rp[r + 1] <= c0 + hi) {
        if (s_out[r] >= 0) store_vec<F16OUT, NPL>(C, K, s_out[r], li * NPL, acc, s_scale[r]);
      } else if constexpr (DET) {
        // a row shared with other groups: its partial waits for the
        // combine, which adds the groups' partials in group order
        float4* pp = reinterpret_cast<float4*>(part + (q * 2 + (r == r_first ? 0 : 1)) * W + li * NPL);
#pragma unroll
        for (int i = 0; i < NPL; i += 4) pp[i / 4] = make_float4(acc[i], acc[i + 1], acc[i + 2], acc[i + 3]);
      } else {
#pragma unroll
        for (int i = 0; i < NPL; ++i) atomicAdd(dst + r * S + i, acc[i]);
      }
    };
#pragma unroll 1
    for (int t = lo0; t < lo0 + seg; t += U) {
      uint4 b[U];
      uint32_t v[U / 2];
      const bool full = __all_sync(0xffffffffu, t + U <= hi);
#pragma unroll
      for (int u = 0; u < U; u += 2) {
        // entries at or past hi are not used; their slot is clamped into sent[]
        const int4 p0 = sent[full ? t + u : min(t + u, kStage)];
        const int4 p1 = sent[full ? t + u + 1 : min(t + u + 1, kStage)];
        if (full) {
          b[u] = seg_ldg<WIDE>(Gf, p0.x, uK);
          b[u + 1] = seg_ldg<WIDE>(Gf, p1.x, uK);
        } else {
          b[u] = t + u < hi ? seg_ldg<WIDE>(Gf, p0.x, uK) : make_uint4(0u, 0u, 0u, 0u);
          b[u + 1] = t + u + 1 < hi ? seg_ldg<WIDE>(Gf, p1.x, uK) : make_uint4(0u, 0u, 0u, 0u);
        }
        v[u / 2] = __byte_perm((uint32_t)p0.y, (uint32_t)p1.y, 0x5410);
      }
      float d[U];
      if (__all_sync(0xffffffffu, t + U <= nb && t + U <= hi)) {   // no boundary, full
#pragma unroll
        for (int u = 0; u < U; ++u) {
          seg_fma(acc, (uint16_t)(v[u / 2] >> (16 * (u & 1))), b[u]);
          d[u] = dot_chunk(hv, b[u], TB());
        }
      } else {
#pragma unroll
        for (int u = 0; u < U; ++u) {
          const int j = t + u;
          d[u] = 0.f;
          if (j < hi) {
            if (j >= nb) {                     // row r ends before entry j
              flush();
#pragma unroll
              for (int i = 0; i < NPL; ++i) acc[i] = 0.f;
              do ++r; while (rp[r + 1] - c0 <= j);
              nb = rp[r + 1] - c0;
              hv = load_h();
            }
            seg_fma(acc, (uint16_t)(v[u / 2] >> (16 * (u & 1))), b[u]);
            d[u] = dot_chunk(hv, b[u], TB());
          }
        }
        __syncwarp();                          // reconverge the lane groups
      }
      const float tot = group_reduce_scatter8<L>(d, li);
      if (li < 8 && t + li < hi) dval[sent[t + li].z] = tot;
    }
    if (lo < hi) flush();
    if constexpr (!DET) continue;
    // Deterministic combine: each row the chunk's segments share gets its
    // partials added in segment order.  Row r's entries a .. b of the chunk
    // lie in segments a / seg .. (b - 1) / seg; in each it is the segment's
    // first row (slot 0) unless it starts inside it (its first segment, when
    // a is not the segment's start: slot 1).  The ranges are found once per
    // row; rows a single segment stored, or without entries here, are skipped.
    if (tid < kBlockRows) {
      const int a = rp[tid] - c0, b = rp[tid + 1] - c0;
      const int a1 = max(a, 0), b1 = min(b, n);
      int qa = 0, qb = -1, s0 = 0;
      if (a1 < b1 && !(a >= 0 && b <= n && a / seg == (b - 1) / seg)) {
        qa = a1 / seg;
        qb = (b1 - 1) / seg;
        s0 = a > qa * seg ? 1 : 0;
      }
      s_cqa[tid] = qa;
      s_cqb[tid] = qb;
      s_cs0[tid] = s0;
    }
    __syncthreads();                           // every partial of this chunk is in
    for (int rr = 0; rr < kBlockRows; ++rr) {
      const int qa = s_cqa[rr], qb = s_cqb[rr];
      if (qa > qb) continue;                   // the same for every thread
      for (int f = tid; f < K; f += kThreads) {
        float sum = part[(qa * 2 + s_cs0[rr]) * W + f];
        for (int g = qa + 1; g <= qb; ++g) sum += part[g * 2 * W + f];
        racc[seg_slot_w<S>(rr, f)] += sum;
      }
    }
  }
  __syncthreads();                             // every combined row has landed
  for (int r = warp; r < kBlockRows; r += kWarps)
    if (!s_own[r] && s_out[r] >= 0)
      for (int f = lane * 4; f < K; f += 128) {
        float x[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) x[i] = racc[seg_slot_w<S>(r, f + i)];
        store_vec<F16OUT, 4>(C, K, s_out[r], f, x, s_scale[r]);
      }
}

// Any K: one thread per entry.
template <class TB = __half>
__global__ void sddmm_generic_kernel(const int32_t* __restrict__ indptr,
                                     const int32_t* __restrict__ indices, int M,
                                     const TB* __restrict__ X, const TB* __restrict__ Y,
                                     int K, float* __restrict__ out,
                                     const int32_t* __restrict__ out_id) {
  for (int r = blockIdx.x; r < M; r += gridDim.x)
    for (int e = indptr[r] + threadIdx.x; e < indptr[r + 1]; e += blockDim.x) {
      const int64_t c = indices[e];
      float acc = 0.f;
      for (int f = 0; f < K; ++f)
        acc = fmaf(feat_f32(X[(int64_t)r * K + f]), feat_f32(Y[c * K + f]), acc);
      out[out_id ? out_id[e] : e] = acc;
    }
}

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }

}  // namespace

int launch_csr(const int32_t* indptr, const int32_t* indices, const uint16_t* values, int32_t m,
               const uint16_t* b, int32_t k, void* c, int c_dtype, cudaStream_t stream) {
  if (m == 0 || k == 0) return TR_OK;
  const __half* vh = reinterpret_cast<const __half*>(values);
  const __half* bh = reinterpret_cast<const __half*>(b);
  const bool f16 = c_dtype == TR_OUT_F16;
  if (k % 8 == 0 && aligned16(b)) {
    const int blocks = (m + kBlockRows - 1) / kBlockRows;
    // natural row order, no row scaling, 64-bit B offsets (B's row count is
    // not known here)
    if (f16)
      seg_block_kernel<true, false, true><<<blocks, kThreads, 0, stream>>>(
          indptr, indices, vh, m, bh, k, c, nullptr, nullptr, nullptr);
    else
      seg_block_kernel<false, false, true><<<blocks, kThreads, 0, stream>>>(
          indptr, indices, vh, m, bh, k, c, nullptr, nullptr, nullptr);
  } else {
    const int64_t n = (int64_t)m * k;
    const int blocks = (int)((n + 255) / 256);
    if (f16) csr_generic_kernel<true><<<blocks, 256, 0, stream>>>(indptr, indices, vh, m, bh, k, c);
    else csr_generic_kernel<false><<<blocks, 256, 0, stream>>>(indptr, indices, vh, m, bh, k, c);
  }
  TRS_CUDA(cudaGetLastError());
  return TR_OK;
}

namespace {

// The plan's CUDA-core residual as a plain CSR over plan rows, each result
// row scaled and stored to its output row (every output row is written).
int launch_residual(const PlanView& v, const __half* bh, int32_t k, void* c, bool f16,
                    cudaStream_t stream) {
  const int rows = v.n_windows * kBlockRows;
  const __half* rv = reinterpret_cast<const __half*>(v.res_val);
  const bool wide = (int64_t)v.n_cols * k >= ((int64_t)1 << 31);
  if (f16) {
    if (wide)
      seg_block_kernel<true, true, true><<<v.n_windows, kThreads, 0, stream>>>(
          v.res_ptr, v.res_col, rv, rows, bh, k, c, v.row_out, v.row_scale, v.win_order);
    else
      seg_block_kernel<true, true, false><<<v.n_windows, kThreads, 0, stream>>>(
          v.res_ptr, v.res_col, rv, rows, bh, k, c, v.row_out, v.row_scale, v.win_order);
  } else {
    if (wide)
      seg_block_kernel<false, true, true><<<v.n_windows, kThreads, 0, stream>>>(
          v.res_ptr, v.res_col, rv, rows, bh, k, c, v.row_out, v.row_scale, v.win_order);
    else
      seg_block_kernel<false, true, false><<<v.n_windows, kThreads, 0, stream>>>(
          v.res_ptr, v.res_col, rv, rows, bh, k, c, v.row_out, v.row_scale, v.win_order);
  }
  TRS_CUDA(cudaGetLastError());
  return TR_OK;
}

// One CTA per window (tiles on tcgen05, residual on CUDA cores, in one
// kernel); with ACC the result is added to C.
template <bool ACC>
int launch_per_window(const PlanView& v, const __half* bh, int32_t k, void* c, bool f16,
                      int route_mask, cudaStream_t stream) {
  if (int rc = kernel_smem_limit(f16 ? (const void*)routed_kernel<true, ACC>
                                     : (const void*)routed_kernel<false, ACC>, kSmemRouted))
    return rc;
  if (f16) routed_kernel<true, ACC><<<v.n_windows, kThreads, kSmemRouted, stream>>>(v, bh, k, c, route_mask);
  else routed_kernel<false, ACC><<<v.n_windows, kThreads, kSmemRouted, stream>>>(v, bh, k, c, route_mask);
  TRS_CUDA(cudaGetLastError());
  return TR_OK;
}

}  // namespace

// Full product (route_mask == TR_ROUTE_ALL, K % 8 == 0): the CUDA-core
// residual runs as its own kernel over every window and writes C, then the
// tensor-core tiles are added to C, by the pipelined kernel where K allows
// (K % 64 == 0, K <= 256) or by the per-window kernel in accumulate mode.
// A plan without residual entries needs only the tile kernel; a plan
// without tiles only the residual kernel.  TR_ROUTE_PER_WINDOW runs the
// single fused per-window kernel instead; TR_ROUTE_PIPELINED the single
// pipelined kernel (its epilogue adding any residual).
int launch_routed(const tr_plan* p, const uint16_t* b, int32_t k, void* c, int c_dtype,
                  int route_mask, cudaStream_t stream) {
  const PlanView& v = p->view;
  if (v.n_rows == 0 || k == 0) return TR_OK;
  const __half* bh = reinterpret_cast<const __half*>(b);
  const bool f16 = c_dtype == TR_OUT_F16;
  const int sel = route_mask & (TR_ROUTE_PER_WINDOW | TR_ROUTE_PIPELINED);
  const bool residual_pass = (route_mask & TR_ROUTE_RESIDUAL_PASS) != 0;
  route_mask &= TR_ROUTE_ALL;
  const bool vec = k % 8 == 0 && aligned16(b);
  if (residual_pass && route_mask == TR_ROUTE_ALL && vec)
    return launch_residual(v, bh, k, c, f16, stream);
  const bool pipe_ok = pipe_supported(k, b) && pipe_fits(p);
  if (route_mask == TR_ROUTE_ALL && vec && sel == 0) {
    const bool tiles = p->info.tc_tiles + p->info.sptc_tiles + p->info.promoted_tiles > 0;
    const bool res = p->info.residual_nnz > 0;
    if (!tiles) return launch_residual(v, bh, k, c, f16, stream);
    if (!res && pipe_ok) return launch_pipe(p, b, k, c, c_dtype, false, stream);
    int rc = launch_residual(v, bh, k, c, f16, stream);
    if (rc) return rc;
    if (pipe_ok) return launch_pipe(p, b, k, c, c_dtype, true, stream);
    return launch_per_window<true>(v, bh, k, c, f16, TR_ROUTE_ALL | kTilesOnly, stream);
  }
  if (route_mask == TR_ROUTE_ALL && sel == TR_ROUTE_PIPELINED && pipe_ok)
    return launch_pipe(p, b, k, c, c_dtype, false, stream);
  if (vec) return launch_per_window<false>(v, bh, k, c, f16, route_mask, stream);
  const int64_t n = (int64_t)v.n_rows * k;
  const int blocks = (int)((n + 255) / 256);
  if (f16) routed_generic_kernel<true><<<blocks, 256, 0, stream>>>(v, bh, k, c, route_mask);
  else routed_generic_kernel<false><<<blocks, 256, 0, stream>>>(v, bh, k, c, route_mask);
  TRS_CUDA(cudaGetLastError());
  return TR_OK;
}

// FP32-feature route: the residual on the segment engine with FP32 B rows
// (writes every output row; zeros are stored instead when the residual is
// not selected), then the selected tiles on CUDA cores added to C.  K not a
// multiple of 4 or unaligned buffers take the scalar kernel.
int launch_routed_f32(const tr_plan* p, const float* b, int32_t k, void* c, int c_dtype,
                      int route_mask, cudaStream_t stream) {
  const PlanView& v = p->view;
  if (v.n_rows == 0 || k == 0) return TR_OK;
  const bool f16 = c_dtype == TR_OUT_F16;
  route_mask &= TR_ROUTE_ALL;
  const bool vec = k % 4 == 0 && aligned16(b) && aligned16(c);
  if (!vec) {
    const int64_t n = (int64_t)v.n_rows * k;
    const int blocks = (int)((n + 255) / 256);
    if (f16) routed_generic_kernel<true, float><<<blocks, 256, 0, stream>>>(v, b, k, c, route_mask);
    else routed_generic_kernel<false, float><<<blocks, 256, 0, stream>>>(v, b, k, c, route_mask);
    TRS_CUDA(cudaGetLastError());
    return TR_OK;
  }
  if (route_mask & TR_ROUTE_CUDA) {
    const int rows = v.n_windows * kBlockRows;
    const __half* rv = reinterpret_cast<const __half*>(v.res_val);
    const bool wide = (int64_t)v.n_cols * k >= ((int64_t)1 << 31);
#define TRS_SEGF32(F16, W)                                                                   \
  seg_block_kernel<F16, true, W, float><<<v.n_windows, kThreads, 0, stream>>>(                \
      v.res_ptr, v.res_col, rv, rows, b, k, c, v.row_out, v.row_scale, v.win_order)
    if (f16) { if (wide) TRS_SEGF32(true, true); else TRS_SEGF32(true, false); }
    else { if (wide) TRS_SEGF32(false, true); else TRS_SEGF32(false, false); }
#undef TRS_SEGF32
    TRS_CUDA(cudaGetLastError());
  } else {
    TRS_CUDA(cudaMemsetAsync(c, 0, (size_t)v.n_rows * k * (f16 ? 2 : 4), stream));
  }
  if (p->info.tc_tiles + p->info.sptc_tiles + p->info.promoted_tiles > 0) {
    if (f16) tile_f32_kernel<true><<<v.n_windows, kThreads, 0, stream>>>(v, b, k, c, route_mask);
    else tile_f32_kernel<false><<<v.n_windows, kThreads, 0, stream>>>(v, b, k, c, route_mask);
    TRS_CUDA(cudaGetLastError());
  }
  return TR_OK;
}

int launch_sddmm_f32(const int32_t* indptr, const int32_t* indices, int32_t m, int64_t nnz,
                     const float* x, const float* y, int32_t k, float* out, cudaStream_t stream,
                     const int32_t* out_id) {
  if (m == 0 || nnz == 0) return TR_OK;
  if (k == 0) {
    TRS_CUDA(cudaMemsetAsync(out, 0, (size_t)nnz * 4, stream));
    return TR_OK;
  }
  const bool vec = k % 4 == 0 && aligned16(x) && aligned16(y);
  const int blocks = (int)std::min<int64_t>(((int64_t)m + 7) / 8, 148 * 16);
  if (vec && k == 64) {
    sddmm_group_kernel<16, 1, float><<<blocks, 256, 0, stream>>>(indptr, indices, m, x, y, out, out_id);
  } else if (vec && k == 128) {
    sddmm_group_kernel<32, 1, float><<<blocks, 256, 0, stream>>>(indptr, indices, m, x, y, out, out_id);
  } else if (vec && k == 256) {
    sddmm_group_kernel<32, 2, float><<<blocks, 256, 0, stream>>>(indptr, indices, m, x, y, out, out_id);
  } else if (vec) {
    sddmm_kernel<float><<<blocks, 256, 0, stream>>>(indptr, indices, m, x, y, k, out, out_id);
  } else {
    const int blocks = (int)std::min<int64_t>(m, 148 * 32);
    sddmm_generic_kernel<float><<<blocks, 128, 0, stream>>>(indptr, indices, m, x, y, k, out, out_id);
  }
  TRS_CUDA(cudaGetLastError());
  return TR_OK;
}

int launch_set_values(tr_plan* p, const float* values, cudaStream_t stream) {
  const int64_t n = p->n_edges;
  if (n == 0) return TR_OK;
  const int threads = 256;
  const int blocks = (int)std::min<int64_t>((n + threads - 1) / threads, 148 * 32);
  if (p->row_scaled) {
    TRS_CUDA(cudaMemsetAsync(p->row_scale, 0, (size_t)p->view.n_windows * kBlockRows * 4, stream));
    row_absmax_kernel<<<blocks, threads, 0, stream>>>(values, p->edge_row, n, p->row_scale);
    TRS_CUDA(cudaGetLastError());
  }
  scatter_values_kernel<<<blocks, threads, 0, stream>>>(
      values, p->val_slot, p->edge_row, p->row_scaled ? p->row_scale : nullptr, n, p->n_tile_vals,
      reinterpret_cast<__half*>(p->tile_a), reinterpret_cast<__half*>(p->res_val));
  TRS_CUDA(cudaGetLastError());
  return TR_OK;
}

int launch_sddmm(const int32_t* indptr, const int32_t* indices, int32_t m, int64_t nnz,
                 const uint16_t* x, const uint16_t* y, int32_t k, float* out,
                 cudaStream_t stream, const int32_t* out_id) {
  if (m == 0 || nnz == 0) return TR_OK;
  const __half* xh = reinterpret_cast<const __half*>(x);
  const __half* yh = reinterpret_cast<const __half*>(y);
  if (k == 0) {
    TRS_CUDA(cudaMemsetAsync(out, 0, (size_t)nnz * 4, stream));
    return TR_OK;
  }
  const bool vec = k % 8 == 0 && aligned16(x) && aligned16(y);
  if (vec && (k == 64 || k == 128 || k == 256)) {
    const int blocks = (int)std::min<int64_t>(((int64_t)m + 7) / 8, 148 * 16);
    if (k == 64) sddmm_group_kernel<8><<<blocks, 256, 0, stream>>>(indptr, indices, m, xh, yh, out, out_id);
    else if (k == 128) sddmm_group_kernel<16><<<blocks, 256, 0, stream>>>(indptr, indices, m, xh, yh, out, out_id);
    else sddmm_group_kernel<32><<<blocks, 256, 0, stream>>>(indptr, indices, m, xh, yh, out, out_id);
  } else if (vec) {
    const int blocks = (int)std::min<int64_t>(((int64_t)m + 7) / 8, 148 * 16);
    sddmm_kernel<<<blocks, 256, 0, stream>>>(indptr, indices, m, xh, yh, k, out, out_id);
  } else {
    const int blocks = (int)std::min<int64_t>(m, 148 * 32);
    sddmm_generic_kernel<<<blocks, 128, 0, stream>>>(indptr, indices, m, xh, yh, k, out, out_id);
  }
  TRS_CUDA(cudaGetLastError());
  return TR_OK;
}

// dB = A^T . dC through the adjoint plan and dval = SDDMM(dC, B) on A's
// pattern.  Fused into one pass when the adjoint plan keeps every entry of A
// in its CUDA-core residual with its entry id (native exact plans without
// tiles), K <= 256 and K % 8 == 0; otherwise the routed adjoint and the
// SDDMM run as two launches.
int launch_adjoint_sddmm(const tr_plan* p, const int32_t* a_indptr, const int32_t* a_indices,
                         int32_t a_rows, int64_t nnz, const uint16_t* dc, const uint16_t* b,
                         int32_t k, void* db, int db_dtype, float* dval, cudaStream_t stream) {
  const PlanView& v = p->view;
  const bool f16 = db_dtype == TR_OUT_F16;
  const bool tiles = p->info.tc_tiles + p->info.sptc_tiles + p->info.promoted_tiles > 0;
  // lane groups of 8, 16 or 32 lanes (K in (32, 256]): the reduce-scatter needs 8+ lanes
  const bool fused = !tiles && k > 32 && k <= kSegChunk && k % 8 == 0 && aligned16(dc) && aligned16(b) &&
                     p->n_edges == nnz && p->info.residual_nnz == nnz && v.n_rows > 0;
  if (!fused) {
    int rc = launch_routed(p, dc, k, db, db_dtype, TR_ROUTE_ALL, stream);
    if (rc) return rc;
    return launch_sddmm(a_indptr, a_indices, a_rows, nnz, dc, b, k, dval, stream, p->edge_id);
  }
  const int rows = v.n_windows * kBlockRows;
  const int32_t* edges = p->res_edge_identity ? nullptr : v.res_edge;
  const __half* g = reinterpret_cast<const __half*>(dc);
  const __half* h = reinterpret_cast<const __half*>(b);
  const __half* rv = reinterpret_cast<const __half*>(v.res_val);
#define TRS_SEGADJ_D(F16, L, W, D)                                                        \
  do {                                                                                     \
    const int part_bytes = D ? 2 * kWarps * 32 * 8 * 4 : 0;                                \
    if (int rc = kernel_smem_limit(                                                        \
            (const void*)seg_adjoint_sddmm_kernel<F16, L, W, __half, D>, part_bytes))      \
      return rc;                                                                           \
    seg_adjoint_sddmm_kernel<F16, L, W, __half, D><<<v.n_windows, kThreads, part_bytes, stream>>>( \
        v.res_ptr, v.res_col, rv, edges, rows, g, k, db, v.row_out, v.row_scale, h, dval,      \
        v.win_order);                                                                      \
  } while (0)
#define TRS_SEGADJ(F16, L, W)                                                             \
  do {                                                                                     \
    if (p->deterministic) TRS_SEGADJ_D(F16, L, W, true);                                   \
    else TRS_SEGADJ_D(F16, L, W, false);                                                   \
  } while (0)
  const bool wide = (int64_t)v.n_cols * k >= ((int64_t)1 << 31);
  if (k > 128) {
    if (wide) { if (f16) TRS_SEGADJ(true, 32, true); else TRS_SEGADJ(false, 32, true); }
    else { if (f16) TRS_SEGADJ(true, 32, false); else TRS_SEGADJ(false, 32, false); }
  } else if (k > 64) {
    if (wide) { if (f16) TRS_SEGADJ(true, 16, true); else TRS_SEGADJ(false, 16, true); }
    else { if (f16) TRS_SEGADJ(true, 16, false); else TRS_SEGADJ(false, 16, false); }
  } else {
    if (wide) { if (f16) TRS_SEGADJ(true, 8, true); else TRS_SEGADJ(false, 8, true); }
    else { if (f16) TRS_SEGADJ(true, 8, false); else TRS_SEGADJ(false, 8, false); }
  }
#undef TRS_SEGADJ
#undef TRS_SEGADJ_D
  TRS_CUDA(cudaGetLastError());
  return TR_OK;
}

// The same with FP32 dC and B (FP32-feature route): fused for 16 < K <= 128
// (K % 4 == 0, lane groups of 8, 16 or 32 lanes of 4 features), otherwise the
// FP32 routed adjoint and the FP32 SDDMM one after the other.
int launch_adjoint_sddmm_f32(const tr_plan* p, const int32_t* a_indptr, const int32_t* a_indices,
                             int32_t a_rows, int64_t nnz, const float* dc, const float* b,
                             int32_t k, void* db, int db_dtype, float* dval, cudaStream_t stream) {
  const PlanView& v = p->view;
  const bool f16 = db_dtype == TR_OUT_F16;
  const bool tiles = p->info.tc_tiles + p->info.sptc_tiles + p->info.promoted_tiles > 0;
  const bool fused = !tiles && k > 16 && k <= kChunk && k % 4 == 0 && aligned16(dc) &&
                     aligned16(b) && aligned16(db) && p->n_edges == nnz &&
                     p->info.residual_nnz == nnz && v.n_rows > 0;
  if (!fused) {
    int rc = launch_routed_f32(p, dc, k, db, db_dtype, TR_ROUTE_ALL, stream);
    if (rc) return rc;
    return launch_sddmm_f32(a_indptr, a_indices, a_rows, nnz, dc, b, k, dval, stream, p->edge_id);
  }
  const int rows = v.n_windows * kBlockRows;
  const __half* rv = reinterpret_cast<const __half*>(v.res_val);
  const int32_t* edges = p->res_edge_identity ? nullptr : v.res_edge;
#define TRS_SEGADJ32_D(F16, L, W, D)                                                      \
  do {                                                                                     \
    const int part_bytes = D ? 2 * kWarps * 32 * 4 * 4 : 0;                                \
    if (int rc = kernel_smem_limit(                                                        \
            (const void*)seg_adjoint_sddmm_kernel<F16, L, W, float, D>, part_bytes))       \
      return rc;                                                                           \
    seg_adjoint_sddmm_kernel<F16, L, W, float, D><<<v.n_windows, kThreads, part_bytes, stream>>>( \
        v.res_ptr, v.res_col, rv, edges, rows, dc, k, db, v.row_out, v.row_scale, b, dval,      \
        v.win_order);                                                                      \
  } while (0)
#define TRS_SEGADJ32(F16, L, W)                                                           \
  do {                                                                                     \
    if (p->deterministic) TRS_SEGADJ32_D(F16, L, W, true);                                 \
    else TRS_SEGADJ32_D(F16, L, W, false);                                                 \
  } while (0)
  const bool wide = (int64_t)v.n_cols * k >= ((int64_t)1 << 31);
  if (k > 64) {
    if (wide) { if (f16) TRS_SEGADJ32(true, 32, true); else TRS_SEGADJ32(false, 32, true); }
    else { if (f16) TRS_SEGADJ32(true, 32, false); else TRS_SEGADJ32(false, 32, false); }
  } else if (k > 32) {
    if (wide) { if (f16) TRS_SEGADJ32(true, 16, true); else TRS_SEGADJ32(false, 16, true); }
    else { if (f16) TRS_SEGADJ32(true, 16, false); else TRS_SEGADJ32(false, 16, false); }
  } else {
    if (wide) { if (f16) TRS_SEGADJ32(true, 8, true); else TRS_SEGADJ32(false, 8, true); }
    else { if (f16) TRS_SEGADJ32(true, 8, false); else TRS_SEGADJ32(false, 8, false); }
  }
#undef TRS_SEGADJ32
#undef TRS_SEGADJ32_D
  TRS_CUDA(cudaGetLastError());
  return TR_OK;
}

}  // namespace trs
