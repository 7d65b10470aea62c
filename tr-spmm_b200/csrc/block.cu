// Block engine for sm_100a: C = A_plan . B over the block layout (plan.h).
//
// A block is 128 consecutive plan rows; its distinct columns are the K slots
// of 16-slot chunks.  Per chunk the tensor core computes
//     D[128 rows, N = K features] += A_chunk[128 rows, 16 slots] . B_g[16 slots, N]
// with B_g the chunk's 16 gathered feature rows, so every gathered row of B
// serves all 128 rows of the block in one tcgen05.mma (kind::f16, FP32
// accumulation in TMEM).  Each output row belongs to exactly one block and
// is written once, by one thread, in a fixed summation order: results are
// bitwise repeatable and no atomics are involved.
//
// One persistent CTA per SM walks its share of the blocks (round robin over
// the plan's cost order) as one continuous stream of chunks:
//
//   producer warps 4-7 (chunk q taken by warp 4 + q % 4)
//       wait until the chunk's stage slot is free (empty barrier), clear the
//       entries the slot's previous chunk wrote into its A tile, write this
//       chunk's FP16 values at their packed byte offsets (the tile is zero
//       elsewhere), and gather the 16 feature rows with 16-byte cp.async
//       copies straight into the 128-byte-swizzled MN-major operand layout
//       (absent slots zero-filled).  Each warp keeps up to four chunks of
//       copies in flight (cp.async groups); once a chunk's group completed it
//       fences its shared-memory writes for the async proxy and arrives on
//       the chunk's full barrier;
//   MMA warp 8 (one elected thread)
//       per chunk: wait full, one tcgen05.mma (M = 128, N = K, K = 16) into
//       the block's accumulator, commit to the slot's empty barrier; after a
//       block's last chunk commit to the accumulator's full barrier; two TMEM
//       accumulators alternate so a block's MMAs overlap the previous
//       block's epilogue;
//   epilogue warps 0-3 (thread t <-> block row t <-> TMEM lane t)
//       wait for the accumulator, tcgen05.ld the row's K values 32 at a
//       time, apply the row scale and store the row to its output position
//       (row_out); release the accumulator.  Rows of blocks without chunks
//       are written as zeros.
//
// Every wait is bounded (about a second of %globaltimer); a wait that runs
// out raises a CTA-wide abort flag, every role leaves its loop, copies and
// MMAs in flight are waited for, TMEM is freed and the plan's error word is
// set for the host to report.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "block.h"
#include "common.cuh"
#include "plan.h"

namespace trs {
namespace {

constexpr int kStages = 16;             // chunk stage slots in shared memory
constexpr int kProdWarps = 4;
constexpr int kDepth = 3;               // copy groups a producer retires late
constexpr int kEpiWarps = 4;
constexpr int kProdWarp0 = kEpiWarps;   // warps 4..7
constexpr int kMmaWarp = kProdWarp0 + kProdWarps;  // warp 8
constexpr int kBlkThreads = (kMmaWarp + 1) * 32;
constexpr int kATile = 4096;            // 128 rows x 16 slots, FP16
static_assert(kStages % kProdWarps == 0, "a stage slot always returns to the same producer warp");
static_assert(kDepth < kStages / kProdWarps, "a chunk is released before its slot is reused");

template <int NA>
struct BlkCfg {
  static constexpr int kN = 64 * NA;               // features = MMA N
  static constexpr int kBTile = 2048 * NA;         // 16 slots x kN features, FP16
  static constexpr int kStage = kBTile + kATile;   // a multiple of 1024
  static constexpr int kBarOff = kStages * kStage;
  // full[S], empty[S], acc_full[2], acc_empty[2], done; then tmem slot, abort flag
  static constexpr int kSmem = 1024 + kBarOff + (2 * kStages + 5) * 8 + 16;
  static constexpr uint32_t kTmemCols = 2 * kN <= 128 ? 128 : (2 * kN <= 256 ? 256 : 512);
  static_assert(kStage % 1024 == 0, "B tiles keep the 1024-byte swizzle alignment");
  static_assert(kSmem <= 227 * 1024, "shared memory budget");
};

int sm_count() {
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
    return 0;
  return sms;
}

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

template <bool F16OUT, int NA>
__global__ void __launch_bounds__(kBlkThreads, 1)
    block_mma_kernel(PlanView pv, const __half* __restrict__ B, void* C) {
  using Cfg = BlkCfg<NA>;
  constexpr int K = Cfg::kN;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + Cfg::kBarOff);
  uint64_t* full = bars;
  uint64_t* empty = bars + kStages;
  uint64_t* acc_full = bars + 2 * kStages;
  uint64_t* acc_empty = acc_full + 2;
  uint64_t* done = acc_empty + 2;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int NB = pv.n_blocks;
  const int nblk = NB > (int)blockIdx.x ? (NB - (int)blockIdx.x + (int)gridDim.x - 1) / (int)gridDim.x : 0;

  if (warp == kMmaWarp) {
    tmem_alloc(smem_u32(tmem_slot), Cfg::kTmemCols);
    tmem_relinquish();
  }
  if (tid == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(smem_u32(&full[s]), 1);
      mbar_init(smem_u32(&empty[s]), 1);
    }
    for (int a = 0; a < 2; ++a) {
      mbar_init(smem_u32(&acc_full[a]), 1);
      mbar_init(smem_u32(&acc_empty[a]), kEpiWarps);
    }
    mbar_init(smem_u32(done), 1);
    *abort_flag = 0;
    fence_mbar_init();
  }
  // A tiles start as zeros (a chunk writes its entries, and clears them
  // again before the slot takes the next chunk); B tiles start as zeros so
  // that no stale bit pattern meets a zero of A as Inf or NaN
  for (int s = 0; s < kStages; ++s) {
    uint4* st = reinterpret_cast<uint4*>(smem + s * Cfg::kStage);
    for (int i = tid; i < Cfg::kStage / 16; i += kBlkThreads) st[i] = make_uint4(0, 0, 0, 0);
  }
  fence_proxy_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp >= kProdWarp0 && warp < kMmaWarp) {
    // ------------------------------------------------------------ producers
    const int p = warp - kProdWarp0;
    const uint64_t pol_keep = l2_policy_evict_last(), pol_stream = l2_policy_evict_first();
    int prev0[kStages / kProdWarps], prev1[kStages / kProdWarps];   // entries of this warp's
#pragma unroll                                                     // last chunks, oldest first
    for (int i = 0; i < kStages / kProdWarps; ++i) prev0[i] = prev1[i] = 0;
    int n = 0, q = 0;
    bool ok = true;
    for (int i = 0; i < nblk && ok; ++i) {
      const int b = __ldg(pv.blk_order + blockIdx.x + i * gridDim.x);
      const int c0 = __ldg(pv.blk_chunk + b), nc = __ldg(pv.blk_chunk + b + 1) - c0;
      for (int j = ((p - q) % kProdWarps + kProdWarps) % kProdWarps; j < nc; j += kProdWarps, ++n) {
        const int chunk = c0 + j, gq = q + j;          // gq == kProdWarps * n + p
        const int s = gq % kStages, use = gq / kStages;
        const int my_col = lane < kChunkCols ? __ldg(pv.chunk_col + (int64_t)chunk * kChunkCols + lane) : -1;
        const int e0 = __ldg(pv.chunk_ent + chunk), e1 = __ldg(pv.chunk_ent + chunk + 1);
        if (!wait_bar(smem_u32(&empty[s]), (use & 1) ^ 1, abort_flag)) { ok = false; break; }
        uint8_t* st = smem + s * Cfg::kStage;
        const uint32_t a_tile = smem_u32(st + Cfg::kBTile);
        // clear the slot's previous chunk, then write this one
        for (int e = prev0[0] + lane; e < prev1[0]; e += 32)
          sts_u16(a_tile + ld_stream_u16(pv.ent_pos + e, pol_stream), 0);
        __syncwarp();
        for (int e = e0 + lane; e < e1; e += 32)
          sts_u16(a_tile + ld_stream_u16(pv.ent_pos + e, pol_stream),
                  ld_stream_u16(pv.ent_val + e, pol_stream));
#pragma unroll
        for (int t = 0; t + 1 < kStages / kProdWarps; ++t) {
          prev0[t] = prev0[t + 1];
          prev1[t] = prev1[t + 1];
        }
        prev0[kStages / kProdWarps - 1] = e0;
        prev1[kStages / kProdWarps - 1] = e1;
        // gather: 16 rows x (8 * NA) 16-byte segments, 4 * NA per lane
        const uint32_t b_tile = smem_u32(st);
#pragma unroll
        for (int t = 0; t < 4 * NA; ++t) {
          const int idx = lane + 32 * t;
          const int k = idx / (8 * NA), g = idx % (8 * NA);
          const int col = __shfl_sync(0xffffffffu, my_col, k);
          const uint32_t dst = b_tile + (k >> 3) * (NA * 1024) + (g >> 3) * 1024 + (k & 7) * 128 +
                               (((g & 7) ^ (k & 7)) << 4);
          const __half* src = B + (int64_t)(col >= 0 ? col : 0) * K + g * 8;
          cp_async16_hint(dst, src, col >= 0 ? 16 : 0, pol_keep);
        }
        cp_async_commit();
        if (n >= kDepth) {
          // the chunk kDepth behind has landed: publish it to the MMA warp
          cp_async_wait_group<kDepth>();
          fence_proxy_async_smem();
          __syncwarp();
          if (lane == 0) mbar_arrive(smem_u32(&full[(kProdWarps * (n - kDepth) + p) % kStages]));
        }
      }
      q += nc;
    }
    cp_async_wait_all();
    fence_proxy_async_smem();
    __syncwarp();
    if (ok && lane == 0)
      for (int m = max(0, n - kDepth); m < n; ++m)
        mbar_arrive(smem_u32(&full[(kProdWarps * m + p) % kStages]));
  } else if (warp == kMmaWarp) {
    // ------------------------------------------------------------ MMA issuer
    if (lane == 0) {
      constexpr uint32_t idesc = umma_idesc_f16(128, Cfg::kN, /*a MN-major*/ false, /*b MN-major*/ true);
      int q = 0, nacc = 0;
      bool ok = true;
      for (int i = 0; i < nblk && ok; ++i) {
        const int b = __ldg(pv.blk_order + blockIdx.x + i * gridDim.x);
        const int c0 = __ldg(pv.blk_chunk + b), c1 = __ldg(pv.blk_chunk + b + 1);
        if (c1 == c0) continue;
        const int a = nacc & 1, ua = nacc >> 1;
        if (!wait_bar(smem_u32(&acc_empty[a]), (ua & 1) ^ 1, abort_flag)) { ok = false; break; }
        tc_fence_after();
        const uint32_t d = tmem + (uint32_t)(a * Cfg::kN);
        for (int c = c0; c < c1; ++c, ++q) {
          const int s = q % kStages;
          if (!wait_bar(smem_u32(&full[s]), (q / kStages) & 1, abort_flag)) { ok = false; break; }
          tc_fence_after();
          const uint32_t st = smem_u32(smem + s * Cfg::kStage);
          const uint64_t adesc = umma_smem_desc(st + Cfg::kBTile, 128, 256, 0);
          const uint64_t bdesc = umma_smem_desc(st, 1024, NA * 1024, 2);
          umma_f16(d, adesc, bdesc, idesc, c > c0 ? 1u : 0u);
          umma_commit(smem_u32(&empty[s]));
        }
        if (!ok) break;
        umma_commit(smem_u32(&acc_full[a]));
        ++nacc;
      }
      // every MMA this thread issued is complete before TMEM is released
      umma_commit(smem_u32(done));
      volatile int never = 0;
      if (!wait_bar(smem_u32(done), 0, &never)) *abort_flag = 1;
    }
    __syncwarp();
  } else {
    // ------------------------------------------------------------ epilogue
    const int w = warp;                     // TMEM lanes 32w .. 32w+31
    int nacc = 0;
    for (int i = 0; i < nblk; ++i) {
      const int b = __ldg(pv.blk_order + blockIdx.x + i * gridDim.x);
      const int nc = __ldg(pv.blk_chunk + b + 1) - __ldg(pv.blk_chunk + b);
      const int64_t r = (int64_t)b * kBlkRows + tid;
      const int ro = __ldg(pv.row_out + r);
      const float sc = __ldg(pv.row_scale + r);
      if (nc == 0) {
        if (ro >= 0)
#pragma unroll
          for (int j = 0; j < 2 * NA; ++j) store_zero32<F16OUT>(C, (int64_t)ro * K + 32 * j);
        continue;
      }
      const int a = nacc & 1, ua = nacc >> 1;
      if (!wait_bar(smem_u32(&acc_full[a]), ua & 1, abort_flag)) break;
      tc_fence_after();
#pragma unroll 1
      for (int j = 0; j < 2 * NA; ++j) {
        float v[32];
        tmem_ld_x32(tmem + ((uint32_t)(32 * w) << 16) + (uint32_t)(a * Cfg::kN + 32 * j), v);
        if (ro >= 0) store_row32<F16OUT>(C, (int64_t)ro * K + 32 * j, v, sc);
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(smem_u32(&acc_empty[a]));
      ++nacc;
    }
  }

  __syncthreads();
  if (tid == 0 && *abort_flag) atomicExch(pv.err, kErrMbarTimeout);
  tc_fence_after();
  if (warp == kMmaWarp) tmem_dealloc(tmem, Cfg::kTmemCols);
}

// Any K, FP16 or FP32 features, on CUDA cores: one CTA per block and 64
// features at a time; thread (g, f) owns rows m = g (mod 4) of feature f and
// adds the block's entries in plan order (deterministic, no atomics).
template <typename TB, bool F16OUT>
__global__ void __launch_bounds__(256)
    block_generic_kernel(PlanView pv, const TB* __restrict__ B, int K, void* C) {
  __shared__ float acc[kBlkRows][64];
  __shared__ int cols[kChunkCols];
  const int tid = threadIdx.x, g = tid >> 6, f = tid & 63;
  for (int b = blockIdx.x; b < pv.n_blocks; b += gridDim.x) {
    const int c0 = pv.blk_chunk[b], c1 = pv.blk_chunk[b + 1];
    for (int f0 = 0; f0 < K; f0 += 64) {
      for (int m = g; m < kBlkRows; m += 4) acc[m][f] = 0.f;
      const bool on = f0 + f < K;
      for (int c = c0; c < c1; ++c) {
        __syncthreads();
        if (tid < kChunkCols) cols[tid] = pv.chunk_col[(int64_t)c * kChunkCols + tid];
        __syncthreads();
        for (int e = pv.chunk_ent[c]; e < pv.chunk_ent[c + 1]; ++e) {
          const int pos = pv.ent_pos[e];
          const int m = ((pos >> 8) << 3) | ((pos >> 4) & 7);
          if ((m & 3) != g || !on) continue;
          const int k = (((pos >> 7) & 1) << 3) | ((pos >> 1) & 7);
          const float v = __half2float(__ushort_as_half(pv.ent_val[e]));
          float x;
          if constexpr (sizeof(TB) == 2) x = __half2float(B[(int64_t)cols[k] * K + f0 + f]);
          else x = B[(int64_t)cols[k] * K + f0 + f];
          acc[m][f] = fmaf(v, x, acc[m][f]);
        }
      }
      for (int m = g; m < kBlkRows; m += 4) {
        const int64_t r = (int64_t)b * kBlkRows + m;
        const int ro = pv.row_out[r];
        if (ro < 0 || !on) continue;
        const float out = acc[m][f] * pv.row_scale[r];
        if (F16OUT) reinterpret_cast<__half*>(C)[(int64_t)ro * K + f0 + f] = __float2half_rn(out);
        else reinterpret_cast<float*>(C)[(int64_t)ro * K + f0 + f] = out;
      }
      __syncthreads();
    }
  }
}

template <bool F16OUT, int NA>
int launch_mma_t(const tr_plan* p, const __half* b, void* c, cudaStream_t stream) {
  using Cfg = BlkCfg<NA>;
  if (int rc = kernel_smem_limit((const void*)block_mma_kernel<F16OUT, NA>, Cfg::kSmem)) return rc;
  const int sms = sm_count();
  if (sms <= 0) return fail(TR_ERR_CUDA, "no CUDA device");
  const int grid = std::max(1, std::min(sms, p->view.n_blocks));
  block_mma_kernel<F16OUT, NA><<<grid, kBlkThreads, Cfg::kSmem, stream>>>(p->view, b, c);
  TRS_CUDA(cudaGetLastError());
  return TR_OK;
}

template <typename TB>
int launch_generic_t(const tr_plan* p, const TB* b, int32_t k, void* c, bool f16, cudaStream_t stream) {
  const int grid = std::max(1, std::min(p->view.n_blocks, 148 * 8));
  if (f16) block_generic_kernel<TB, true><<<grid, 256, 0, stream>>>(p->view, b, k, c);
  else block_generic_kernel<TB, false><<<grid, 256, 0, stream>>>(p->view, b, k, c);
  TRS_CUDA(cudaGetLastError());
  return TR_OK;
}

}  // namespace

bool block_mma_supported(int32_t k, const void* b) {
  return k >= 64 && k <= 256 && k % 64 == 0 && (reinterpret_cast<uintptr_t>(b) & 15) == 0;
}

int launch_block(const tr_plan* p, const uint16_t* b, int32_t k, void* c, int c_dtype,
                 bool force_generic, cudaStream_t stream) {
  if (p->view.n_blocks == 0 || k == 0) return TR_OK;
  const bool f16 = c_dtype == TR_OUT_F16;
  const __half* bh = reinterpret_cast<const __half*>(b);
  if (!force_generic && block_mma_supported(k, b) &&
      (reinterpret_cast<uintptr_t>(c) & 15) == 0) {
    switch (k / 64) {
      case 1: return f16 ? launch_mma_t<true, 1>(p, bh, c, stream) : launch_mma_t<false, 1>(p, bh, c, stream);
      case 2: return f16 ? launch_mma_t<true, 2>(p, bh, c, stream) : launch_mma_t<false, 2>(p, bh, c, stream);
      case 3: return f16 ? launch_mma_t<true, 3>(p, bh, c, stream) : launch_mma_t<false, 3>(p, bh, c, stream);
      default: return f16 ? launch_mma_t<true, 4>(p, bh, c, stream) : launch_mma_t<false, 4>(p, bh, c, stream);
    }
  }
  return launch_generic_t(p, bh, k, c, f16, stream);
}

int launch_block_f32(const tr_plan* p, const float* b, int32_t k, void* c, int c_dtype,
                     cudaStream_t stream) {
  if (p->view.n_blocks == 0 || k == 0) return TR_OK;
  return launch_generic_t(p, b, k, c, c_dtype == TR_OUT_F16, stream);
}

}  // namespace trs
