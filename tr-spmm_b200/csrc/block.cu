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
// One persistent CTA per SM takes its blocks from the plan's schedule
// (longest-processing-time assignment made at upload) as one stream of
// chunks.  Every block holds a whole number of groups of four or eight
// chunks (the layout pads it with chunks that have no entries); the stage
// slots of a group share one full and one empty barrier.  Roles:
//
//   producer warps (kProd of them, warps 5.., one stage slot each; chunk q
//   of the stream taken by producer q % kProd)
//       per chunk: wait until the slot is free, clear from its A tile the
//       positions the slot's previous chunk set and write this chunk's
//       values (packed entries value << 16 | tile byte offset, loaded into
//       registers two chunks ahead), issue the 16-byte cp.async copies of
//       the chunk's 16 feature rows straight into the 128-byte-swizzled
//       MN-major operand layout (absent slots zero-filled) and arrive on
//       the group's full barrier: each lane's copies arrive by themselves
//       when they land (cp.async.mbarrier.arrive.noinc), the warp once for
//       the A tile.  A producer never waits for its own copies.  Column
//       lists and entry ranges come from a per-warp ring in shared memory
//       filled eight chunks ahead.  Many producer warps keep enough gathers in
//       flight: a warp's cp.async issue, not the memory system, sets the rate
//       of one warp;
//   MMA warp 4 (one elected thread)
//       per group: wait full, one proxy fence (the operands were written
//       through the generic proxy; the tensor core reads them through the
//       async proxy), one tcgen05.mma per chunk (M = 128, N = K, K = 16) into the
//       block's accumulator, one commit to the group's empty barrier; after
//       a block's last group a commit to the accumulator's full barrier.
//       The loop is straight-line per group (stage descriptors are base +
//       stage * stride): the issuing thread's own instruction latency would
//       otherwise set the MMA rate.  Two TMEM accumulators alternate, so a
//       block's MMAs overlap the previous block's epilogue;
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
#include <type_traits>

#include "block.h"
#include "block_common.cuh"
#include "common.cuh"
#include "plan.h"

namespace trs {
namespace {

using namespace blk;


constexpr int kEpiWarps = 4;
constexpr int kMmaWarp = kEpiWarps;     // warp 4
template <int NA>
struct BlkCfg {
  // chunks per barrier group: the MMA starts once a group's chunks have all
  // landed; groups of four measured faster at K = 192/256 (fewer, larger
  // stages), eight at K = 64/128 (blocks hold whole groups: the layout pads
  // them to multiples of kChunkGroup)
  static constexpr int kGroup = NA >= 3 ? 4 : 8;
  static_assert(kChunkGroup % kGroup == 0, "blocks hold whole groups");
  static constexpr int kN = 64 * NA;               // features = MMA N
  static constexpr int kBTile = 2048 * NA;         // 16 slots x kN features, FP16
  static constexpr int kStage = kBTile + kATile;   // a multiple of 1024
  // as many stage slots as shared memory (and registers) allow; two per
  // producer warp
  static constexpr int kStages = NA <= 2 ? 24 : 16;
  // stage slots per producer warp: one (a warp's gather issue is
  // latency-bound, so more warps gather faster)
  static constexpr int kRing = 1;
  static constexpr int kProd = kStages / kRing;
  static constexpr int kGroups = kStages / kGroup;
  // warps 0-3 epilogue, warp 4 MMA, producers from warp 5
  static constexpr int kThreads = (kEpiWarps + 1 + kProd) * 32;
  static constexpr int kBarOff = kStages * kStage;
  // full[G], empty[G], acc_full[2], acc_empty[2], done; tmem slot, abort flag
  static constexpr int kBlkOff = (kBarOff + (2 * kGroups + 5) * 8 + 16 + 127) / 128 * 128;
  // the ring is read with 16-byte loads: 128-byte aligned
  static constexpr int kMetaOff = (kBlkOff + 3 * kMaxBlk * 4 + 127) / 128 * 128;
  static constexpr int kSmem = 1024 + kMetaOff + kProd * kMetaRing * kMetaStride * 4;
  static constexpr uint32_t kTmemCols = 2 * kN <= 128 ? 128 : (2 * kN <= 256 ? 256 : 512);
  // arrivals that complete a group: 32 lanes and one warp arrival per chunk
  static constexpr uint32_t kFullCount = kGroup * 33;
  static_assert(kStages % kGroup == 0 && kGroups >= 2, "whole groups of stage slots");
  static_assert(kStage % 1024 == 0, "B tiles keep the 1024-byte swizzle alignment");
  static_assert(kSmem <= 227 * 1024, "shared memory budget");
  static_assert(kThreads <= 1024, "one CTA");
  static_assert(kBlkOff % 16 == 0 && kMetaOff % 128 == 0 && (kMetaStride * 4) % 16 == 0,
                "16-byte shared loads of the metadata ring stay aligned");
};

template <bool F16OUT, int NA>
__global__ void __launch_bounds__(BlkCfg<NA>::kThreads, 1)
    block_mma_kernel(PlanView pv, const __half* __restrict__ B, int ldb, void* C, int ldc) {
  using Cfg = BlkCfg<NA>;
  constexpr int S = Cfg::kStages, NG = Cfg::kGroups, P = Cfg::kProd, kGroup = Cfg::kGroup;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + Cfg::kBarOff);
  uint64_t* full = bars;
  uint64_t* empty = bars + NG;
  uint64_t* acc_full = bars + 2 * NG;
  uint64_t* acc_empty = acc_full + 2;
  uint64_t* done = acc_empty + 2;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);
  int* s_b = reinterpret_cast<int*>(smem + Cfg::kBlkOff);
  int* s_c0 = s_b + kMaxBlk;
  int* s_c1 = s_c0 + kMaxBlk;

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int bfirst = __ldg(pv.cta_ptr + blockIdx.x);
  const int nblk = __ldg(pv.cta_ptr + blockIdx.x + 1) - bfirst;

  if (warp == kMmaWarp) {
    tmem_alloc(smem_u32(tmem_slot), Cfg::kTmemCols);
    tmem_relinquish();
  }
  if (tid == 0) {
    for (int g = 0; g < NG; ++g) {
      mbar_init(smem_u32(&full[g]), Cfg::kFullCount);
      mbar_init(smem_u32(&empty[g]), 1);
    }
    for (int a = 0; a < 2; ++a) {
      mbar_init(smem_u32(&acc_full[a]), 1);
      mbar_init(smem_u32(&acc_empty[a]), kEpiWarps);
    }
    mbar_init(smem_u32(done), 1);
    *abort_flag = 0;
    fence_mbar_init();
  }
  // this CTA's blocks, staged once
  for (int i = tid; i < nblk; i += Cfg::kThreads) {
    const int b = __ldg(pv.cta_blk + bfirst + i);
    s_b[i] = b;
    s_c0[i] = __ldg(pv.blk_chunk + b);
    s_c1[i] = __ldg(pv.blk_chunk + b + 1);
  }
  // A tiles start as zeros (a chunk writes its entries, and clears them
  // again before the slot takes the next chunk); B tiles start as zeros so
  // that no stale bit pattern meets a zero of A as Inf or NaN
  for (int i = tid; i < S * Cfg::kStage / 16; i += Cfg::kThreads)
    reinterpret_cast<uint4*>(smem)[i] = make_uint4(0, 0, 0, 0);
  fence_proxy_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  const int prod = warp > kMmaWarp ? warp - kMmaWarp - 1 : -1;
  if (prod >= 0 && prod < P) {
    // ------------------------------------------------------------ producers
    const int p = prod;
    const uint64_t pol_keep = l2_policy_evict_last(), pol_stream = l2_policy_evict_first();
    int total = 0;
    for (int i = lane; i < nblk; i += 32) total += s_c1[i] - s_c0[i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) total += __shfl_xor_sync(0xffffffffu, total, o);
    const int nloc = total > p ? (total - p + P - 1) / P : 0;
    StreamCursor cur{s_c0, s_c1, nblk};
    // columns and entry range of this warp's chunk m in ring slot m % kMetaRing
    const uint32_t ring = smem_u32(smem + Cfg::kMetaOff) + p * kMetaRing * kMetaStride * 4;
    auto copy_meta = [&](int m) {
      if (m >= nloc) return;
      const int c = cur.chunk(P * m + p);
      const uint32_t dst = ring + (m % kMetaRing) * kMetaStride * 4 + lane * 4;
      if (lane < kChunkCols)        // row k at ring position col_pos(k)
        cp_async4(dst - lane * 4 + col_pos<NA>(lane) * 4, pv.chunk_col + (int64_t)c * kChunkCols + lane);
      else if (lane < kMetaInts) cp_async4(dst, pv.chunk_ent + c + (lane - kChunkCols));
    };
    // the first kEntReg * 32 entry words of chunk m (its range has landed)
    auto load_ents = [&](int m, uint32_t (&w)[kEntReg]) {
      const uint32_t slot = ring + (m % kMetaRing) * kMetaStride * 4;
      const int e0 = m < nloc ? (int)lds_u32(slot + 64) : 0;
      const int e1 = m < nloc ? (int)lds_u32(slot + 68) : 0;
#pragma unroll
      for (int r = 0; r < kEntReg; ++r) {
        const int e = e0 + lane + 32 * r;
        w[r] = e < e1 ? ld_stream_u32(pv.ent_pv + e, pol_stream) : kNoEntry;
      }
    };
    for (int m = 0; m < kMetaRing; ++m) copy_meta(m);
    cp_async_wait_all();
    __syncwarp();
    // entry words of the chunk each register set serves next (chunks n and
    // n + 1 at the top of the loop), and of the chunk it served before
    // entry words: two register sets alternate (chunk n in set n % 2, loaded
    // two chunks ahead); the entries each of this warp's stage slots holds
    // (slot n % kRing) are cleared before the slot's next chunk
    constexpr int R = Cfg::kRing;
    uint32_t ent[2][kEntReg], old[R][kEntReg];
    int oldcnt[R] = {};
    load_ents(0, ent[0]);
    load_ents(1, ent[1]);
#pragma unroll
    for (int r = 0; r < kEntReg; ++r)
#pragma unroll
      for (int o = 0; o < R; ++o) old[o][r] = kNoEntry;

    // chunk n with register set SET (= n % 2, a compile-time index)
    auto body = [&](auto set_tag, int n) -> bool {
      constexpr int SET = decltype(set_tag)::value;
      cp_async_wait_group<kMetaWait>();    // metadata of chunk n + 2 (and earlier) has landed
      __syncwarp();
      const uint32_t mslot = ring + (n % kMetaRing) * kMetaStride * 4;
      // the columns of the rows this lane copies (see col_pos)
      int cols[RowsPerLane<NA>::value];
      if constexpr (NA == 3) {
        const int my_col = lane < kChunkCols ? (int)lds_u32(mslot + lane * 4) : -1;
#pragma unroll
        for (int t = 0; t < 4 * NA; ++t) cols[t] = __shfl_sync(0xffffffffu, my_col, (lane + 32 * t) / 24);
      } else {
        constexpr int R = RowsPerLane<NA>::value;   // rows per lane
        const uint32_t at = mslot + (lane / (8 * NA)) * R * 4;
#pragma unroll
        for (int t = 0; t < R; t += 4) {
          const uint4 v = lds_u128(at + t * 4);
          cols[t] = (int)v.x; cols[t + 1] = (int)v.y; cols[t + 2] = (int)v.z; cols[t + 3] = (int)v.w;
        }
      }
      const int e0 = (int)lds_u32(mslot + 64), e1 = (int)lds_u32(mslot + 68);
      const int q = P * n + p, s = q % S, gs = s / kGroup;
      if (!wait_bar(smem_u32(&empty[gs]), ((q / S) & 1) ^ 1, abort_flag)) return false;
      uint8_t* st = smem + s * Cfg::kStage;
      const uint32_t b_tile = smem_u32(st), a_tile = b_tile + Cfg::kBTile;
      // the slot's previous chunk leaves the A tile
      constexpr int OS = R == 1 ? 0 : SET;      // this chunk's stage slot among the warp's
      if (oldcnt[OS] > kEntReg * 32) {
        uint4* at = reinterpret_cast<uint4*>(st + Cfg::kBTile);
        for (int i = lane; i < kATile / 16; i += 32) at[i] = make_uint4(0, 0, 0, 0);
      } else {
#pragma unroll
        for (int r = 0; r < kEntReg; ++r)
          if ((old[OS][r] & 0xFFFFu) < (uint32_t)kATile) sts_u16(a_tile + (old[OS][r] & 0xFFFFu), 0);
      }
      __syncwarp();
      // this chunk's values
#pragma unroll
      for (int r = 0; r < kEntReg; ++r) {
        const uint32_t w = ent[SET][r];
        if ((w & 0xFFFFu) < (uint32_t)kATile) sts_u16(a_tile + (w & 0xFFFFu), (uint16_t)(w >> 16));
        old[OS][r] = w;
      }
      for (int e = e0 + kEntReg * 32 + lane; e < e1; e += 32) {
        const uint32_t w = __ldg(pv.ent_pv + e);
        sts_u16(a_tile + (w & 0xFFFFu), (uint16_t)(w >> 16));
      }
      oldcnt[OS] = e1 - e0;
      // gather: 16 rows x (8 * NA) 16-byte segments, 4 * NA per lane
#pragma unroll
      for (int t = 0; t < 4 * NA; ++t) {
        const int idx = lane + 32 * t;
        const int k = idx / (8 * NA), g = idx % (8 * NA);
        const int col = cols[t];
        const uint32_t dst = b_tile + (k >> 3) * (NA * 1024) + (g >> 3) * 1024 + (k & 7) * 128 +
                             (((g & 7) ^ (k & 7)) << 4);
        const __half* src = B + (int64_t)(col >= 0 ? col : 0) * ldb + g * 8;
        cp_async16_hint(dst, src, col >= 0 ? 16 : 0, pol_keep);
      }
      cp_async_arrive_noinc(smem_u32(&full[gs]));
      __syncwarp();
      if (lane == 0) mbar_arrive(smem_u32(&full[gs]));
      // the same register set serves chunk n + 2; the ring slot takes chunk
      // n + kMetaRing
      load_ents(n + 2, ent[SET]);
      __syncwarp();
      copy_meta(n + kMetaRing);
      cp_async_commit();
      return true;
    };
    bool ok = true;
    int n = 0;
    for (; n + 1 < nloc && ok; n += 2) {
      ok = body(std::integral_constant<int, 0>{}, n);
      if (ok) ok = body(std::integral_constant<int, 1>{}, n + 1);
    }
    if (ok && n < nloc) body(std::integral_constant<int, 0>{}, n);
    cp_async_wait_all();
  } else if (warp == kMmaWarp) {
    // ------------------------------------------------------------ MMA issuer
    if (lane == 0) {
      constexpr uint32_t idesc = umma_idesc_f16(128, Cfg::kN, /*a MN-major*/ false, /*b MN-major*/ true);
      // stage s's descriptors: the start-address field (address >> 4) grows by
      // kStage >> 4 per stage
      const uint32_t base = smem_u32(smem);
      const uint64_t adesc0 = umma_smem_desc(base + Cfg::kBTile, 128, 256, 0);
      const uint64_t bdesc0 = umma_smem_desc(base, 1024, NA * 1024, 2);
      constexpr uint64_t kStep = Cfg::kStage >> 4;
      // stage group slot gs (phase ph of its barriers) of the current group
      int gs = 0, ph = 0, nacc = 0;
      bool ok = true;
      for (int i = 0; i < nblk && ok; ++i) {
        const int ngb = (s_c1[i] - s_c0[i]) / kGroup;       // every block: whole groups
        if (ngb == 0) continue;
        const int a = nacc & 1;
        if (!wait_bar(smem_u32(&acc_empty[a]), ((nacc >> 1) & 1) ^ 1, abort_flag)) { ok = false; break; }
        tc_fence_after();
        const uint32_t d = tmem + (uint32_t)(a * Cfg::kN);
        for (int t = 0; t < ngb; ++t) {
          if (!wait_bar(smem_u32(&full[gs]), ph, abort_flag)) { ok = false; break; }
          fence_proxy_async_smem();
          tc_fence_after();
          const uint64_t off = (uint64_t)(gs * kGroup) * kStep;
          umma_f16(d, adesc0 + off, bdesc0 + off, idesc, t > 0 ? 1u : 0u);
#pragma unroll
          for (int j = 1; j < kGroup; ++j)
            umma_f16(d, adesc0 + off + j * kStep, bdesc0 + off + j * kStep, idesc, 1u);
          umma_commit(smem_u32(&empty[gs]));
          if (++gs == NG) {
            gs = 0;
            ph ^= 1;
          }
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
  } else if (warp < kEpiWarps) {
    // ------------------------------------------------------------ epilogue
    const int w = warp;                     // TMEM lanes 32w .. 32w+31
    int nacc = 0;
    for (int i = 0; i < nblk; ++i) {
      const int b = s_b[i];
      const int nc = s_c1[i] - s_c0[i];
      const int64_t r = (int64_t)b * kBlkRows + tid;
      const int ro = __ldg(pv.row_out + r);
      const float sc = __ldg(pv.row_scale + r);
      if (nc == 0) {
        if (ro >= 0)
#pragma unroll
          for (int j = 0; j < 2 * NA; ++j) store_zero32<F16OUT>(C, (int64_t)ro * ldc + 32 * j);
        continue;
      }
      const int a = nacc & 1, ua = nacc >> 1;
      if (!wait_bar(smem_u32(&acc_full[a]), ua & 1, abort_flag)) break;
      tc_fence_after();
#pragma unroll 1
      for (int j = 0; j < 2 * NA; ++j) {
        float v[32];
        tmem_ld_x32(tmem + ((uint32_t)(32 * w) << 16) + (uint32_t)(a * Cfg::kN + 32 * j), v);
        if (ro >= 0) store_row32<F16OUT>(C, (int64_t)ro * ldc + 32 * j, v, sc);
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
          const uint32_t w = pv.ent_pv[e];
          const int pos = (int)(w & 0xFFFFu);
          const int m = ((pos >> 8) << 3) | ((pos >> 4) & 7);
          if ((m & 3) != g || !on) continue;
          const int k = (((pos >> 7) & 1) << 3) | ((pos >> 1) & 7);
          const float v = __half2float(__ushort_as_half((uint16_t)(w >> 16)));
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

// One feature tile: B and C already offset to the tile's first feature,
// rows ldb / ldc elements apart.
template <bool F16OUT, int NA>
int launch_mma_t(const tr_plan* p, const __half* b, int ldb, void* c, int ldc, cudaStream_t stream) {
  using Cfg = BlkCfg<NA>;
  if (int rc = kernel_smem_limit((const void*)block_mma_kernel<F16OUT, NA>, Cfg::kSmem)) return rc;
  block_mma_kernel<F16OUT, NA><<<std::max(1, p->view.n_sched), Cfg::kThreads, Cfg::kSmem, stream>>>(
      p->view, b, ldb, c, ldc);
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
  return k >= 64 && k % 64 == 0 && (reinterpret_cast<uintptr_t>(b) & 15) == 0;
}

int block_k_tile(const tr_plan* p, int32_t k) {
  const int t = p->k_tile > 0 ? p->k_tile : 256;
  return std::min<int32_t>(t, k);
}

int launch_block(const tr_plan* p, const uint16_t* b, int32_t k, void* c, int c_dtype,
                 bool force_generic, cudaStream_t stream) {
  if (p->view.n_blocks == 0 || k == 0) return TR_OK;
  const bool f16 = c_dtype == TR_OUT_F16;
  const __half* bh = reinterpret_cast<const __half*>(b);
  // every CTA's block list fits the staged list
  bool fits = p->max_sched_blocks <= kMaxBlk;
  if (!force_generic && fits && block_mma_supported(k, b) &&
      (reinterpret_cast<uintptr_t>(c) & 15) == 0) {
    // feature tiles of k_tile (a multiple of 64, at most 256: the MMA's N),
    // one launch each; every tile gathers its slice of the same B rows
    const int kt = block_k_tile(p, k);
    for (int f0 = 0; f0 < k; f0 += kt) {
      const int w = std::min(kt, k - f0);
      const __half* bt = bh + f0;
      void* ct = static_cast<char*>(c) + (size_t)f0 * (f16 ? 2 : 4);
      int rc;
      switch (w / 64) {
        case 1: rc = f16 ? launch_mma_t<true, 1>(p, bt, k, ct, k, stream) : launch_mma_t<false, 1>(p, bt, k, ct, k, stream); break;
        case 2: rc = f16 ? launch_mma_t<true, 2>(p, bt, k, ct, k, stream) : launch_mma_t<false, 2>(p, bt, k, ct, k, stream); break;
        case 3: rc = f16 ? launch_mma_t<true, 3>(p, bt, k, ct, k, stream) : launch_mma_t<false, 3>(p, bt, k, ct, k, stream); break;
        default: rc = f16 ? launch_mma_t<true, 4>(p, bt, k, ct, k, stream) : launch_mma_t<false, 4>(p, bt, k, ct, k, stream); break;
      }
      if (rc) return rc;
    }
    return TR_OK;
  }
  return launch_generic_t(p, bh, k, c, f16, stream);
}

int launch_block_f32(const tr_plan* p, const float* b, int32_t k, void* c, int c_dtype,
                     cudaStream_t stream) {
  if (p->view.n_blocks == 0 || k == 0) return TR_OK;
  return launch_generic_t(p, b, k, c, c_dtype == TR_OUT_F16, stream);
}

}  // namespace trs
