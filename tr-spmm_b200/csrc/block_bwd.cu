// Block engine backward for sm_100a: dB = A^T . dC and dval = SDDMM(dC, B)
// in one pass over a block plan of A^T, both products on the tensor cores.
//
// The plan's blocks are 128 rows of A^T (columns c of A, rows of B and dB);
// a chunk's 16 slots are distinct rows r of A, whose dC rows the producers
// gather once per block.  Per group of four chunks the tensor core computes
//     D1[128 c, K]      += A_chunk[128 c, 16 r] . dC_g[16 r, K]      (dB)
//     D2[128 c, 64 r']   = B_blk[128 c, K] . dC_4g[64 r', K]^T        (dval)
// D2 holds <B[c], dC[r]> for every (c, r) pair of the group; the entries of
// the four chunks are read out of it (dval[e] = D2[c(e), r(e)]).  The
// gathered dC tile serves both: as the MN-major B operand of D1 (features
// contiguous) and, four stages at once, as the K-major B operand of D2 (the
// same bytes: a 128-byte-swizzled atom of 8 rows x 64 features reads either
// way).  B_blk, the block's 128 rows of B, is the A operand of D2 and lives
// in tensor memory (two buffers, one per block in flight), so the dval MMAs
// read only the 2 KB of the group's dC rows per K step from shared memory.
//
// Roles (one persistent CTA per SM, blocks from the plan's schedule):
//   producers (warps 5-7, 12..): as in the forward kernel — entries into
//     the stage's A tile, the chunk's 16 dC rows gathered by cp.async into
//     the stage's B tile; the B tiles of all stages are contiguous, so four
//     consecutive stages form the 64-row operand of D2;
//   MMA warp 4 (one thread): per group four D1 MMAs (N = K) and K/16 D2
//     MMAs (N = 64, A from tensor memory), one commit releasing the four
//     stages, one marking the group's D2 tile full; per block a commit to
//     the dB accumulator;
//   dB warps 0-3 (thread t <-> block row t <-> TMEM lane t): load the rows
//     of B of the blocks two ahead into tensor memory (tcgen05.st), drain
//     the dB accumulator (row scale, one store per row, deterministic);
//   dval warps 8-11: copy each group's D2 tile to shared memory and write
//     every entry's value at its position (sequential when the plan's edges
//     are numbered in its entry order, else through ent_src).
//
// Every wait is bounded (about a second of %globaltimer); on a timeout every
// role leaves, TMEM is freed and the plan's error word is set.
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

constexpr int kBG = 4;                  // chunks per barrier group (D2: N = 16 * kBG)
constexpr int kD2N = 16 * kBG;
constexpr int kEpiWarps = 4;            // warps 0-3: dB
constexpr int kMmaWarp = 4;
constexpr int kValWarp0 = 8;            // warps 8-11: dval
constexpr int kStgStride = 68;          // floats per staged D2 row (conflict-free 16-byte stores)
constexpr int kValBarrier = 1;          // named barrier of the dval warps

template <int NA>
struct BwdCfg {
  static constexpr int kN = 64 * NA;               // features
  static constexpr int kBTile = 2048 * NA;         // 16 slots x kN features, FP16
  static constexpr int kStages = NA == 1 ? 24 : 20;
  // stage slots per producer warp: two (with one, the 64-register cap of
  // 29 warps spills the dval and dB paths: 1.0 ms against 0.51 ms)
  static constexpr int kRing = 2;
  static constexpr int kProd = kStages / kRing;
  static constexpr int kGroups = kStages / kBG;
  // warps 0-3 dB, 4 MMA, 5-7 producers, 8-11 dval, 12.. producers
  static constexpr int kWarps = 12 + (kProd - 3);
  static constexpr int kThreads = kWarps * 32;
  static constexpr int kAOff = kStages * kBTile;
  static constexpr int kStgOff = kAOff + kStages * kATile;
  static constexpr int kBarOff = kStgOff + kBlkRows * kStgStride * 4;
  // full[G], empty[G], acc_full[2], acc_empty[2], d2_full[2], d2_empty[2],
  // bb_full[2], done; then tmem slot, abort flag, go word
  static constexpr int kNumBars = 2 * kGroups + 11;
  static constexpr int kBlkOff = (kBarOff + kNumBars * 8 + 16 + 127) / 128 * 128;
  static constexpr int kMetaOff = (kBlkOff + 3 * kMaxBlk * 4 + 127) / 128 * 128;
  static constexpr int kSmem = 1024 + kMetaOff + kProd * kMetaRing * kMetaStride * 4;
  // TMEM: dB accumulators [0, 2N), B rows [2N, 3N) (two buffers of N/2
  // columns, FP16 pairs), D2 tiles [3N, 3N + 2 * 64)
  static constexpr uint32_t kBbCol = 2 * kN;
  static constexpr uint32_t kD2Col = 3 * kN;
  static constexpr uint32_t kTmemCols = 512;
  static constexpr uint32_t kFullCount = kBG * 33;
  static_assert(NA == 1 || NA == 2, "K = 64 or 128");
  static_assert(kStages % kBG == 0 && kGroups >= 2, "whole groups of stage slots");
  static_assert(kBTile % 1024 == 0 && kAOff % 1024 == 0, "B tiles keep the 1024-byte swizzle alignment");
  static_assert(kStgOff % 16 == 0 && kBarOff % 8 == 0, "aligned staging and barriers");
  static_assert(kBlkOff % 16 == 0 && kMetaOff % 128 == 0 && (kMetaStride * 4) % 16 == 0,
                "16-byte shared loads of the metadata ring stay aligned");
  static_assert(kSmem <= 227 * 1024, "shared memory budget");
  static_assert(kThreads <= 1024, "one CTA");
  static_assert(kD2Col + 2 * kD2N <= kTmemCols, "tensor memory budget");
};

// 32 lanes x 16 consecutive 32-bit TMEM columns from registers.
__device__ __forceinline__ void tmem_st_x16(uint32_t taddr, const uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,"
      "%14,%15,%16};\n" ::"r"(taddr),
      "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]),
      "r"(r[8]), "r"(r[9]), "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]), "r"(r[14]), "r"(r[15])
      : "memory");
}
__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;\n" ::: "memory"); }

// D[tmem] (+)= A[tmem] * B[smem desc], kind::f16: A's 128 rows in TMEM lanes,
// two FP16 values per 32-bit column.
__device__ __forceinline__ void umma_f16_ts(uint32_t d_tmem, uint32_t a_tmem, uint64_t b_desc,
                                            uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, p;\n}\n" ::"r"(d_tmem),
      "r"(a_tmem), "l"(b_desc), "r"(idesc), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void named_bar_sync(int id, int count) {
  asm volatile("bar.sync %0, %1;\n" ::"r"(id), "r"(count) : "memory");
}

template <bool F16OUT, int NA>
__global__ void __launch_bounds__(BwdCfg<NA>::kThreads, 1)
    block_bwd_kernel(PlanView pv, const __half* __restrict__ G, const __half* __restrict__ Bm,
                     void* DB, float* __restrict__ dval, const int32_t* __restrict__ dval_at) {
  using Cfg = BwdCfg<NA>;
  constexpr int K = Cfg::kN, S = Cfg::kStages, NG = Cfg::kGroups, P = Cfg::kProd;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + Cfg::kBarOff);
  uint64_t* full = bars;
  uint64_t* empty = bars + NG;
  uint64_t* acc_full = bars + 2 * NG;
  uint64_t* acc_empty = acc_full + 2;
  uint64_t* d2_full = acc_empty + 2;
  uint64_t* d2_empty = d2_full + 2;
  uint64_t* bb_full = d2_empty + 2;
  uint64_t* done = bb_full + 2;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);
  volatile int* go = reinterpret_cast<volatile int*>(tmem_slot + 2);
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
      mbar_init(smem_u32(&d2_full[a]), 1);
      mbar_init(smem_u32(&d2_empty[a]), 1);
      mbar_init(smem_u32(&bb_full[a]), kEpiWarps);
    }
    mbar_init(smem_u32(done), 1);
    *abort_flag = 0;
    *go = 0;
    fence_mbar_init();
  }
  for (int i = tid; i < nblk; i += Cfg::kThreads) {
    const int b = __ldg(pv.cta_blk + bfirst + i);
    s_b[i] = b;
    s_c0[i] = __ldg(pv.blk_chunk + b);
    s_c1[i] = __ldg(pv.blk_chunk + b + 1);
  }
  // B and A tiles start as zeros (see the forward kernel)
  for (int i = tid; i < Cfg::kStgOff / 16; i += Cfg::kThreads)
    reinterpret_cast<uint4*>(smem)[i] = make_uint4(0, 0, 0, 0);
  fence_proxy_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  const int prod = (warp >= 5 && warp <= 7) ? warp - 5 : (warp >= 12 ? warp - 9 : -1);
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
    const uint32_t ring = smem_u32(smem + Cfg::kMetaOff) + p * kMetaRing * kMetaStride * 4;
    auto copy_meta = [&](int m) {
      if (m >= nloc) return;
      const int c = cur.chunk(P * m + p);
      const uint32_t dst = ring + (m % kMetaRing) * kMetaStride * 4 + lane * 4;
      if (lane < kChunkCols)
        cp_async4(dst - lane * 4 + col_pos<NA>(lane) * 4, pv.chunk_col + (int64_t)c * kChunkCols + lane);
      else if (lane < kMetaInts) cp_async4(dst, pv.chunk_ent + c + (lane - kChunkCols));
    };
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
    constexpr int R = Cfg::kRing;
    uint32_t ent[2][kEntReg], old[R][kEntReg];
    int oldcnt[R] = {};
    load_ents(0, ent[0]);
    load_ents(1, ent[1]);
#pragma unroll
    for (int r = 0; r < kEntReg; ++r)
#pragma unroll
      for (int o = 0; o < R; ++o) old[o][r] = kNoEntry;

    auto body = [&](auto set_tag, int n) -> bool {
      constexpr int SET = decltype(set_tag)::value;
      cp_async_wait_group<kMetaWait>();
      __syncwarp();
      const uint32_t mslot = ring + (n % kMetaRing) * kMetaStride * 4;
      int cols[RowsPerLane<NA>::value];
      {
        constexpr int R = RowsPerLane<NA>::value;
        const uint32_t at = mslot + (lane / (8 * NA)) * R * 4;
#pragma unroll
        for (int t = 0; t < R; t += 4) {
          const uint4 v = lds_u128(at + t * 4);
          cols[t] = (int)v.x; cols[t + 1] = (int)v.y; cols[t + 2] = (int)v.z; cols[t + 3] = (int)v.w;
        }
      }
      const int e0 = (int)lds_u32(mslot + 64), e1 = (int)lds_u32(mslot + 68);
      const int q = P * n + p, s = q % S, gs = s / kBG;
      if (!wait_bar(smem_u32(&empty[gs]), ((q / S) & 1) ^ 1, abort_flag)) return false;
      uint8_t* st_a = smem + Cfg::kAOff + s * kATile;
      const uint32_t b_tile = smem_u32(smem + s * Cfg::kBTile), a_tile = smem_u32(st_a);
      constexpr int OS = R == 1 ? 0 : SET;      // this chunk's stage slot among the warp's
      if (oldcnt[OS] > kEntReg * 32) {
        uint4* at = reinterpret_cast<uint4*>(st_a);
        for (int i = lane; i < kATile / 16; i += 32) at[i] = make_uint4(0, 0, 0, 0);
      } else {
#pragma unroll
        for (int r = 0; r < kEntReg; ++r)
          if ((old[OS][r] & 0xFFFFu) < (uint32_t)kATile) sts_u16(a_tile + (old[OS][r] & 0xFFFFu), 0);
      }
      __syncwarp();
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
#pragma unroll
      for (int t = 0; t < 4 * NA; ++t) {
        const int idx = lane + 32 * t;
        const int k = idx / (8 * NA), g = idx % (8 * NA);
        const int col = cols[t];
        const uint32_t dst = b_tile + (k >> 3) * (NA * 1024) + (g >> 3) * 1024 + (k & 7) * 128 +
                             (((g & 7) ^ (k & 7)) << 4);
        const __half* src = G + (int64_t)(col >= 0 ? col : 0) * K + g * 8;
        cp_async16_hint(dst, src, col >= 0 ? 16 : 0, pol_keep);
      }
      cp_async_arrive_noinc(smem_u32(&full[gs]));
      __syncwarp();
      if (lane == 0) mbar_arrive(smem_u32(&full[gs]));
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
      constexpr uint32_t idesc1 = umma_idesc_f16(128, K, /*a MN-major*/ false, /*b MN-major*/ true);
      constexpr uint32_t idesc2 = umma_idesc_f16(128, kD2N, false, false);
      const uint32_t base = smem_u32(smem);
      const uint64_t adesc0 = umma_smem_desc(base + Cfg::kAOff, 128, 256, 0);
      const uint64_t bdesc1 = umma_smem_desc(base, 1024, NA * 1024, 2);
      // the same tiles as a K-major operand: 8-row groups NA * 1024 bytes apart
      // (within a stage and across consecutive stages); a K step of 16
      // features is 32 bytes inside the 128-byte atom, four steps an atom
      const uint64_t bdesc2 = umma_smem_desc(base, 16, NA * 1024, 2);
      constexpr uint64_t kAStep = kATile >> 4, kBStep = Cfg::kBTile >> 4;
      int gs = 0, ph = 0, nacc = 0, dn = 0;
      bool ok = true;
      for (int i = 0; i < nblk && ok; ++i) {
        const int ngb = (s_c1[i] - s_c0[i]) / kBG;
        if (ngb == 0) continue;
        const int a = nacc & 1;
        if (!wait_bar(smem_u32(&acc_empty[a]), ((nacc >> 1) & 1) ^ 1, abort_flag)) { ok = false; break; }
        if (!wait_bar(smem_u32(&bb_full[a]), (nacc >> 1) & 1, abort_flag)) { ok = false; break; }
        tc_fence_after();
        const uint32_t d1 = tmem + (uint32_t)(a * K);
        const uint32_t bb = tmem + Cfg::kBbCol + (uint32_t)(a * (K / 2));
        for (int t = 0; t < ngb; ++t) {
          if (!wait_bar(smem_u32(&full[gs]), ph, abort_flag)) { ok = false; break; }
          fence_proxy_async_smem();
          tc_fence_after();
          const uint64_t s0 = (uint64_t)(gs * kBG);
#pragma unroll
          for (int j = 0; j < kBG; ++j)
            umma_f16(d1, adesc0 + (s0 + j) * kAStep, bdesc1 + (s0 + j) * kBStep, idesc1,
                     (t > 0 || j > 0) ? 1u : 0u);
          const int ds = dn & 1;
          if (!wait_bar(smem_u32(&d2_empty[ds]), ((dn >> 1) & 1) ^ 1, abort_flag)) { ok = false; break; }
          tc_fence_after();
          const uint32_t d2 = tmem + Cfg::kD2Col + (uint32_t)(ds * kD2N);
          const uint64_t b2 = bdesc2 + s0 * kBStep;
#pragma unroll
          for (int kk = 0; kk < K / 16; ++kk)
            umma_f16_ts(d2, bb + (uint32_t)(kk * 8), b2 + (uint64_t)((kk >> 2) * (1024 >> 4) + (kk & 3) * 2),
                        idesc2, kk > 0 ? 1u : 0u);
          umma_commit(smem_u32(&empty[gs]));
          umma_commit(smem_u32(&d2_full[ds]));
          ++dn;
          if (++gs == NG) {
            gs = 0;
            ph ^= 1;
          }
        }
        if (!ok) break;
        umma_commit(smem_u32(&acc_full[a]));
        ++nacc;
      }
      umma_commit(smem_u32(done));
      volatile int never = 0;
      if (!wait_bar(smem_u32(done), 0, &never)) *abort_flag = 1;
    }
    __syncwarp();
  } else if (warp < kEpiWarps) {
    // ------------------------------------------------------------ dB
    const int w = warp;                     // TMEM lanes 32w .. 32w+31
    const uint32_t lane_base = tmem + ((uint32_t)(32 * w) << 16);
    // block list position i's rows of B into buffer buf (row t of the block:
    // its A^T row's output position = the row of B)
    auto load_rows = [&](int i, int buf) {
      const int64_t r = (int64_t)s_b[i] * kBlkRows + tid;
      const int c = __ldg(pv.row_out + r);
      const uint4* src = reinterpret_cast<const uint4*>(Bm + (int64_t)(c >= 0 ? c : 0) * K);
#pragma unroll
      for (int j = 0; j < K / 32; ++j) {           // 32 features = 16 columns
        uint32_t v[16];
#pragma unroll
        for (int h = 0; h < 4; ++h) {
          const uint4 x = c >= 0 ? __ldg(src + 4 * j + h) : make_uint4(0u, 0u, 0u, 0u);
          v[4 * h] = x.x; v[4 * h + 1] = x.y; v[4 * h + 2] = x.z; v[4 * h + 3] = x.w;
        }
        tmem_st_x16(lane_base + Cfg::kBbCol + (uint32_t)(buf * (K / 2) + 16 * j), v);
      }
      tmem_wait_st();
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(smem_u32(&bb_full[buf]));
    };
    auto next_busy = [&](int from) {
      while (from < nblk && s_c1[from] == s_c0[from]) ++from;
      return from;
    };
    int pending = next_busy(0);
    for (int buf = 0; buf < 2 && pending < nblk; ++buf) {
      load_rows(pending, buf);
      pending = next_busy(pending + 1);
    }
    int nacc = 0;
    for (int i = 0; i < nblk; ++i) {
      const int64_t r = (int64_t)s_b[i] * kBlkRows + tid;
      const int ro = __ldg(pv.row_out + r);
      const float sc = __ldg(pv.row_scale + r);
      if (s_c1[i] == s_c0[i]) {
        if (ro >= 0)
#pragma unroll
          for (int j = 0; j < 2 * NA; ++j) store_zero32<F16OUT>(DB, (int64_t)ro * K + 32 * j);
        continue;
      }
      const int a = nacc & 1;
      if (!wait_bar(smem_u32(&acc_full[a]), (nacc >> 1) & 1, abort_flag)) break;
      tc_fence_after();
#pragma unroll 1
      for (int j = 0; j < 2 * NA; ++j) {
        float v[32];
        tmem_ld_x32(lane_base + (uint32_t)(a * K + 32 * j), v);
        if (ro >= 0) store_row32<F16OUT>(DB, (int64_t)ro * K + 32 * j, v, sc);
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(smem_u32(&acc_empty[a]));
      // every MMA of this block is complete: its B-row buffer takes the
      // block two ahead
      if (pending < nblk) {
        load_rows(pending, a);
        pending = next_busy(pending + 1);
      }
      ++nacc;
    }
  } else if (warp >= kValWarp0 && warp < kValWarp0 + 4) {
    // ------------------------------------------------------------ dval
    const int td = tid - kValWarp0 * 32;    // D2 row (TMEM lane)
    const uint32_t lane_base = tmem + ((uint32_t)(32 * (warp - kValWarp0)) << 16);
    float* stg = reinterpret_cast<float*>(smem + Cfg::kStgOff);
    // the groups of this CTA's chunk stream, in order: first chunk of the
    // next group (-1 at the end)
    int gi = 0, gt = 0;
    auto next_group = [&]() -> int {
      while (gi < nblk && gt >= (s_c1[gi] - s_c0[gi]) / kBG) {
        ++gi;
        gt = 0;
      }
      if (gi >= nblk) return -1;
      return s_c0[gi] + kBG * gt++;
    };
    // a group's chunk bounds and this thread's first two entry words, loaded
    // one group ahead so that their latency hides behind the current group
    int nb[kBG + 1];
    uint32_t nw[2];
    auto prefetch = [&](int cb) {
#pragma unroll
      for (int j = 0; j <= kBG; ++j) nb[j] = cb >= 0 ? __ldg(pv.chunk_ent + cb + j) : 0;
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int e = nb[0] + td + 128 * h;
        nw[h] = e < nb[kBG] ? __ldg(pv.ent_pv + e) : kNoEntry;
      }
    };
    int cb = next_group();
    prefetch(cb);
    int dn = 0;
    while (cb >= 0) {
      int bnd[kBG + 1];
#pragma unroll
      for (int j = 0; j <= kBG; ++j) bnd[j] = nb[j];
      const uint32_t w0 = nw[0], w1 = nw[1];
      const int cb_next = next_group();
      prefetch(cb_next);
      const int e0 = bnd[0], e1 = bnd[kBG];
      const int ds = dn & 1;
      if (td == 0) *go = wait_bar(smem_u32(&d2_full[ds]), (dn >> 1) & 1, abort_flag) ? 1 : 0;
      named_bar_sync(kValBarrier, 128);
      if (!*go) break;                        // read after the barrier: the same for all 128
      tc_fence_after();
#pragma unroll
      for (int h = 0; h < kD2N / 32; ++h) {
        float v[32];
        tmem_ld_x32(lane_base + Cfg::kD2Col + (uint32_t)(ds * kD2N + 32 * h), v);
        float4* row = reinterpret_cast<float4*>(stg + td * kStgStride + 32 * h);
#pragma unroll
        for (int q = 0; q < 8; ++q) row[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
      }
      tc_fence_before();
      named_bar_sync(kValBarrier, 128);
      if (td == 0) mbar_arrive(smem_u32(&d2_empty[ds]));
      for (int e = e0 + td, h = 0; e < e1; e += 128, ++h) {
        const uint32_t w = h == 0 ? w0 : (h == 1 ? w1 : __ldg(pv.ent_pv + e));
        const int pos = (int)(w & 0xFFFFu);
        const int m = ((pos >> 8) << 3) | ((pos >> 4) & 7);
        const int kk = (((pos >> 7) & 1) << 3) | ((pos >> 1) & 7);
        int j = 0;
#pragma unroll
        for (int c = 1; c < kBG; ++c) j += e >= bnd[c] ? 1 : 0;
        const float v = stg[m * kStgStride + 16 * j + kk];
        dval[dval_at ? __ldg(dval_at + e) : e] = v;
      }
      ++dn;
      cb = cb_next;
    }
  }

  __syncthreads();
  if (tid == 0 && *abort_flag) atomicExch(pv.err, kErrMbarTimeout);
  tc_fence_after();
  if (warp == kMmaWarp) tmem_dealloc(tmem, Cfg::kTmemCols);
}

template <bool F16OUT, int NA>
int launch_bwd_t(const tr_plan* p, const __half* dc, const __half* b, void* db, float* dval,
                 cudaStream_t stream) {
  using Cfg = BwdCfg<NA>;
  if (int rc = kernel_smem_limit((const void*)block_bwd_kernel<F16OUT, NA>, Cfg::kSmem)) return rc;
  const int32_t* at = p->res_edge_identity ? nullptr : p->view.ent_src;
  block_bwd_kernel<F16OUT, NA><<<std::max(1, p->view.n_sched), Cfg::kThreads, Cfg::kSmem, stream>>>(
      p->view, dc, b, db, dval, at);
  TRS_CUDA(cudaGetLastError());
  return TR_OK;
}

bool aligned16_(const void* q) { return (reinterpret_cast<uintptr_t>(q) & 15) == 0; }

}  // namespace

bool block_bwd_supported(const tr_plan* p, int32_t k, const void* dc, const void* b, const void* db,
                         const float* dval) {
  return p->blocked && (k == 64 || k == 128) && aligned16_(dc) && aligned16_(b) && aligned16_(db) &&
         p->max_sched_blocks <= kMaxBlk && p->n_edges == p->info.nnz && dval != nullptr &&
         p->view.n_blocks > 0;
}

int launch_block_bwd(const tr_plan* p, const uint16_t* dc, const uint16_t* b, int32_t k, void* db,
                     int db_dtype, float* dval, cudaStream_t stream) {
  const __half* g = reinterpret_cast<const __half*>(dc);
  const __half* bh = reinterpret_cast<const __half*>(b);
  const bool f16 = db_dtype == TR_OUT_F16;
  if (k == 64) return f16 ? launch_bwd_t<true, 1>(p, g, bh, db, dval, stream)
                          : launch_bwd_t<false, 1>(p, g, bh, db, dval, stream);
  return f16 ? launch_bwd_t<true, 2>(p, g, bh, db, dval, stream)
             : launch_bwd_t<false, 2>(p, g, bh, db, dval, stream);
}

}  // namespace trs
