// Persistent, warp-specialised routed forward for sm_100a.
//
// One CTA per SM walks its share of the plan's 16-row windows (round robin
// over the cost-ordered window list, staged once in shared memory) as one
// continuous stream of tensor-core tiles, so the gather pipeline never drains
// between windows:
//
//   producer warps (kProd of them, stage g taken by warp g % kProd)
//       per stage: wait until the stage slot's last MMAs have finished
//       (empty barrier), announce the stage's bytes on its full barrier, and
//       let every lane issue one TMA gather (cp.async.bulk.tensor tile::gather4:
//       4 B rows x 64 features, 128-byte swizzle, straight into the tcgen05
//       MN-major operand layout) plus one bulk copy per tile of its 16x16 A
//       block; the full barrier completes when all bytes have landed, so no
//       thread waits for its own copies;
//   MMA warp (one elected thread)
//       per stage: wait full, issue NCH x tiles tcgen05.mma kind::f16
//       (M = 128 features, N = 16 window rows, K = 16 columns) into the
//       window's accumulator, commit to the slot's empty barrier; after a
//       window's last stage commit to the accumulator's full barrier;
//       accumulators rotate through kAcc TMEM buffers so later windows'
//       MMAs overlap earlier windows' epilogues;
//   epilogue warps 0-3 (thread t <-> TMEM lane t <-> feature t of a chunk)
//       per window: wait for the accumulator, tcgen05.ld its 16 columns,
//       add the window's CUDA-core residual entries (if the plan kept any),
//       apply the row scale and store each output element once, to the
//       row's original position; release the accumulator.  Row metadata is
//       prefetched one window ahead.  In accumulate mode (ACC) the residual
//       has already been written by the CUDA-core kernel: the epilogue reads
//       those values before it waits for the accumulator (all loads ahead of
//       all stores), adds the tiles' product and leaves windows without
//       tiles alone.  kAcc accumulators let the MMAs run up to kAcc windows
//       ahead of the epilogue.
//
// Every wait is bounded (about a second of %globaltimer); a wait that runs
// out raises a CTA-wide abort flag, every role leaves its loop, in-flight
// MMAs are waited for, TMEM is freed and the plan's error word is set for
// the host to report.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <string>

#include "common.cuh"
#include "plan.h"
#include "spmm.h"

namespace trs {
namespace {

constexpr int kSlots = 11;                // stage slots in shared memory
constexpr int kProd = 2;                  // producer warps
constexpr int kEpiWarps = 4;
constexpr int kMmaWarp = kEpiWarps;       // warp 4
constexpr int kProdWarp0 = kEpiWarps + 1; // warps 5 .. 5 + kProd - 1
constexpr int kPipeThreads = (kEpiWarps + 1 + kProd) * 32;
constexpr int kTileAop = 4096;            // 16 columns x 128 features, FP16
constexpr int kTileBop = 512;             // 16 x 16 A block, FP16
constexpr int kMaxWin = 512;              // windows per CTA held in shared memory
constexpr int kAcc = 8;                   // TMEM accumulators (windows in flight)

template <int NCH, int TPS>
struct PipeCfg {
  static constexpr int kSlotAop = TPS * NCH * kTileAop;
  static constexpr int kSlotBop = TPS * kTileBop;
  static constexpr int kSlotBytes = kSlotAop + kSlotBop;   // a multiple of 1024
  static constexpr int kBarOff = kSlots * kSlotBytes;
  // full[S], empty[S], acc_full[kAcc], acc_empty[kAcc], done, tmem slot, abort flag
  static constexpr int kWinOff = kBarOff + (2 * kSlots + 2 * kAcc + 1) * 8 + 16;
  // per window of this CTA: id, first tile, end tile
  static constexpr int kSmem = 1024 + kWinOff + 3 * kMaxWin * 4;
  static constexpr uint32_t kTmemCols = kAcc * NCH * 16;   // 128 or 256 columns
  static_assert(kSlotBytes % 1024 == 0, "stage slots must keep 1024-byte alignment");
  static_assert(kSmem <= 227 * 1024, "shared memory budget");
  static_assert(TPS * 4 * 2 * NCH <= 32, "one gather per lane per stage");
};

int sm_count() {
  static int sms = 0;
  if (!sms) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
      sms = 0;
  }
  return sms;
}

constexpr uint32_t kIdescPipe = umma_idesc_f16(128, 16, /*a MN-major*/ true, /*b MN-major*/ false);

// Bounded wait that also gives up once another role raised the abort flag.
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

__device__ __forceinline__ void mbar_arrive_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(bytes)
               : "memory");
}

// Four rows y0..y3 of the 2-D tensor map, features [x, x + 64), into 512
// bytes of shared memory (128-byte swizzle by address); rows past the end
// of B read as zeros.
__device__ __forceinline__ void tma_gather4(uint32_t dst, const CUtensorMap* map, int x, int y0,
                                            int y1, int y2, int y3, uint32_t bar, uint64_t policy) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile::gather4.mbarrier::complete_tx::bytes"
      ".L2::cache_hint [%0], [%1, {%2, %3, %4, %5, %6}], [%7], %8;\n" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y0), "r"(y1), "r"(y2), "r"(y3), "r"(bar),
      "l"(policy)
      : "memory");
}

// Contiguous global -> shared copy completing on an mbarrier (16-byte aligned).
__device__ __forceinline__ void bulk_copy(uint32_t dst, const void* src, uint32_t bytes,
                                          uint32_t bar, uint64_t policy) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint"
      " [%0], [%1], %2, [%3], %4;\n" ::"r"(dst),
      "l"(src), "r"(bytes), "r"(bar), "l"(policy)
      : "memory");
}

__device__ __forceinline__ void tmem_ld_32x32b_x16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

template <bool F16OUT>
__device__ __forceinline__ void store_out(void* C, int K, int64_t row, int f, float v) {
  if (F16OUT)
    __stcs(reinterpret_cast<__half*>(C) + row * K + f, __float2half_rn(v));
  else
    __stcs(reinterpret_cast<float*>(C) + row * K + f, v);
}

template <bool F16OUT, int NCH, int TPS, bool ACC>
__global__ void __launch_bounds__(kPipeThreads, 1)
    pipe_kernel(PlanView pv, const __grid_constant__ CUtensorMap tmap_b,
                const __half* __restrict__ B, int K, void* C) {
  using Cfg = PipeCfg<NCH, TPS>;
  extern __shared__ uint8_t smem_raw[];
  // 1024-byte aligned base, derived by offsetting the __shared__ array so the
  // compiler keeps it in the shared address space (LDS/STS/ATOMS, not generic)
  uint8_t* smem = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + Cfg::kBarOff);
  uint64_t* full = bars;
  uint64_t* empty = bars + kSlots;
  uint64_t* acc_full = bars + 2 * kSlots;
  uint64_t* acc_empty = acc_full + kAcc;
  uint64_t* done = acc_empty + kAcc;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int W = pv.n_windows;

  if (warp == 0) {
    tmem_alloc(smem_u32(tmem_slot), Cfg::kTmemCols);
    tmem_relinquish();
  }
  if (tid == 32) {
    for (int s = 0; s < kSlots; ++s) {
      mbar_init(smem_u32(&full[s]), 1);
      mbar_init(smem_u32(&empty[s]), 1);
    }
    for (int a = 0; a < kAcc; ++a) {
      mbar_init(smem_u32(&acc_full[a]), 1);
      mbar_init(smem_u32(&acc_empty[a]), kEpiWarps);
    }
    mbar_init(smem_u32(done), 1);
    *abort_flag = 0;
    fence_mbar_init();
  }
  // this CTA's windows (round robin over the cost-ordered list), staged once
  int* s_w = reinterpret_cast<int*>(smem + Cfg::kWinOff);
  int* s_t0 = s_w + kMaxWin;
  int* s_t1 = s_t0 + kMaxWin;
  const int nwin =
      W > (int)blockIdx.x ? (W - (int)blockIdx.x + (int)gridDim.x - 1) / (int)gridDim.x : 0;
  for (int i = tid; i < nwin; i += blockDim.x) {
    const int w = pv.win_order[blockIdx.x + i * gridDim.x];
    s_w[i] = w;
    s_t0[i] = pv.win_tile[w];
    s_t1[i] = pv.win_tile[w + 1];
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp >= kProdWarp0) {
    // ------------------------------------------------------------ producers
    const int p = warp - kProdWarp0;
    const uint64_t pol_keep = l2_policy_evict_last(), pol_stream = l2_policy_evict_first();
    const int nh = K >> 6;                       // 64-feature boxes per B row (1..4)
    const int ops_per_tile = 4 * nh;             // gather4 ops per tile
    const int n_b_rows = pv.n_cols;              // row index past the end: zero fill
    // Stage cursor: stage g of the CTA's stream is window i's tiles [t, t+TPS);
    // this warp takes the stages with g % kProd == p.
    int ci = 0, ct = nwin > 0 ? s_t0[0] : 0, cg = 0;
    auto advance = [&]() -> bool {
      while (ci < nwin) {
        if (ct >= s_t1[ci]) {
          if (++ci < nwin) ct = s_t0[ci];
          continue;
        }
        if (cg % kProd == p) return true;
        ct += TPS;
        ++cg;
      }
      return false;
    };
    // the lane's gather of a stage: tile op_i, rows 4*op_q .. 4*op_q+3, box op_h
    const int op_i = lane / ops_per_tile, op_r = lane % ops_per_tile;
    const int op_q = op_r / nh, op_h = op_r % nh;
    auto load_quad = [&](int t, int nt) -> int4 {
      if (op_i < nt)
        return __ldg(reinterpret_cast<const int4*>(pv.tile_col + (int64_t)(t + op_i) * 16 + op_q * 4));
      return make_int4(-1, -1, -1, -1);
    };
    bool have = advance();
    int nx_t = ct, nx_nt = have ? min(TPS, s_t1[ci] - ct) : 0, nx_g = cg;
    int4 q_nx = have ? load_quad(nx_t, nx_nt) : make_int4(-1, -1, -1, -1);
    while (have) {
      const int t = nx_t, nt = nx_nt, g = nx_g;
      const int4 q = q_nx;
      ct += TPS;
      ++cg;
      have = advance();
      if (have) {                                // prefetch the next stage's columns
        nx_t = ct;
        nx_nt = min(TPS, s_t1[ci] - ct);
        nx_g = cg;
        q_nx = load_quad(nx_t, nx_nt);
      }
      const int sl = g % kSlots, use = g / kSlots;
      if (!wait_bar(smem_u32(&empty[sl]), (use & 1) ^ 1, abort_flag)) break;
      uint8_t* slot = smem + sl * Cfg::kSlotBytes;
      const uint32_t fb = smem_u32(&full[sl]);
      if (lane == 0) mbar_arrive_expect_tx(fb, (uint32_t)nt * (uint32_t)(nh * 2048 + kTileBop));
      __syncwarp();
      if (op_i < nt) {
        const uint32_t dst = smem_u32(slot + op_i * NCH * kTileAop + (op_h >> 1) * kTileAop) +
                             (op_q >> 1) * 2048 + (op_h & 1) * 1024 + (op_q & 1) * 512;
        tma_gather4(dst, &tmap_b, op_h * 64, q.x >= 0 ? q.x : n_b_rows, q.y >= 0 ? q.y : n_b_rows,
                    q.z >= 0 ? q.z : n_b_rows, q.w >= 0 ? q.w : n_b_rows, fb, pol_keep);
      }
      if (lane < nt)
        bulk_copy(smem_u32(slot + Cfg::kSlotAop + lane * kTileBop),
                  pv.tile_a + (int64_t)(t + lane) * 256, kTileBop, fb, pol_stream);
    }
  } else if (warp == kMmaWarp) {
    // ------------------------------------------------------------ MMA issuer
    if (lane == 0) {
      int g = 0, nacc = 0;
      bool ok = true;
      for (int i = 0; i < nwin && ok; ++i) {
        const int t0 = s_t0[i], t1 = s_t1[i];
        if (t1 == t0) continue;
        const int a = nacc % kAcc, u = nacc / kAcc;
        if (!wait_bar(smem_u32(&acc_empty[a]), (u & 1) ^ 1, abort_flag)) { ok = false; break; }
        tc_fence_after();
        const uint32_t dcol = tmem + (uint32_t)(a * NCH * 16);
        for (int t = t0; t < t1; t += TPS, ++g) {
          const int s = g % kSlots, use = g / kSlots;
          if (!wait_bar(smem_u32(&full[s]), use & 1, abort_flag)) { ok = false; break; }
          tc_fence_after();
          const int nt = min(TPS, t1 - t);
          uint8_t* slot = smem + s * Cfg::kSlotBytes;
          for (int j = 0; j < nt; ++j) {
            const uint64_t bdesc =
                umma_smem_desc(smem_u32(slot + Cfg::kSlotAop + j * kTileBop), 128, 256, 0);
#pragma unroll
            for (int c = 0; c < NCH; ++c) {
              const uint64_t adesc =
                  umma_smem_desc(smem_u32(slot + (j * NCH + c) * kTileAop), 1024, 2048, 2);
              umma_f16(dcol + c * 16, adesc, bdesc, kIdescPipe, (t + j > t0) ? 1u : 0u);
            }
          }
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
    const int e = warp;                          // TMEM lanes 32e .. 32e+31
    // row metadata of a window, lane r < 16 holding row r
    auto load_rows = [&](int i, int& ro, float& sc, int& rp0, int& rp1) {
      ro = -1; sc = 1.f; rp0 = rp1 = 0;
      if (i < nwin && lane < 16) {
        const int64_t r = (int64_t)s_w[i] * 16 + lane;
        ro = __ldg(pv.row_out + r);
        sc = __ldg(pv.row_scale + r);
        rp0 = __ldg(pv.res_ptr + r);
        rp1 = __ldg(pv.res_ptr + r + 1);
      }
    };
    int nro, nrp0, nrp1;
    float nsc;
    load_rows(0, nro, nsc, nrp0, nrp1);
    int nacc = 0;
    for (int i = 0; i < nwin; ++i) {
      const int ro = nro, rp0 = nrp0, rp1 = nrp1;
      const float scl = nsc;
      load_rows(i + 1, nro, nsc, nrp0, nrp1);
      const bool has = s_t1[i] > s_t0[i];
      if (ACC && !has) continue;
      // accumulate mode: C already holds the residual (written by an earlier
      // kernel on the stream), so its values are read before the wait
      float prev[NCH][16];
      if (ACC) {
#pragma unroll
        for (int r = 0; r < 16; ++r) {
          const int out = __shfl_sync(0xffffffffu, ro, r);
#pragma unroll
          for (int c = 0; c < NCH; ++c) {
            const int f = c * 128 + e * 32 + lane;
            const int64_t at = (int64_t)(out < 0 ? 0 : out) * K + (f < K ? f : 0);
            prev[c][r] = F16OUT ? __half2float(reinterpret_cast<const __half*>(C)[at])
                                : reinterpret_cast<const float*>(C)[at];
          }
        }
      }
      float d[NCH][16];
      if (has) {
        const int a = nacc % kAcc, u = nacc / kAcc;
        if (!wait_bar(smem_u32(&acc_full[a]), u & 1, abort_flag)) break;
        tc_fence_after();
#pragma unroll
        for (int c = 0; c < NCH; ++c)
          tmem_ld_32x32b_x16(tmem + ((uint32_t)(32 * e) << 16) + (uint32_t)((a * NCH + c) * 16), d[c]);
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(smem_u32(&acc_empty[a]));
        ++nacc;
      } else {
#pragma unroll
        for (int c = 0; c < NCH; ++c)
#pragma unroll
          for (int r = 0; r < 16; ++r) d[c][r] = 0.f;
      }
      if (ACC) {
#pragma unroll
        for (int r = 0; r < 16; ++r) {
          const int out = __shfl_sync(0xffffffffu, ro, r);
          const float sc = __shfl_sync(0xffffffffu, scl, r);
          if (out < 0) continue;
#pragma unroll
          for (int c = 0; c < NCH; ++c) {
            const int f = c * 128 + e * 32 + lane;
            if (f < K) store_out<F16OUT>(C, K, out, f, prev[c][r] + d[c][r] * sc);
          }
        }
        continue;
      }
#pragma unroll
      for (int r = 0; r < 16; ++r) {
        const int out = __shfl_sync(0xffffffffu, ro, r);
        const float sc = __shfl_sync(0xffffffffu, scl, r);
        const int e0 = __shfl_sync(0xffffffffu, rp0, r), e1 = __shfl_sync(0xffffffffu, rp1, r);
        if (out < 0) continue;
#pragma unroll
        for (int c = 0; c < NCH; ++c) {
          const int f = c * 128 + e * 32 + lane;
          float acc = d[c][r];
          if (f < K) {
            for (int q = e0; q < e1; ++q) {
              const float v = __half2float(__ushort_as_half(__ldg(pv.res_val + q)));
              acc = fmaf(v, __half2float(B[(int64_t)__ldg(pv.res_col + q) * K + f]), acc);
            }
            store_out<F16OUT>(C, K, out, f, acc * sc);
          }
        }
      }
    }
  }

  __syncthreads();
  if (tid == 0 && *abort_flag) atomicExch(pv.err, kErrMbarTimeout);
  tc_fence_after();
  if (warp == 0) tmem_dealloc(tmem, Cfg::kTmemCols);
}

// Tensor map over B [n_cols, K] FP16 for the gathers: boxes of 1 row x 64
// features (128 bytes), 128-byte swizzle, zero fill past the last row.
int make_b_map(CUtensorMap* map, const void* b, int32_t n_cols, int32_t k) {
  static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
  if (!encode) {
    cudaDriverEntryPointQueryResult q;
    void* fn = nullptr;
    TRS_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q));
    if (q != cudaDriverEntryPointSuccess || !fn)
      return fail(TR_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
    encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
  }
  const cuuint64_t dims[2] = {(cuuint64_t)k, (cuuint64_t)std::max(n_cols, 1)};
  const cuuint64_t strides[1] = {(cuuint64_t)k * 2};
  const cuuint32_t box[2] = {64, 1};
  const cuuint32_t estr[2] = {1, 1};
  const CUresult r = encode(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 2, const_cast<void*>(b), dims,
                            strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                            CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS)
    return fail(TR_ERR_CUDA, "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
  return TR_OK;
}

template <bool F16OUT, int NCH, int TPS, bool ACC>
int launch_pipe_t(const tr_plan* p, const __half* b, int32_t k, void* c, cudaStream_t stream) {
  using Cfg = PipeCfg<NCH, TPS>;
  if (int rc = kernel_smem_limit((const void*)pipe_kernel<F16OUT, NCH, TPS, ACC>, Cfg::kSmem))
    return rc;
  CUtensorMap map;
  int rc = make_b_map(&map, b, p->view.n_cols, k);
  if (rc) return rc;
  const int grid = std::max(1, std::min(sm_count(), p->view.n_windows));
  pipe_kernel<F16OUT, NCH, TPS, ACC><<<grid, kPipeThreads, Cfg::kSmem, stream>>>(p->view, map, b, k, c);
  TRS_CUDA(cudaGetLastError());
  return TR_OK;
}

}  // namespace

// TMA boxes are 64 features wide and lie fully inside B's rows.
bool pipe_supported(int32_t k, const void* b) {
  return k > 0 && k % 64 == 0 && k <= 256 && (reinterpret_cast<uintptr_t>(b) & 15) == 0;
}

bool pipe_fits(const tr_plan* p) {
  const int sms = sm_count();
  return sms > 0 && (int64_t)p->view.n_windows <= (int64_t)sms * kMaxWin;
}

int launch_pipe(const tr_plan* p, const uint16_t* b, int32_t k, void* c, int c_dtype,
                bool accumulate, cudaStream_t stream) {
  if (p->view.n_rows == 0 || k == 0) return TR_OK;
  if (!pipe_supported(k, b) || !pipe_fits(p))
    return fail(TR_ERR_UNSUPPORTED,
                "pipelined kernel needs K % 64 == 0, K <= 256 and at most 512 windows per SM");
  const __half* bh = reinterpret_cast<const __half*>(b);
  const bool f16 = c_dtype == TR_OUT_F16;
  if (accumulate) {
    if (k <= 128)
      return f16 ? launch_pipe_t<true, 1, 4, true>(p, bh, k, c, stream)
                 : launch_pipe_t<false, 1, 4, true>(p, bh, k, c, stream);
    return f16 ? launch_pipe_t<true, 2, 2, true>(p, bh, k, c, stream)
               : launch_pipe_t<false, 2, 2, true>(p, bh, k, c, stream);
  }
  if (k <= 128)
    return f16 ? launch_pipe_t<true, 1, 4, false>(p, bh, k, c, stream)
               : launch_pipe_t<false, 1, 4, false>(p, bh, k, c, stream);
  return f16 ? launch_pipe_t<true, 2, 2, false>(p, bh, k, c, stream)
             : launch_pipe_t<false, 2, 2, false>(p, bh, k, c, stream);
}

}  // namespace trs
