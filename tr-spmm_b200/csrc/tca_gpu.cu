// GPU stages of the TCA row clustering: MinHash signatures with their LSH
// band digests, and the set intersections behind the exact Jaccard
// similarity of every candidate pair.  Integer work, bound by the hashing
// (signatures: 128 hashes per column entry) and by scattered list reads
// (intersections); the host keeps the bucket sort and the clustering.
// Both stages compute exactly what the host stages in tca.cpp compute.
#include <cuda_runtime.h>

#include <algorithm>
#include <string>
#include <vector>

#include "../../include/trspmm.h"
#include "tca.h"

namespace trs {
namespace {

constexpr int kSigWarps = 8;                 // rows per CTA (one warp each)
constexpr int kPermPerLane = kTcaPerm / 32;

// One warp per row: lane l keeps permutations l, l + 32, l + 64, l + 96;
// the warp walks the row's columns 32 at a time (each lane hashes one
// column id into its key, keys are broadcast with shuffles).  Band j's
// digest is taken from the signature staged in shared memory.
__global__ void __launch_bounds__(kSigWarps * 32) tca_signature_kernel(
    const int64_t* __restrict__ ptr, const int32_t* __restrict__ col, int32_t n, uint64_t seed,
    int bands, int rows, uint32_t* __restrict__ sig, uint64_t* __restrict__ dig) {
  __shared__ uint32_t stage[kSigWarps][kTcaPerm];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  uint64_t a[kPermPerLane], b[kPermPerLane];
#pragma unroll
  for (int k = 0; k < kPermPerLane; ++k) {
    a[k] = tca_perm_a(seed, lane + 32 * k);
    b[k] = tca_perm_b(seed, lane + 32 * k);
  }
  for (int64_t r = (int64_t)blockIdx.x * kSigWarps + w; r < n; r += (int64_t)gridDim.x * kSigWarps) {
    uint32_t v[kPermPerLane];
#pragma unroll
    for (int k = 0; k < kPermPerLane; ++k) v[k] = 0xFFFFFFFFu;
    const int64_t e0 = ptr[r], e1 = ptr[r + 1];
    for (int64_t base = e0; base < e1; base += 32) {
      const int cnt = (int)(e1 - base < 32 ? e1 - base : 32);
      const uint32_t mine = lane < cnt ? tca_key(col[base + lane]) : 0u;
      for (int i = 0; i < cnt; ++i) {
        const uint32_t key = __shfl_sync(0xffffffffu, mine, i);
#pragma unroll
        for (int k = 0; k < kPermPerLane; ++k) v[k] = min(v[k], tca_hash(a[k], b[k], key));
      }
    }
#pragma unroll
    for (int k = 0; k < kPermPerLane; ++k) {
      stage[w][lane + 32 * k] = v[k];
      sig[r * kTcaPerm + lane + 32 * k] = v[k];
    }
    __syncwarp();
    for (int j = lane; j < bands; j += 32) dig[r * bands + j] = tca_band_digest(&stage[w][j * rows], rows, j);
    __syncwarp();
  }
}

__device__ int32_t intersect_count_dev(const int32_t* x, int64_t nx, const int32_t* y, int64_t ny) {
  if (nx > ny) {
    const int32_t* t = x;
    x = y;
    y = t;
    const int64_t tn = nx;
    nx = ny;
    ny = tn;
  }
  int32_t c = 0;
  if (nx * 8 < ny) {                         // lopsided: binary search the long list
    for (int64_t i = 0; i < nx; ++i) {
      const int32_t v = x[i];
      int64_t lo = 0, hi = ny;
      while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if (y[mid] < v) lo = mid + 1;
        else hi = mid;
      }
      c += (lo < ny && y[lo] == v) ? 1 : 0;
    }
    return c;
  }
  for (int64_t i = 0, j = 0; i < nx && j < ny;) {
    const int32_t p = x[i], q = y[j];
    c += p == q ? 1 : 0;
    i += p <= q ? 1 : 0;
    j += q <= p ? 1 : 0;
  }
  return c;
}

__global__ void tca_intersect_kernel(const int64_t* __restrict__ ptr, const int32_t* __restrict__ col,
                                     const int32_t* __restrict__ pa, const int32_t* __restrict__ pb,
                                     int64_t n_pairs, int32_t* __restrict__ inter) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n_pairs;
       k += (int64_t)gridDim.x * blockDim.x) {
    const int32_t i = pa[k], j = pb[k];
    inter[k] = intersect_count_dev(col + ptr[i], ptr[i + 1] - ptr[i], col + ptr[j], ptr[j + 1] - ptr[j]);
  }
}

// Device buffers of one call, freed on every exit path.
struct Bufs {
  std::vector<void*> p;
  ~Bufs() {
    for (void* x : p) cudaFree(x);
  }
  template <class T> cudaError_t alloc(T** out, size_t count) {
    void* x = nullptr;
    const cudaError_t e = cudaMalloc(&x, std::max<size_t>(count, 1) * sizeof(T));
    if (e == cudaSuccess) p.push_back(x);
    *out = static_cast<T*>(x);
    return e;
  }
};

int cuda_err(cudaError_t e, const char* what, std::string& err) {
  err = std::string(what) + ": " + cudaGetErrorString(e);
  return TR_ERR_CUDA;
}

int sm_count() {
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return sms;
}

}  // namespace

int tca_signatures_gpu(const std::vector<int64_t>& ptr, const std::vector<int32_t>& col,
                       uint64_t seed, int bands, int rows, std::vector<uint32_t>& sig,
                       std::vector<uint64_t>& dig, std::string& err) {
  const int64_t n = (int64_t)ptr.size() - 1;
  sig.resize((size_t)n * kTcaPerm);
  dig.resize((size_t)n * bands);
  if (n == 0) return TR_OK;
  Bufs B;
  int64_t* d_ptr;
  int32_t* d_col;
  uint32_t* d_sig;
  uint64_t* d_dig;
  cudaError_t e = B.alloc(&d_ptr, ptr.size());
  if (e == cudaSuccess) e = B.alloc(&d_col, col.size());
  if (e == cudaSuccess) e = B.alloc(&d_sig, sig.size());
  if (e == cudaSuccess) e = B.alloc(&d_dig, dig.size());
  if (e == cudaSuccess) e = cudaMemcpy(d_ptr, ptr.data(), ptr.size() * 8, cudaMemcpyHostToDevice);
  if (e == cudaSuccess && !col.empty()) e = cudaMemcpy(d_col, col.data(), col.size() * 4, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return cuda_err(e, "TCA signatures (upload)", err);
  const int64_t want = (n + kSigWarps - 1) / kSigWarps;
  const int grid = (int)std::min<int64_t>(want, (int64_t)sm_count() * 8);
  tca_signature_kernel<<<grid, kSigWarps * 32>>>(d_ptr, d_col, (int32_t)n, seed, bands, rows, d_sig, d_dig);
  e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpy(sig.data(), d_sig, sig.size() * 4, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(dig.data(), d_dig, dig.size() * 8, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_err(e, "TCA signatures", err);
  return TR_OK;
}

int tca_intersections_gpu(const std::vector<int64_t>& ptr, const std::vector<int32_t>& col,
                          const std::vector<int32_t>& pa, const std::vector<int32_t>& pb,
                          std::vector<int32_t>& inter, std::string& err) {
  const int64_t P = (int64_t)pa.size();
  inter.resize(P);
  if (P == 0) return TR_OK;
  Bufs B;
  int64_t* d_ptr;
  int32_t *d_col, *d_pa, *d_pb, *d_out;
  cudaError_t e = B.alloc(&d_ptr, ptr.size());
  if (e == cudaSuccess) e = B.alloc(&d_col, col.size());
  if (e == cudaSuccess) e = B.alloc(&d_pa, P);
  if (e == cudaSuccess) e = B.alloc(&d_pb, P);
  if (e == cudaSuccess) e = B.alloc(&d_out, P);
  if (e == cudaSuccess) e = cudaMemcpy(d_ptr, ptr.data(), ptr.size() * 8, cudaMemcpyHostToDevice);
  if (e == cudaSuccess && !col.empty()) e = cudaMemcpy(d_col, col.data(), col.size() * 4, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d_pa, pa.data(), P * 4, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d_pb, pb.data(), P * 4, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return cuda_err(e, "TCA intersections (upload)", err);
  const int grid = (int)std::min<int64_t>((P + 255) / 256, (int64_t)sm_count() * 16);
  tca_intersect_kernel<<<grid, 256>>>(d_ptr, d_col, d_pa, d_pb, P, d_out);
  e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpy(inter.data(), d_out, P * 4, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_err(e, "TCA intersections", err);
  return TR_OK;
}

}  // namespace trs
