// Edge numbering of a device plan.
//
// A plan addresses the per-entry values of A (tr_plan_set_values' input, the
// SDDMM's dval output) by edge number, and edges start numbered as A's CSR
// entries.  A caller that keeps its per-entry arrays in another order — the
// adjoint plan's own entry order makes both the value upload and the fused
// backward's dval stores sequential — renumbers the plan's edges once:
// every per-edge map of the plan is permuted to the new numbering, and the
// SDDMM over A's CSR (the non-fused backward) writes through edge_id.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "common.cuh"
#include "plan.h"
#include "spmm.h"

namespace trs {
namespace {

constexpr int kThreads = 256;

int grid_for(int64_t n) { return (int)std::min<int64_t>((n + kThreads - 1) / kThreads, 148 * 32); }

// order[q] = e for the edge e whose value slot is plan position q.
__global__ void entry_order_kernel(const int32_t* __restrict__ slot, int64_t n, int64_t n_pos,
                                   int64_t base, bool blocked, int32_t* __restrict__ order,
                                   int* bad) {
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t s = slot[e];
    if (s < 0) continue;
    const int64_t q = blocked ? (s - 1) >> 1 : s - base;
    if (q < 0 || q >= n_pos) { atomicOr(bad, 1); continue; }
    order[q] = (int32_t)e;
  }
}

// Counts how often each new number is taken; flags numbers out of range.
__global__ void count_ids_kernel(const int32_t* __restrict__ id, int64_t n, int* hits, int* bad) {
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int32_t v = id[e];
    if (v < 0 || v >= n) atomicOr(bad, 1);
    else atomicAdd(hits + v, 1);
  }
}

__global__ void check_hits_kernel(const int* __restrict__ hits, int64_t n, int* bad) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    if (hits[i] != 1) atomicOr(bad, 1);
}

// out_a[id[e]] = a[e], out_b[id[e]] = b[e]
__global__ void permute_maps_kernel(const int32_t* __restrict__ id, int64_t n,
                                    const int32_t* __restrict__ a, const int32_t* __restrict__ b,
                                    int32_t* __restrict__ out_a, int32_t* __restrict__ out_b) {
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n;
       e += (int64_t)gridDim.x * blockDim.x) {
    const int32_t t = id[e];
    out_a[t] = a[e];
    out_b[t] = b[e];
  }
}

// x[q] = id[x[q]] for x[q] >= 0; *moved = 1 if any x[q] != q afterwards.
__global__ void renumber_kernel(int32_t* __restrict__ x, int64_t m, const int32_t* __restrict__ id,
                                int* moved) {
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < m;
       q += (int64_t)gridDim.x * blockDim.x) {
    int32_t v = x[q];
    if (v >= 0) {
      v = id[v];
      x[q] = v;
    }
    if (v != q) atomicOr(moved, 1);
  }
}

// Stream-ordered scratch, released on every return path.
struct AsyncScratch {
  void* p = nullptr;
  cudaStream_t stream;
  explicit AsyncScratch(cudaStream_t s) : stream(s) {}
  ~AsyncScratch() { if (p) cudaFreeAsync(p, stream); }
};

}  // namespace

int launch_entry_order(const tr_plan* p, int32_t* order, cudaStream_t stream) {
  const int64_t n = p->n_edges;
  if (!p->blocked && p->n_tile_vals > 0)
    return fail(TR_ERR_UNSUPPORTED, "the plan has tensor-core tiles: its entries have no single order");
  if (n == 0) return TR_OK;
  AsyncScratch scratch(stream);
  TRS_CUDA(cudaMallocAsync(&scratch.p, sizeof(int), stream));
  int* bad = static_cast<int*>(scratch.p);
  TRS_CUDA(cudaMemsetAsync(bad, 0, sizeof(int), stream));
  TRS_CUDA(cudaMemsetAsync(order, 0xFF, (size_t)n * 4, stream));
  entry_order_kernel<<<grid_for(n), kThreads, 0, stream>>>(p->val_slot, n, n, p->n_tile_vals,
                                                           p->blocked, order, bad);
  TRS_CUDA(cudaGetLastError());
  int h_bad = 0;
  TRS_CUDA(cudaMemcpyAsync(&h_bad, bad, sizeof(int), cudaMemcpyDeviceToHost, stream));
  TRS_CUDA(cudaStreamSynchronize(stream));
  if (h_bad) return fail(TR_ERR_ARG, "a value slot lies outside the plan's entry range");
  return TR_OK;
}

int launch_renumber_edges(tr_plan* p, const int32_t* new_id, cudaStream_t stream) {
  const int64_t n = p->n_edges;
  if (n == 0) return TR_OK;
  // scratch: hits / permuted val_slot (n), permuted edge_row (n), two flags
  AsyncScratch scratch(stream);
  TRS_CUDA(cudaMallocAsync(&scratch.p, (size_t)(2 * n + 2) * 4, stream));
  int32_t* tmp = static_cast<int32_t*>(scratch.p);
  int* hits = tmp;
  int* flags = tmp + 2 * n;
  TRS_CUDA(cudaMemsetAsync(hits, 0, (size_t)n * 4, stream));
  TRS_CUDA(cudaMemsetAsync(flags, 0, 8, stream));
  count_ids_kernel<<<grid_for(n), kThreads, 0, stream>>>(new_id, n, hits, flags);
  check_hits_kernel<<<grid_for(n), kThreads, 0, stream>>>(hits, n, flags);
  TRS_CUDA(cudaGetLastError());
  int h_flags[2] = {0, 0};
  TRS_CUDA(cudaMemcpyAsync(h_flags, flags, 4, cudaMemcpyDeviceToHost, stream));
  TRS_CUDA(cudaStreamSynchronize(stream));
  if (h_flags[0]) return fail(TR_ERR_ARG, "new edge numbers must be a permutation of 0 .. n_edges - 1");
  int32_t* slot2 = tmp;
  int32_t* row2 = tmp + n;
  permute_maps_kernel<<<grid_for(n), kThreads, 0, stream>>>(new_id, n, p->val_slot, p->edge_row,
                                                            slot2, row2);
  TRS_CUDA(cudaGetLastError());
  TRS_CUDA(cudaMemcpyAsync(p->val_slot, slot2, (size_t)n * 4, cudaMemcpyDeviceToDevice, stream));
  TRS_CUDA(cudaMemcpyAsync(p->edge_row, row2, (size_t)n * 4, cudaMemcpyDeviceToDevice, stream));
  // the stream maps of the kernels (res_edge of window plans, ent_src of
  // block plans) live in the plan's own allocation
  const int64_t m = p->blocked ? p->info.nnz : p->info.residual_nnz;
  int32_t* stream_map = const_cast<int32_t*>(p->blocked ? p->view.ent_src : p->view.res_edge);
  if (m > 0 && stream_map) {
    renumber_kernel<<<grid_for(m), kThreads, 0, stream>>>(stream_map, m, new_id, flags + 1);
    TRS_CUDA(cudaGetLastError());
  }
  if (!p->edge_id) {
    TRS_CUDA(cudaMalloc(&p->edge_id, (size_t)n * 4));
    TRS_CUDA(cudaMemcpyAsync(p->edge_id, new_id, (size_t)n * 4, cudaMemcpyDeviceToDevice, stream));
  } else {
    int* ignore = hits;   // slot2 is no longer needed
    renumber_kernel<<<grid_for(n), kThreads, 0, stream>>>(p->edge_id, n, new_id, ignore);
    TRS_CUDA(cudaGetLastError());
  }
  TRS_CUDA(cudaMemcpyAsync(h_flags + 1, flags + 1, 4, cudaMemcpyDeviceToHost, stream));
  TRS_CUDA(cudaStreamSynchronize(stream));
  p->res_edge_identity = m > 0 && stream_map && h_flags[1] == 0;
  return TR_OK;
}

}  // namespace trs
