// Kernel launchers (spmm.cu).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "plan.h"

namespace trs {

int launch_csr(const int32_t* indptr, const int32_t* indices, const uint16_t* values, int32_t m,
               const uint16_t* b, int32_t k, void* c, int c_dtype, cudaStream_t stream);
int launch_set_values(tr_plan* p, const float* values, cudaStream_t stream);
// out_id (optional, nnz entries): entry e's result goes to out[out_id[e]]
// (a plan whose edges were renumbered), else to out[e].
int launch_sddmm(const int32_t* indptr, const int32_t* indices, int32_t m, int64_t nnz,
                 const uint16_t* x, const uint16_t* y, int32_t k, float* out, cudaStream_t stream,
                 const int32_t* out_id = nullptr);
bool pipe_supported(int32_t k, const void* b);
bool pipe_fits(const tr_plan* p);
int launch_pipe(const tr_plan* p, const uint16_t* b, int32_t k, void* c, int c_dtype,
                bool accumulate, cudaStream_t stream);
int launch_adjoint_sddmm(const tr_plan* p, const int32_t* a_indptr, const int32_t* a_indices,
                         int32_t a_rows, int64_t nnz, const uint16_t* dc, const uint16_t* b,
                         int32_t k, void* db, int db_dtype, float* dval, cudaStream_t stream);
int launch_routed(const tr_plan* p, const uint16_t* b, int32_t k, void* c, int c_dtype,
                  int route_mask, cudaStream_t stream);
int launch_routed_f32(const tr_plan* p, const float* b, int32_t k, void* c, int c_dtype,
                      int route_mask, cudaStream_t stream);
int launch_adjoint_sddmm_f32(const tr_plan* p, const int32_t* a_indptr, const int32_t* a_indices,
                             int32_t a_rows, int64_t nnz, const float* dc, const float* b,
                             int32_t k, void* db, int db_dtype, float* dval, cudaStream_t stream);
int launch_sddmm_f32(const int32_t* indptr, const int32_t* indices, int32_t m, int64_t nnz,
                     const float* x, const float* y, int32_t k, float* out, cudaStream_t stream,
                     const int32_t* out_id = nullptr);
// Edge numbering of a plan (edges.cu): the plan position of every edge
// (entry_order[q] = the edge at position q) and renumbering a plan's edges.
int launch_entry_order(const tr_plan* p, int32_t* order, cudaStream_t stream);
int launch_renumber_edges(tr_plan* p, const int32_t* new_id, cudaStream_t stream);

}  // namespace trs
