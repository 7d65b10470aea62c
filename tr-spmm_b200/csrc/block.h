// Block engine launchers (block.cu).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "plan.h"

namespace trs {

// K and B alignment the tensor-core block kernel takes (K a multiple of 64,
// 16-byte aligned B; features in tiles of the plan's k_tile, at most 256);
// other shapes run the CUDA-core kernel.
bool block_mma_supported(int32_t k, const void* b);
// Features per tensor-core launch for K (the plan's k_tile, default 256).
int block_k_tile(const tr_plan* p, int32_t k);
// C = A_plan . B over a block plan, FP16 features; every output row written.
int launch_block(const tr_plan* p, const uint16_t* b, int32_t k, void* c, int c_dtype,
                 bool force_generic, cudaStream_t stream);
// The backward of a block plan of A^T on the tensor cores (block_bwd.cu):
// dB = A^T . dC and dval = SDDMM(dC, B) in one pass, for K = 64 or 128.
bool block_bwd_supported(const tr_plan* p, int32_t k, const void* dc, const void* b, const void* db,
                         const float* dval);
int launch_block_bwd(const tr_plan* p, const uint16_t* dc, const uint16_t* b, int32_t k, void* db,
                     int db_dtype, float* dval, cudaStream_t stream);
// The same with FP32 features (CUDA cores, FP32 arithmetic).
int launch_block_f32(const tr_plan* p, const float* b, int32_t k, void* c, int c_dtype,
                     cudaStream_t stream);

}  // namespace trs
