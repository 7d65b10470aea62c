/* ORACLE — test infrastructure only.  Nothing in the shipped library links,
 * loads or calls this file; only tests/, the smoke check and bench.py's CPU
 * baseline leg use it, and only as the checker.
 *
 * CPU restatement of what the reference's routed forward computes once its
 * three routes are summed (TR-source/SpMM/mGCNkernel_online.cu:1529-1727,
 * merge at :1314-1324): C = A·B over the matrix the route tables encode,
 * with FP16 inputs.  Two arithmetic variants:
 *   - oracle_spmm_f64:     FP64 accumulation; the accuracy arbiter.
 *   - oracle_spmm_f16_f32: FP16 operands, FP32 accumulation, FP32 output;
 *     the same arithmetic as the GPU path, multi-threaded, timed as the CPU
 *     baseline of bench.py.
 * Plus the adjoint pieces used by the gradient checks:
 *   - oracle_sddmm_f64:    dval[e] = <dC[row(e),:], B[col(e),:]>;
 *   - oracle_sddmm_f16_f32: the same with FP16 operands and FP32 sums, the
 *     arithmetic of the GPU SDDMM (timed in bench.py's CPU baseline).
 */
#include <stdint.h>
#include <string.h>
#include <omp.h>

static inline float h2f(uint16_t b) {
  _Float16 h;
  memcpy(&h, &b, 2);
  return (float)h;
}

void oracle_spmm_f64(const int* rowptr, const int* col, const double* val, int m,
                     const double* b, int k, double* c) {
  #pragma omp parallel for schedule(dynamic, 64)
  for (int r = 0; r < m; ++r) {
    double* cr = c + (int64_t)r * k;
    for (int j = 0; j < k; ++j) cr[j] = 0.0;
    for (int e = rowptr[r]; e < rowptr[r + 1]; ++e) {
      const double v = val[e];
      const double* br = b + (int64_t)col[e] * k;
      for (int j = 0; j < k; ++j) cr[j] += v * br[j];
    }
  }
}

/* FP16 values and features, FP32 accumulation in CSR order, FP32 output.
 * `threads` <= 0 means all OpenMP threads. */
void oracle_spmm_f16_f32(const int* rowptr, const int* col, const uint16_t* val, int m,
                         const uint16_t* b, int k, float* c, int threads) {
  if (threads > 0) omp_set_num_threads(threads);
  #pragma omp parallel
  {
    float* acc = (float*)__builtin_alloca(sizeof(float) * (size_t)k);
    #pragma omp for schedule(dynamic, 64)
    for (int r = 0; r < m; ++r) {
      for (int j = 0; j < k; ++j) acc[j] = 0.f;
      for (int e = rowptr[r]; e < rowptr[r + 1]; ++e) {
        const float v = h2f(val[e]);
        const uint16_t* br = b + (int64_t)col[e] * k;
        for (int j = 0; j < k; ++j) acc[j] += v * h2f(br[j]);
      }
      memcpy(c + (int64_t)r * k, acc, sizeof(float) * (size_t)k);
    }
  }
}

int oracle_max_threads(void) { return omp_get_max_threads(); }

void oracle_sddmm_f64(const int* rowptr, const int* col, int m, const double* dc,
                      const double* b, int k, double* dval) {
  #pragma omp parallel for schedule(dynamic, 64)
  for (int r = 0; r < m; ++r) {
    const double* g = dc + (int64_t)r * k;
    for (int e = rowptr[r]; e < rowptr[r + 1]; ++e) {
      const double* br = b + (int64_t)col[e] * k;
      double s = 0.0;
      for (int j = 0; j < k; ++j) s += g[j] * br[j];
      dval[e] = s;
    }
  }
}

void oracle_sddmm_f16_f32(const int* rowptr, const int* col, int m, const uint16_t* dc,
                          const uint16_t* b, int k, float* dval, int threads) {
  if (threads > 0) omp_set_num_threads(threads);
  #pragma omp parallel for schedule(dynamic, 64)
  for (int r = 0; r < m; ++r) {
    const uint16_t* g = dc + (int64_t)r * k;
    for (int e = rowptr[r]; e < rowptr[r + 1]; ++e) {
      const uint16_t* br = b + (int64_t)col[e] * k;
      float s = 0.f;
      for (int j = 0; j < k; ++j) s += h2f(g[j]) * h2f(br[j]);
      dval[e] = s;
    }
  }
}
