// extern "C" entry points of libtrspmm.so (declared in include/trspmm.h).
#include <cuda_runtime.h>

#include <chrono>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

#include "../../include/trspmm.h"
#include "common.cuh"
#include "block.h"
#include "plan.h"
#include "route_gpu.h"
#include "route_full_gpu.h"
#include "router.h"
#include "spmm.h"
#include "tca.h"

namespace trs {

int match_online_gpu(const int32_t* indptr, const int32_t* indices, int32_t n_rows,
                     int32_t dense_threshold, int32_t t_max, tr_match_stats* st,
                     std::string& err);
int save_host_plan(const HostPlan& hp, const char* path, std::string& err);
int load_host_plan(const char* path, HostPlan& hp, std::string& err);

int match_2to4(const int32_t* indptr, const int32_t* indices, int32_t n_rows, int variant,
               int32_t window_size, int32_t dense_threshold, int32_t t_max, tr_match_stats* out,
               std::string& err);

namespace {
thread_local std::string g_error;
}

void set_error(const std::string& msg) { g_error = msg; }
int fail(int code, const std::string& msg) {
  g_error = msg;
  return code;
}
int cuda_fail(cudaError_t e, const char* what) {
  g_error = std::string(what) + ": " + cudaGetErrorString(e);
  return TR_ERR_CUDA;
}

int kernel_smem_limit(const void* kernel, int bytes) {
  static std::mutex mu;
  static std::map<std::pair<int, const void*>, int> set_to;
  int dev = 0;
  TRS_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lock(mu);
  int& have = set_to[std::make_pair(dev, kernel)];
  if (have >= bytes) return TR_OK;
  TRS_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  have = bytes;
  return TR_OK;
}

namespace {

// Device buffer that frees itself.
struct DevBuf {
  void* p = nullptr;
  ~DevBuf() { if (p) cudaFree(p); }
  int alloc(size_t bytes) {
    cudaError_t e = cudaMalloc(&p, bytes > 0 ? bytes : 1);
    return e == cudaSuccess ? TR_OK : cuda_fail(e, "cudaMalloc");
  }
};

struct PlanGuard {
  tr_plan* p = nullptr;
  ~PlanGuard() { if (p) tr_plan_free(p); }
};

// Reads and clears the plan's device error word.
int check_plan_error(const tr_plan* p) {
  int flag = 0;
  TRS_CUDA(cudaMemcpy(&flag, p->view.err, sizeof(int), cudaMemcpyDeviceToHost));
  if (flag != kErrNone) {
    cudaMemset(p->view.err, 0, sizeof(int));
    return fail(TR_ERR_TIMEOUT, "routed kernel: a bounded tensor-core wait gave up");
  }
  return TR_OK;
}

// Times `epoches` launches of the plan after 10 warm-up launches (the
// reference's protocol, mGCNkernel_online.cu:1604-1674), then leaves one
// clean result in d_out.  ms = average per launch.
int timed_routed(const tr_plan* p, const uint16_t* d_b, int32_t k, float* d_out, int mask,
                 int epoches, float* ms) {
  cudaStream_t s;
  TRS_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  int rc = TR_OK;
  for (int i = 0; i < 10 && rc == TR_OK; ++i) rc = launch_routed(p, d_b, k, d_out, TR_OUT_F32, mask, s);
  if (rc == TR_OK) {
    cudaEventRecord(e0, s);
    for (int i = 0; i < epoches && rc == TR_OK; ++i)
      rc = launch_routed(p, d_b, k, d_out, TR_OUT_F32, mask, s);
    cudaEventRecord(e1, s);
  }
  cudaError_t ce = cudaStreamSynchronize(s);
  float t = 0.f;
  if (rc == TR_OK && ce == cudaSuccess) {
    cudaEventElapsedTime(&t, e0, e1);
    *ms = t / (float)epoches;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaStreamDestroy(s);
  if (rc != TR_OK) return rc;
  if (ce != cudaSuccess) return cuda_fail(ce, "routed kernel");
  return check_plan_error(p);
}

// Common tail of the reference-compatible calls: upload B, run the plan
// (timed), copy the FP32 result back.
int run_compat(const HostPlan& hp, const uint16_t* rhs, int64_t n_rhs, int32_t dimN, int32_t mOri,
               int32_t kOri, int32_t epoches, float* out, float* ms_out, bool per_route) {
  if (n_rhs != (int64_t)kOri * dimN) return fail(TR_ERR_ARG, "rhs_matrix must have kOri * dimN elements");
  tr_plan* p = nullptr;
  int rc = plan_upload(hp, &p);
  if (rc) return rc;
  PlanGuard pg{p};
  DevBuf db, dc;
  if ((rc = db.alloc((size_t)n_rhs * 2))) return rc;
  if ((rc = dc.alloc((size_t)mOri * dimN * 4))) return rc;
  TRS_CUDA(cudaMemcpy(db.p, rhs, (size_t)n_rhs * 2, cudaMemcpyHostToDevice));
  TRS_CUDA(cudaMemset(dc.p, 0, (size_t)mOri * dimN * 4));
  float ms[5] = {0, 0, 0, 0, 0};
  if (per_route) {
    if ((rc = timed_routed(p, (uint16_t*)db.p, dimN, (float*)dc.p, TR_ROUTE_TC, epoches, &ms[1]))) return rc;
    if ((rc = timed_routed(p, (uint16_t*)db.p, dimN, (float*)dc.p, TR_ROUTE_CUDA, epoches, &ms[2]))) return rc;
    ms[3] = ms[2];
    if ((rc = timed_routed(p, (uint16_t*)db.p, dimN, (float*)dc.p, TR_ROUTE_SPTC, epoches, &ms[4]))) return rc;
  }
  if ((rc = timed_routed(p, (uint16_t*)db.p, dimN, (float*)dc.p, TR_ROUTE_ALL, epoches, &ms[0]))) return rc;
  TRS_CUDA(cudaMemcpy(out, dc.p, (size_t)mOri * dimN * 4, cudaMemcpyDeviceToHost));
  if (ms_out) std::memcpy(ms_out, ms, sizeof(ms));
  return TR_OK;
}

int check_common(int32_t window, int32_t dimN, int32_t mOri, int32_t kOri, int32_t epoches,
                 int max_window) {
  if (!(window > 0 && window <= max_window))
    return fail(TR_ERR_ARG, "window must be in (0, " + std::to_string(max_window) + "]");
  if (dimN <= 0) return fail(TR_ERR_ARG, "dimN must be positive");
  if (mOri <= 0) return fail(TR_ERR_ARG, "mOri must be positive");
  if (kOri <= 0) return fail(TR_ERR_ARG, "kOri must be positive");
  if (epoches <= 0) return fail(TR_ERR_ARG, "epoches must be positive");
  return TR_OK;
}

}  // namespace
}  // namespace trs

using namespace trs;

struct tr_route {
  RouteTables t;
  // device router: the tables live on the device; a table's host copy in
  // `t` is made on its first tr_route_table call
  std::unique_ptr<DeviceTables> dev;
  std::mutex mu;
  bool fetched[29] = {};
};

struct tr_host_plan {
  HostPlan hp;
};

namespace {
// Host copy of one device table of a tr_route_device route.
template <typename T>
int fetch_table(std::vector<T>& dst, const void* src, int64_t count) {
  dst.resize((size_t)count);
  if (count > 0)
    TRS_CUDA(cudaMemcpy(dst.data(), src, (size_t)count * sizeof(T), cudaMemcpyDeviceToHost));
  return TR_OK;
}
}  // namespace

extern "C" {

const char* tr_last_error(void) { return g_error.c_str(); }
int tr_version(void) { return 1; }

int tr_device_info(int* num_sms, int* cc_major, int* cc_minor) {
  int dev = 0;
  TRS_CUDA(cudaGetDevice(&dev));
  if (num_sms) TRS_CUDA(cudaDeviceGetAttribute(num_sms, cudaDevAttrMultiProcessorCount, dev));
  if (cc_major) TRS_CUDA(cudaDeviceGetAttribute(cc_major, cudaDevAttrComputeCapabilityMajor, dev));
  if (cc_minor) TRS_CUDA(cudaDeviceGetAttribute(cc_minor, cudaDevAttrComputeCapabilityMinor, dev));
  return TR_OK;
}

int tr_route_build(const int32_t* indptr, const int32_t* indices, const float* values,
                   int32_t n_rows, const tr_route_params* params, tr_route** out) {
  if (!indptr || !params || !out) return fail(TR_ERR_ARG, "null argument");
  std::unique_ptr<tr_route> r(new tr_route());
  std::string err;
  const int rc = build_route(indptr, indices, values, n_rows, *params, r->t, err);
  if (rc) return fail(rc, err);
  *out = r.release();
  return TR_OK;
}

int tr_route_device(const int32_t* d_indptr, const int32_t* d_indices, const float* d_values,
                    int32_t n_rows, const tr_route_params* params, tr_route** out) {
  if (!d_indptr || !params || !out) return fail(TR_ERR_ARG, "null argument");
  if (n_rows < 0) return fail(TR_ERR_ARG, "n_rows must be >= 0");
  const tr_route_params& q = *params;
  if (!(q.window > 0 && q.window <= 32 && q.wide > 0 && q.wide <= 32))
    return fail(TR_ERR_ARG, "window and wide must be in (0, 32]");
  if (q.window > 16)
    return fail(TR_ERR_UNSUPPORTED, "window > 16 is not supported (the 2-bit row vector overflows 32 bits)");
  if (q.partsize_t <= 0 || q.partsize_c <= 0 || q.shortsize < 0)
    return fail(TR_ERR_ARG, "partsize_t / partsize_c must be positive and shortsize >= 0");
  if (q.mode != TR_ROUTE_COMPAT && q.mode != TR_ROUTE_EXACT) return fail(TR_ERR_ARG, "bad route mode");
  RouteFullParams gp;
  gp.window = q.window;
  gp.density = q.density;
  gp.tc_min_util = q.tc_min_util;
  gp.partsize_t = q.partsize_t;
  gp.partsize_c = q.partsize_c;
  gp.shortsize = q.shortsize;
  gp.unit_min_nnz = q.unit_min_nnz;
  gp.skip_tc = q.skip_tc;
  gp.skip_sptc = q.skip_sptc;
  gp.mode = q.mode;
  std::unique_ptr<tr_route> r(new tr_route());
  r->dev.reset(new DeviceTables());
  std::string err;
  const int rc = route_full_gpu(d_indptr, d_indices, d_values, n_rows, gp, *r->dev, r->t, err);
  if (rc) return err.empty() ? rc : fail(rc, err);
  // the offset tables were formed on the host
  for (int i : {0, 1, 7, 12, 22, 28}) r->fetched[i] = true;
  *out = r.release();
  return TR_OK;
}

int tr_route_table_device(const tr_route* r, int idx, const void** d_data, int64_t* count) {
  if (!r || !d_data || !count) return fail(TR_ERR_ARG, "null argument");
  if (idx < 0 || idx >= 29) return fail(TR_ERR_ARG, "table index out of range");
  if (!r->dev) return fail(TR_ERR_UNSUPPORTED, "the tables of a host-built route are on the host");
  *d_data = r->dev->ptr[idx];
  *count = r->dev->count[idx];
  return TR_OK;
}

int tr_route_table(const tr_route* r, int idx, const void** data, int64_t* count) {
  if (!r || !data || !count) return fail(TR_ERR_ARG, "null argument");
  if (r->dev && idx >= 0 && idx < 29) {
    tr_route* m = const_cast<tr_route*>(r);
    std::lock_guard<std::mutex> lock(m->mu);
    if (!m->fetched[idx]) {
      RouteTables& H = m->t;
      const void* src = r->dev->ptr[idx];
      const int64_t n = r->dev->count[idx];
      int rc = TR_OK;
#define TRS_F(i, v) case i: rc = fetch_table(H.v, src, n); break;
      switch (idx) {
        TRS_F(2, t_column) TRS_F(3, t_value) TRS_F(4, t_window_row) TRS_F(5, t_atomic)
        TRS_F(6, t_binary) TRS_F(8, c_row) TRS_F(9, c_atomic) TRS_F(10, c_column)
        TRS_F(11, c_value) TRS_F(13, cs_row) TRS_F(14, cs_atomic) TRS_F(15, cs_column)
        TRS_F(16, cs_value) TRS_F(17, s_column) TRS_F(18, s_mask) TRS_F(19, s_value)
        TRS_F(20, s_pos) TRS_F(21, s_window) TRS_F(23, s_tile_window) TRS_F(24, s_tile_group)
        TRS_F(25, s_tile_column) TRS_F(26, s_packed_a) TRS_F(27, s_packed_meta)
        default: break;
      }
#undef TRS_F
      if (rc) return rc;
      m->fetched[idx] = true;
    }
  }
  const RouteTables& T = r->t;
#define TRS_T(i, v) case i: *data = T.v.data(); *count = (int64_t)T.v.size(); return TR_OK;
  switch (idx) {
    TRS_T(0, t_row_offset) TRS_T(1, t_block_offset) TRS_T(2, t_column) TRS_T(3, t_value)
    TRS_T(4, t_window_row) TRS_T(5, t_atomic) TRS_T(6, t_binary)
    TRS_T(7, c_row_offset) TRS_T(8, c_row) TRS_T(9, c_atomic) TRS_T(10, c_column) TRS_T(11, c_value)
    TRS_T(12, cs_row_offset) TRS_T(13, cs_row) TRS_T(14, cs_atomic) TRS_T(15, cs_column)
    TRS_T(16, cs_value) TRS_T(17, s_column) TRS_T(18, s_mask) TRS_T(19, s_value) TRS_T(20, s_pos)
    TRS_T(21, s_window) TRS_T(22, s_offsets) TRS_T(23, s_tile_window) TRS_T(24, s_tile_group)
    TRS_T(25, s_tile_column) TRS_T(26, s_packed_a) TRS_T(27, s_packed_meta)
    TRS_T(28, s_window_tile_offset)
    default: return fail(TR_ERR_ARG, "table index out of range");
  }
#undef TRS_T
}

int tr_route_tc_device(const int32_t* d_indptr, const int32_t* d_indices, const float* d_values,
                       int32_t n_rows, const tr_route_params* params, tr_route** out) {
  if (!d_indptr || !params || !out) return fail(TR_ERR_ARG, "null argument");
  if (n_rows < 0) return fail(TR_ERR_ARG, "negative row count");
  if (params->window != 16) return fail(TR_ERR_UNSUPPORTED, "the device router uses 16-row windows");
  RouteGpuParams gp;
  gp.window = 16;
  gp.density = params->density;
  gp.tc_min_util = params->tc_min_util;
  gp.partsize_t = params->partsize_t;
  gp.skip_tc = params->skip_tc;
  TcTables tc;
  std::string err;
  const auto t0 = std::chrono::high_resolution_clock::now();
  int rc = route_tc_gpu(d_indptr, d_indices, d_values, n_rows, gp, tc, err);
  if (rc) return err.empty() ? rc : fail(rc, err);
  std::unique_ptr<tr_route> r(new tr_route());
  r->t.t_row_offset = std::move(tc.t_row_offset);
  r->t.t_block_offset = std::move(tc.t_block_offset);
  r->t.t_column = std::move(tc.t_column);
  r->t.t_value = std::move(tc.t_value);
  r->t.t_window_row = std::move(tc.t_window_row);
  r->t.t_binary = std::move(tc.t_binary);
  r->t.t_edge = std::move(tc.t_edge);
  r->t.seconds = std::chrono::duration<double>(std::chrono::high_resolution_clock::now() - t0).count();
  *out = r.release();
  return TR_OK;
}

int tr_route_tc_device_noalloc(const int32_t* d_indptr, const int32_t* d_indices,
                               const float* d_values, int32_t n_rows,
                               const tr_route_params* params, int32_t* t_column,
                               int64_t* t_binary, float* t_value, int32_t* t_block_offset,
                               int64_t cap_sub, int64_t cap_val, int64_t* n_sub_out,
                               int64_t* n_val_out, void* stream) {
  if (!d_indptr || !params) return fail(TR_ERR_ARG, "null argument");
  if (params->window != 16) return fail(TR_ERR_UNSUPPORTED, "the device router uses 16-row windows");
  if (cap_sub > 0 && (!t_column || !t_binary || !t_block_offset))
    return fail(TR_ERR_ARG, "null table buffer with a non-zero sub-block capacity");
  if (cap_val > 0 && !t_value) return fail(TR_ERR_ARG, "null value buffer with a non-zero capacity");
  RouteGpuParams gp;
  gp.window = 16;
  gp.density = params->density;
  gp.tc_min_util = params->tc_min_util;
  gp.partsize_t = params->partsize_t;
  gp.skip_tc = params->skip_tc;
  return route_tc_gpu_noalloc(d_indptr, d_indices, d_values, n_rows, gp, t_column, t_binary,
                              t_value, t_block_offset, cap_sub, cap_val, n_sub_out, n_val_out,
                              (cudaStream_t)stream);
}

int tr_match_2to4(const int32_t* indptr, const int32_t* indices, int32_t n_rows, int variant,
                  int32_t window_size, int32_t dense_threshold, int32_t t_max,
                  tr_match_stats* out) {
  if (!indptr || !out || (n_rows > 0 && indptr[n_rows] > 0 && !indices))
    return fail(TR_ERR_ARG, "null argument");
  std::string err;
  const int rc = match_2to4(indptr, indices, n_rows, variant, window_size, dense_threshold, t_max,
                            out, err);
  return rc ? fail(rc, err) : TR_OK;
}

int tr_match_2to4_online(const int32_t* indptr, const int32_t* indices, int32_t n_rows,
                         int32_t window_size, int32_t dense_threshold, int32_t t_max,
                         tr_match_stats* out) {
  if (!indptr || !out || (n_rows > 0 && indptr[n_rows] > 0 && !indices))
    return fail(TR_ERR_ARG, "null argument");
  if (window_size != 16) return fail(TR_ERR_ARG, "the online matcher uses 16-row windows");
  std::string err;
  const int rc = match_online_gpu(indptr, indices, n_rows, dense_threshold, t_max, out, err);
  return rc ? fail(rc, err) : TR_OK;
}

int tr_tca_order(const int32_t* indptr, const int32_t* indices, int32_t n_rows,
                 const tr_tca_params* params, int32_t* order, tr_tca_stats* stats) {
  if (!indptr || (n_rows > 0 && !order)) return fail(TR_ERR_ARG, "null argument");
  if (n_rows < 0) return fail(TR_ERR_ARG, "negative row count");
  if (indptr[0] != 0) return fail(TR_ERR_ARG, "indptr must start at 0");
  for (int32_t r = 0; r < n_rows; ++r)
    if (indptr[r + 1] < indptr[r]) return fail(TR_ERR_ARG, "indptr must be non-decreasing");
  const int64_t nnz = indptr[n_rows];
  if (nnz > 0 && !indices) return fail(TR_ERR_ARG, "null indices");
  for (int64_t e = 0; e < nnz; ++e)
    if (indices[e] < 0) return fail(TR_ERR_ARG, "column indices must be >= 0");
  TcaParams p;
  if (params) {
    p.thres = params->thres;
    p.cluster_thres = params->cluster_thres;
    p.lsh_threshold = params->lsh_threshold;
    p.seed = params->seed;
    p.max_pairs = params->max_pairs;
    p.device = params->device;
  }
  std::vector<int32_t> ord;
  TcaStats st;
  std::string err;
  const int rc = tca_order(indptr, indices, n_rows, p, ord, st, err);
  if (rc) return fail(rc, err);
  std::copy(ord.begin(), ord.end(), order);
  if (stats) {
    stats->bands = st.bands;
    stats->rows_per_band = st.rows_per_band;
    stats->pairs1 = st.pairs1;
    stats->clusters1 = st.clusters1;
    stats->pairs2 = st.pairs2;
    stats->clusters2 = st.clusters2;
    for (int i = 0; i < 4; ++i) stats->seconds[i] = st.seconds[i];
  }
  return TR_OK;
}

int tr_lsh_params(double threshold, int32_t num_perm, int32_t* bands, int32_t* rows) {
  if (!bands || !rows) return fail(TR_ERR_ARG, "null argument");
  if (!(threshold > 0.0 && threshold < 1.0)) return fail(TR_ERR_ARG, "threshold must be in (0, 1)");
  if (num_perm < 1 || num_perm > 1024) return fail(TR_ERR_ARG, "num_perm must be in [1, 1024]");
  int b = 0, r = 0;
  tca_lsh_params(threshold, num_perm, b, r);
  *bands = b;
  *rows = r;
  return TR_OK;
}

int tr_host_plan_save(const tr_host_plan* h, const char* path) {
  if (!h || !path) return fail(TR_ERR_ARG, "null argument");
  std::string err;
  const int rc = save_host_plan(h->hp, path, err);
  return rc ? fail(rc, err) : TR_OK;
}

int tr_host_plan_load(const char* path, tr_host_plan** out) {
  if (!path || !out) return fail(TR_ERR_ARG, "null argument");
  std::unique_ptr<tr_host_plan> h(new tr_host_plan());
  std::string err;
  const int rc = load_host_plan(path, h->hp, err);
  if (rc) return fail(rc, err);
  *out = h.release();
  return TR_OK;
}

double tr_route_seconds(const tr_route* r) { return r ? r->t.seconds : 0.0; }
void tr_route_free(tr_route* r) { delete r; }

int tr_plan_from_tables(const tr_tables* t, int32_t n_rows, int32_t n_cols, int32_t window,
                        tr_plan** out) {
  if (!t || !out) return fail(TR_ERR_ARG, "null argument");
  HostPlan hp;
  std::string err;
  int rc = plan_from_tables(*t, n_rows, n_cols, window, hp, err);
  if (rc) return fail(rc, err);
  return plan_upload(hp, out);
}

int tr_plan_from_csr(const int32_t* indptr, const int32_t* indices, const float* values,
                     int32_t n_rows, int32_t n_cols, const tr_route_params* params,
                     tr_plan** out) {
  tr_plan_opts opts{};
  return tr_plan_build(indptr, indices, values, n_rows, n_cols, params, &opts, out);
}

int tr_plan_build(const int32_t* indptr, const int32_t* indices, const float* values,
                  int32_t n_rows, int32_t n_cols, const tr_route_params* params,
                  const tr_plan_opts* opts, tr_plan** out) {
  if (!indptr || !params || !opts || !out) return fail(TR_ERR_ARG, "null argument");
  HostPlan hp;
  std::string err;
  const int rc = build_plan(indptr, indices, values, n_rows, n_cols, *params, *opts, hp, err);
  if (rc) return fail(rc, err);
  return plan_upload(hp, out);
}

int tr_label_order(const int32_t* indptr, const int32_t* indices, int32_t n_rows, int32_t n_cols,
                   int32_t transpose, int32_t* order) {
  if (!indptr || !order) return fail(TR_ERR_ARG, "null argument");
  std::string err;
  const int rc = label_order(indptr, indices, n_rows, n_cols, transpose != 0, order, err);
  if (rc) return fail(rc, err);
  return TR_OK;
}

int tr_plan_build_host(const int32_t* indptr, const int32_t* indices, const float* values,
                       int32_t n_rows, int32_t n_cols, const tr_route_params* params,
                       const tr_plan_opts* opts, tr_host_plan** out) {
  if (!indptr || !params || !opts || !out) return fail(TR_ERR_ARG, "null argument");
  std::unique_ptr<tr_host_plan> h(new tr_host_plan());
  std::string err;
  const int rc = build_plan(indptr, indices, values, n_rows, n_cols, *params, *opts, h->hp, err);
  if (rc) return fail(rc, err);
  *out = h.release();
  return TR_OK;
}

int tr_host_plan_array(const tr_host_plan* h, int idx, const void** data, int64_t* count) {
  if (!h || !data || !count) return fail(TR_ERR_ARG, "null argument");
  const HostPlan& P = h->hp;
#define TRS_A(i, v) case i: *data = P.v.data(); *count = (int64_t)P.v.size(); return TR_OK;
  switch (idx) {
    TRS_A(0, win_tile) TRS_A(1, win_split) TRS_A(2, win_prom) TRS_A(3, tile_col)
    TRS_A(4, tile_a) TRS_A(5, res_ptr) TRS_A(6, res_col) TRS_A(7, res_val) TRS_A(8, win_order)
    TRS_A(9, row_scale) TRS_A(10, row_out) TRS_A(11, val_slot) TRS_A(12, edge_row)
    TRS_A(13, res_edge) TRS_A(14, blk_chunk) TRS_A(15, chunk_col) TRS_A(16, chunk_ent)
    TRS_A(17, ent_pos) TRS_A(18, ent_val) TRS_A(19, ent_src) TRS_A(20, blk_order)
    default: return fail(TR_ERR_ARG, "plan array index out of range");
  }
#undef TRS_A
}

int tr_host_plan_upload(const tr_host_plan* h, tr_plan** out) {
  if (!h || !out) return fail(TR_ERR_ARG, "null argument");
  return plan_upload(h->hp, out);
}

void tr_host_plan_free(tr_host_plan* h) { delete h; }

int tr_plan_info_get(const tr_plan* p, tr_plan_info* info) {
  if (!p || !info) return fail(TR_ERR_ARG, "null argument");
  *info = p->info;
  return TR_OK;
}

void tr_plan_free(tr_plan* p) {
  if (!p) return;
  if (p->block) cudaFree(p->block);
  if (p->edge_id) cudaFree(p->edge_id);
  delete p;
}

int tr_spmm_csr(const int32_t* indptr, const int32_t* indices, const uint16_t* values, int32_t m,
                int32_t n_cols, int64_t nnz, const uint16_t* b, int32_t k, void* c, int c_dtype,
                void* stream) {
  if (m < 0 || k < 0 || n_cols < 0 || nnz < 0) return fail(TR_ERR_ARG, "negative size");
  if (c_dtype != TR_OUT_F32 && c_dtype != TR_OUT_F16) return fail(TR_ERR_ARG, "bad output dtype");
  if (m > 0 && k > 0 && (!indptr || !b || !c || (nnz > 0 && (!indices || !values))))
    return fail(TR_ERR_ARG, "null device pointer");
  return launch_csr(indptr, indices, values, m, b, k, c, c_dtype, (cudaStream_t)stream);
}

int tr_spmm_routed(const tr_plan* p, const uint16_t* b, int32_t k, void* c, int c_dtype,
                   int route_mask, void* stream) {
  if (!p) return fail(TR_ERR_ARG, "null plan");
  if (k < 0) return fail(TR_ERR_ARG, "negative K");
  if (c_dtype != TR_OUT_F32 && c_dtype != TR_OUT_F16) return fail(TR_ERR_ARG, "bad output dtype");
  if (p->view.n_rows > 0 && k > 0 && (!b || !c)) return fail(TR_ERR_ARG, "null device pointer");
  if (p->blocked) {
    if ((route_mask & TR_ROUTE_ALL) == 0) {
      if (p->view.n_rows > 0 && k > 0)
        TRS_CUDA(cudaMemsetAsync(c, 0, (size_t)p->view.n_rows * k * (c_dtype == TR_OUT_F16 ? 2 : 4),
                                 (cudaStream_t)stream));
      return TR_OK;
    }
    return launch_block(p, b, k, c, c_dtype, (route_mask & TR_ROUTE_PER_WINDOW) != 0,
                        (cudaStream_t)stream);
  }
  return launch_routed(p, b, k, c, c_dtype,
                       route_mask & (TR_ROUTE_ALL | TR_ROUTE_PER_WINDOW | TR_ROUTE_PIPELINED |
                                     TR_ROUTE_RESIDUAL_PASS),
                       (cudaStream_t)stream);
}

int tr_spmm_routed_f32(const tr_plan* p, const float* b, int32_t k, void* c, int c_dtype,
                       int route_mask, void* stream) {
  if (!p) return fail(TR_ERR_ARG, "null plan");
  if (k < 0) return fail(TR_ERR_ARG, "negative K");
  if (c_dtype != TR_OUT_F32 && c_dtype != TR_OUT_F16) return fail(TR_ERR_ARG, "bad output dtype");
  if (p->view.n_rows > 0 && k > 0 && (!b || !c)) return fail(TR_ERR_ARG, "null device pointer");
  if (p->blocked) {
    if ((route_mask & TR_ROUTE_ALL) == 0) {
      if (p->view.n_rows > 0 && k > 0)
        TRS_CUDA(cudaMemsetAsync(c, 0, (size_t)p->view.n_rows * k * (c_dtype == TR_OUT_F16 ? 2 : 4),
                                 (cudaStream_t)stream));
      return TR_OK;
    }
    return launch_block_f32(p, b, k, c, c_dtype, (cudaStream_t)stream);
  }
  return launch_routed_f32(p, b, k, c, c_dtype, route_mask & TR_ROUTE_ALL, (cudaStream_t)stream);
}

int tr_sddmm_csr_f32(const int32_t* indptr, const int32_t* indices, int32_t m, int32_t n_cols,
                     int64_t nnz, const float* x, const float* y, int32_t k, float* out,
                     void* stream) {
  if (m < 0 || n_cols < 0 || nnz < 0 || k < 0) return fail(TR_ERR_ARG, "negative size");
  if (nnz > 0 && (!indptr || !indices || !out || (k > 0 && (!x || !y))))
    return fail(TR_ERR_ARG, "null device pointer");
  return launch_sddmm_f32(indptr, indices, m, nnz, x, y, k, out, (cudaStream_t)stream);
}

int tr_plan_set_values(tr_plan* p, const float* values, int64_t n_edges, void* stream) {
  if (!p) return fail(TR_ERR_ARG, "null plan");
  if (n_edges != p->n_edges)
    return fail(TR_ERR_ARG, "value count " + std::to_string(n_edges) + " != plan entries " +
                                std::to_string(p->n_edges));
  if (n_edges > 0 && !values) return fail(TR_ERR_ARG, "null device pointer");
  return launch_set_values(p, values, (cudaStream_t)stream);
}

int tr_plan_set_k_tile(tr_plan* p, int32_t k_tile) {
  if (!p) return fail(TR_ERR_ARG, "null plan");
  if (k_tile != 0 && (k_tile < 64 || k_tile > 256 || k_tile % 64 != 0))
    return fail(TR_ERR_ARG, "k_tile must be 0, 64, 128, 192 or 256");
  p->k_tile = k_tile;
  return TR_OK;
}

int tr_plan_set_deterministic(tr_plan* p, int32_t on) {
  if (!p) return fail(TR_ERR_ARG, "null plan");
  p->deterministic = on != 0;
  return TR_OK;
}

int tr_plan_entry_order(const tr_plan* p, int32_t* order, void* stream) {
  if (!p) return fail(TR_ERR_ARG, "null plan");
  if (p->n_edges > 0 && !order) return fail(TR_ERR_ARG, "null device pointer");
  return launch_entry_order(p, order, (cudaStream_t)stream);
}

int tr_plan_renumber_edges(tr_plan* p, const int32_t* new_id, int64_t n_edges, void* stream) {
  if (!p) return fail(TR_ERR_ARG, "null plan");
  if (n_edges != p->n_edges) return fail(TR_ERR_ARG, "n_edges must equal the plan's edge count");
  if (n_edges > 0 && !new_id) return fail(TR_ERR_ARG, "null device pointer");
  return launch_renumber_edges(p, new_id, (cudaStream_t)stream);
}

int tr_adjoint_sddmm(const tr_plan* adj, const int32_t* a_indptr, const int32_t* a_indices,
                     int32_t a_rows, int64_t nnz, const uint16_t* dc, const uint16_t* b, int32_t k,
                     void* db, int db_dtype, float* dval, void* stream) {
  if (!adj) return fail(TR_ERR_ARG, "null plan");
  if (a_rows < 0 || nnz < 0 || k < 0) return fail(TR_ERR_ARG, "negative size");
  if (db_dtype != TR_OUT_F32 && db_dtype != TR_OUT_F16) return fail(TR_ERR_ARG, "bad output dtype");
  if (a_rows != adj->view.n_cols) return fail(TR_ERR_ARG, "a_rows must equal the adjoint plan's column count");
  if (k > 0 && (!dc || !b || !db || (nnz > 0 && (!a_indptr || !a_indices || !dval))))
    return fail(TR_ERR_ARG, "null device pointer");
  if (adj->blocked) {
    if (block_bwd_supported(adj, k, dc, b, db, dval) && nnz == adj->n_edges)
      return launch_block_bwd(adj, dc, b, k, db, db_dtype, dval, (cudaStream_t)stream);
    int rc = launch_block(adj, dc, k, db, db_dtype, false, (cudaStream_t)stream);
    if (rc) return rc;
    return launch_sddmm(a_indptr, a_indices, a_rows, nnz, dc, b, k, dval, (cudaStream_t)stream,
                        adj->edge_id);
  }
  return launch_adjoint_sddmm(adj, a_indptr, a_indices, a_rows, nnz, dc, b, k, db, db_dtype, dval,
                              (cudaStream_t)stream);
}

int tr_adjoint_sddmm_f32(const tr_plan* adj, const int32_t* a_indptr, const int32_t* a_indices,
                         int32_t a_rows, int64_t nnz, const float* dc, const float* b, int32_t k,
                         void* db, int db_dtype, float* dval, void* stream) {
  if (!adj) return fail(TR_ERR_ARG, "null plan");
  if (a_rows < 0 || nnz < 0 || k < 0) return fail(TR_ERR_ARG, "negative size");
  if (db_dtype != TR_OUT_F32 && db_dtype != TR_OUT_F16) return fail(TR_ERR_ARG, "bad output dtype");
  if (a_rows != adj->view.n_cols) return fail(TR_ERR_ARG, "a_rows must equal the adjoint plan's column count");
  if (k > 0 && (!dc || !b || !db || (nnz > 0 && (!a_indptr || !a_indices || !dval))))
    return fail(TR_ERR_ARG, "null device pointer");
  if (adj->blocked) {
    int rc = launch_block_f32(adj, dc, k, db, db_dtype, (cudaStream_t)stream);
    if (rc) return rc;
    return launch_sddmm_f32(a_indptr, a_indices, a_rows, nnz, dc, b, k, dval, (cudaStream_t)stream,
                            adj->edge_id);
  }
  return launch_adjoint_sddmm_f32(adj, a_indptr, a_indices, a_rows, nnz, dc, b, k, db, db_dtype,
                                  dval, (cudaStream_t)stream);
}

int tr_sddmm_csr(const int32_t* indptr, const int32_t* indices, int32_t m, int32_t n_cols,
                 int64_t nnz, const uint16_t* x, const uint16_t* y, int32_t k, float* out,
                 void* stream) {
  if (m < 0 || n_cols < 0 || nnz < 0 || k < 0) return fail(TR_ERR_ARG, "negative size");
  if (nnz > 0 && (!indptr || !indices || !out || (k > 0 && (!x || !y))))
    return fail(TR_ERR_ARG, "null device pointer");
  return launch_sddmm(indptr, indices, m, nnz, x, y, k, out, (cudaStream_t)stream);
}

int tr_forward_fp16_tcu_cuda_sptc_mma_parallel_online(
    const int32_t* t_row_offset, int64_t n_t_row_offset, const int32_t* t_block_offset,
    int64_t n_t_block_offset, const int32_t* t_column, int64_t n_t_column, const uint16_t* t_value,
    int64_t n_t_value, const int32_t* t_window_row, int64_t n_t_window_row, const int32_t* t_atomic,
    int64_t n_t_atomic, const int64_t* t_binary, int64_t n_t_binary, const int32_t* c_row_offset,
    int64_t n_c_row_offset, const int32_t* c_row, int64_t n_c_row, const int32_t* c_atomic,
    int64_t n_c_atomic, const int32_t* c_column, int64_t n_c_column, const uint16_t* c_value,
    int64_t n_c_value, const int32_t* c_row_offset_short, int64_t n_c_row_offset_short,
    const int32_t* c_row_short, int64_t n_c_row_short, const int32_t* c_atomic_short,
    int64_t n_c_atomic_short, const int32_t* c_column_short, int64_t n_c_column_short,
    const uint16_t* c_value_short, int64_t n_c_value_short, const int32_t* s_column,
    int64_t n_s_column, const float* s_value, int64_t n_s_value, const int8_t* s_pos,
    int64_t n_s_pos, const int32_t* s_offsets, int64_t n_s_offsets, const int32_t* s_tile_window,
    int64_t n_s_tile_window, const int32_t* s_tile_column, int64_t n_s_tile_column,
    const int32_t* s_packed_a, int64_t n_s_packed_a, const int32_t* s_packed_meta,
    int64_t n_s_packed_meta, const int32_t* s_window_tile_offset, int64_t n_s_window_tile_offset,
    const uint16_t* rhs_matrix, int64_t n_rhs_matrix, int32_t parts_t, int32_t parts_c,
    int32_t partsize_c, int32_t parts_c_short, int32_t window, int32_t dimN, int32_t mOri,
    int32_t kOri, int32_t epoches, float* out, float* ms_out) {
  (void)t_atomic; (void)n_t_atomic; (void)c_atomic; (void)n_c_atomic; (void)c_atomic_short;
  (void)n_c_atomic_short; (void)partsize_c; (void)s_value; (void)n_s_value; (void)s_pos; (void)n_s_pos;
  int rc = check_common(window, dimN, mOri, kOri, epoches, 16);
  if (rc) return rc;
  // shape checks of mGCN_online.cpp:866-932
  if (n_s_column % 4) return fail(TR_ERR_ARG, "s_column must have shape [groups, 4]");
  if (n_s_offsets < 1) return fail(TR_ERR_ARG, "s_offsets must be 1-D with at least one item");
  const int64_t groups = n_s_column / 4;
  if (s_offsets[0] != 0) return fail(TR_ERR_ARG, "s_offsets must start with 0");
  if (s_offsets[n_s_offsets - 1] != groups)
    return fail(TR_ERR_ARG, "s_offsets end must equal group count");
  int64_t tiles = 0;
  for (int64_t w = 0; w + 1 < n_s_offsets; ++w) {
    const int64_t gc = s_offsets[w + 1] - s_offsets[w];
    if (gc < 0) return fail(TR_ERR_ARG, "s_offsets must be non-decreasing");
    tiles += (gc + 3) / 4;
  }
  if (n_s_tile_column != n_s_tile_window * 16) return fail(TR_ERR_ARG, "s_tile_column tile count mismatch");
  if (n_s_packed_a != n_s_tile_window * 64) return fail(TR_ERR_ARG, "s_packed_a tile count mismatch");
  if (n_s_packed_meta != n_s_tile_window * 8) return fail(TR_ERR_ARG, "s_packed_meta tile count mismatch");
  if (tiles != n_s_tile_window) return fail(TR_ERR_ARG, "packed tile count must match offsets-derived tile count");
  if (parts_t != n_t_row_offset - 1 && !(parts_t == 0 && n_t_row_offset <= 1))
    return fail(TR_ERR_ARG, "parts_t does not match t_row_offset");
  if (parts_c != n_c_row_offset - 1 && !(parts_c == 0 && n_c_row_offset <= 1))
    return fail(TR_ERR_ARG, "parts_c does not match c_row_offset");
  if (parts_c_short != n_c_row_offset_short - 1 && !(parts_c_short == 0 && n_c_row_offset_short <= 1))
    return fail(TR_ERR_ARG, "parts_c_short does not match c_row_offset_short");
  if (window != 16) return fail(TR_ERR_UNSUPPORTED, "the routed tables assume 16-row windows");
  tr_tables tt{};
  tt.t_row_offset = t_row_offset; tt.n_t_row_offset = n_t_row_offset;
  tt.t_block_offset = t_block_offset; tt.n_t_block_offset = n_t_block_offset;
  tt.t_column = t_column; tt.n_t_column = n_t_column;
  tt.t_value = t_value; tt.n_t_value = n_t_value;
  tt.t_window_row = t_window_row; tt.n_t_window_row = n_t_window_row;
  tt.t_binary = t_binary; tt.n_t_binary = n_t_binary;
  tt.c_row_offset = c_row_offset; tt.n_c_row_offset = n_c_row_offset;
  tt.c_row = c_row; tt.n_c_row = n_c_row;
  tt.c_column = c_column; tt.n_c_column = n_c_column;
  tt.c_value = c_value; tt.n_c_value = n_c_value;
  tt.cs_row_offset = c_row_offset_short; tt.n_cs_row_offset = n_c_row_offset_short;
  tt.cs_row = c_row_short; tt.n_cs_row = n_c_row_short;
  tt.cs_column = c_column_short; tt.n_cs_column = n_c_column_short;
  tt.cs_value = c_value_short; tt.n_cs_value = n_c_value_short;
  tt.s_tile_column = s_tile_column; tt.n_s_tile_column = n_s_tile_column;
  tt.s_packed_a = reinterpret_cast<const uint32_t*>(s_packed_a); tt.n_s_packed_a = n_s_packed_a;
  tt.s_packed_meta = reinterpret_cast<const uint32_t*>(s_packed_meta); tt.n_s_packed_meta = n_s_packed_meta;
  tt.s_window_tile_offset = s_window_tile_offset; tt.n_s_window_tile_offset = n_s_window_tile_offset;
  HostPlan hp;
  std::string err;
  rc = plan_from_tables(tt, mOri, kOri, window, hp, err);
  if (rc) return fail(rc, err);
  return run_compat(hp, rhs_matrix, n_rhs_matrix, dimN, mOri, kOri, epoches, out, ms_out, true);
}

int tr_forward_fp16_sptc_online(const int32_t* s_column, int64_t n_s_column, const float* s_value,
                                int64_t n_s_value, const int8_t* s_pos, int64_t n_s_pos,
                                const int32_t* s_window, int64_t n_s_window,
                                const uint16_t* rhs_matrix, int64_t n_rhs_matrix, int32_t window,
                                int32_t dimN, int32_t mOri, int32_t kOri, int32_t epoches,
                                float* out, float* ms_out) {
  int rc = check_common(window, dimN, mOri, kOri, epoches, 1 << 30);
  if (rc) return rc;
  const int64_t groups = n_s_window;
  if (n_s_column != groups * 4) return fail(TR_ERR_ARG, "s_column group count mismatch");
  if (n_s_value != groups * window * 2) return fail(TR_ERR_ARG, "s_value group count mismatch");
  if (n_s_pos != groups * window * 2) return fail(TR_ERR_ARG, "s_pos group count mismatch");
  if (window != 16) return fail(TR_ERR_UNSUPPORTED, "the routed kernels need 16-row windows");
  HostPlan hp;
  std::string err;
  rc = plan_from_groups(s_column, s_value, s_pos, groups, s_window, nullptr, 0, window, mOri, kOri,
                        hp, err);
  if (rc) return fail(rc, err);
  float ms[5];
  rc = run_compat(hp, rhs_matrix, n_rhs_matrix, dimN, mOri, kOri, epoches, out, ms, false);
  if (rc == TR_OK && ms_out) ms_out[0] = ms[0];
  return rc;
}

int tr_forward_fp16_sptc_mma_online(const int32_t* s_column, int64_t n_s_column,
                                    const float* s_value, int64_t n_s_value, const int8_t* s_pos,
                                    int64_t n_s_pos, const int32_t* s_offsets, int64_t n_s_offsets,
                                    const uint16_t* rhs_matrix, int64_t n_rhs_matrix,
                                    int32_t window, int32_t dimN, int32_t mOri, int32_t kOri,
                                    int32_t epoches, float* out, float* ms_out) {
  int rc = check_common(window, dimN, mOri, kOri, epoches, 16);
  if (rc) return rc;
  const int64_t groups = n_s_column / 4;
  if (n_s_column % 4) return fail(TR_ERR_ARG, "s_column must have shape [groups, 4]");
  if (n_s_value != groups * window * 2) return fail(TR_ERR_ARG, "s_value group count mismatch");
  if (n_s_pos != groups * window * 2) return fail(TR_ERR_ARG, "s_pos group count mismatch");
  if (window != 16) return fail(TR_ERR_UNSUPPORTED, "the routed kernels need 16-row windows");
  HostPlan hp;
  std::string err;
  rc = plan_from_groups(s_column, s_value, s_pos, groups, nullptr, s_offsets, n_s_offsets, window,
                        mOri, kOri, hp, err);
  if (rc) return fail(rc, err);
  float ms[5];
  rc = run_compat(hp, rhs_matrix, n_rhs_matrix, dimN, mOri, kOri, epoches, out, ms, false);
  if (rc == TR_OK && ms_out) ms_out[0] = ms[0];
  return rc;
}

int tr_forward_fp16_sptc_mma_packed_online(const int32_t* s_tile_column, int64_t n_s_tile_column,
                                           const int32_t* s_packed_a, int64_t n_s_packed_a,
                                           const int32_t* s_packed_meta, int64_t n_s_packed_meta,
                                           const int32_t* s_window_tile_offset,
                                           int64_t n_s_window_tile_offset,
                                           const uint16_t* rhs_matrix, int64_t n_rhs_matrix,
                                           int32_t window, int32_t dimN, int32_t mOri,
                                           int32_t kOri, int32_t epoches, float* out,
                                           float* ms_out) {
  int rc = check_common(window, dimN, mOri, kOri, epoches, 16);
  if (rc) return rc;
  if (n_s_tile_column % 16) return fail(TR_ERR_ARG, "s_tile_column must have shape [tiles, 16]");
  const int64_t tiles = n_s_tile_column / 16;
  if (n_s_packed_a != tiles * 64) return fail(TR_ERR_ARG, "s_packed_a tile count mismatch");
  if (n_s_packed_meta != tiles * 8) return fail(TR_ERR_ARG, "s_packed_meta tile count mismatch");
  if (n_s_window_tile_offset < 2)
    return fail(TR_ERR_ARG, "s_window_tile_offset must be 1-D with at least 2 elements");
  if (window != 16) return fail(TR_ERR_UNSUPPORTED, "the routed kernels need 16-row windows");
  tr_tables tt{};
  tt.s_tile_column = s_tile_column; tt.n_s_tile_column = n_s_tile_column;
  tt.s_packed_a = reinterpret_cast<const uint32_t*>(s_packed_a); tt.n_s_packed_a = n_s_packed_a;
  tt.s_packed_meta = reinterpret_cast<const uint32_t*>(s_packed_meta); tt.n_s_packed_meta = n_s_packed_meta;
  tt.s_window_tile_offset = s_window_tile_offset; tt.n_s_window_tile_offset = n_s_window_tile_offset;
  HostPlan hp;
  std::string err;
  rc = plan_from_tables(tt, mOri, kOri, window, hp, err);
  if (rc) return fail(rc, err);
  float ms[5];
  rc = run_compat(hp, rhs_matrix, n_rhs_matrix, dimN, mOri, kOri, epoches, out, ms, false);
  if (rc == TR_OK && ms_out) ms_out[0] = ms[0];
  return rc;
}

}  // extern "C"
