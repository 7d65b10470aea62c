/*
 * trspmm.h — C ABI of the B200-native routed FP16 SpMM library (libtrspmm.so).
 *
 * C = A·B with A a sparse adjacency in CSR (int32 indices), B a dense
 * row-major FP16 feature matrix (n_cols x K), FP32 accumulation.
 *
 * Conventions
 *  - Every entry point returns an int status (TR_OK == 0); on failure
 *    tr_last_error() returns a message for the calling thread.  Nothing
 *    aborts the process and no device-side trap is used.
 *  - "host" pointers are CPU memory; "device" pointers are CUDA device
 *    memory of the current device.  `stream` is a cudaStream_t (NULL = the
 *    legacy default stream).
 *  - FP16 data is passed as uint16_t bit patterns (IEEE binary16).
 *  - Device entry points never synchronise the stream and never allocate,
 *    except where noted (plan construction, the reference-compatible host
 *    entry points).
 */
#ifndef TRSPMM_H
#define TRSPMM_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  TR_OK = 0,
  TR_ERR_ARG = 1,          /* invalid argument / malformed CSR or tables */
  TR_ERR_CUDA = 2,         /* CUDA runtime error */
  TR_ERR_TIMEOUT = 3,      /* a bounded device wait gave up (kernel returned early) */
  TR_ERR_NOMEM = 4,
  TR_ERR_UNSUPPORTED = 5   /* shape/alignment outside what the kernels implement */
};

enum { TR_OUT_F32 = 0, TR_OUT_F16 = 1 };

/* Route-mask bits for tr_spmm_routed (all set = full product).
 * The full product (K % 8 == 0) runs the CUDA-core residual as one kernel
 * over every window, then adds the tensor-core tiles (the persistent
 * pipelined kernel where K % 64 == 0, K <= 256 and at most 512 windows per
 * SM, else the per-window kernel in accumulate mode).  A partial mask, or
 * TR_ROUTE_PER_WINDOW, runs the single fused one-CTA-per-window kernel (per-
 * route timing).  TR_ROUTE_PIPELINED with TR_ROUTE_ALL runs the single
 * pipelined kernel (residual added in its epilogue).  TR_ROUTE_RESIDUAL_PASS
 * with TR_ROUTE_ALL runs only the first launch of the full product (C = the
 * residual part), for timing and profiling that kernel alone. */
enum { TR_ROUTE_TC = 1, TR_ROUTE_SPTC = 2, TR_ROUTE_CUDA = 4, TR_ROUTE_ALL = 7,
       TR_ROUTE_PER_WINDOW = 8, TR_ROUTE_PIPELINED = 16, TR_ROUTE_RESIDUAL_PASS = 32 };

const char* tr_last_error(void);
int tr_version(void);
/* Number of SMs and whether the tcgen05 path can run on the current device. */
int tr_device_info(int* num_sms, int* cc_major, int* cc_minor);

/* ------------------------------------------------------------------------
 * Router: three-stage funnel (dense TC columns, 2:4 SPTC groups, CUDA-core
 * residual) over 16-row windows.
 * Replaces Libra5BlockOnline.block_sptc_2to4_online
 * (TR-source/Block/block_online.cpp:545-549, return list :844-870).
 * mode TR_ROUTE_COMPAT reproduces the reference's 29 tables bit for bit,
 * including its per-row two-slot truncation of SPTC groups; TR_ROUTE_EXACT
 * makes the same decisions but moves every truncated entry into the CUDA
 * residual so the tables encode A exactly.
 * ---------------------------------------------------------------------- */
enum { TR_ROUTE_COMPAT = 0, TR_ROUTE_EXACT = 1 };

typedef struct tr_route_params {
  int32_t partsize_t;      /* TC sub-blocks per part (32) */
  int32_t partsize_c;      /* CUDA nnz per part (32) */
  int32_t shortsize;       /* CUDA "short" part limit (3) */
  int32_t density;         /* TC column threshold (8) */
  int32_t window;          /* rows per window, 1..16 (16) */
  int32_t wide;            /* range-checked only, as in the reference */
  float tc_min_util;       /* (0.0) */
  float sptc_min_util;     /* accepted, unused (reference block_online.cpp:548) */
  int32_t sptc_threshold;  /* accepted, unused (reference block_online.cpp:549) */
  int32_t unit_min_nnz;    /* LIBRA_SPTC_UNIT_MIN_NNZ (2) */
  int32_t skip_tc;         /* LIBRA_SKIP_TC (0) */
  int32_t mode;            /* TR_ROUTE_COMPAT / TR_ROUTE_EXACT */
  int32_t threads;         /* host threads, <= 0 = all */
  int32_t skip_sptc;       /* 1: no 2:4 groups; every column outside the dense-TC
                              funnel goes to the CUDA parts (0; the plan builder
                              sets it when demote_below > 16, where every 2:4
                              column would be demoted) */
} tr_route_params;

typedef struct tr_route tr_route;

/* host: indptr[n_rows+1], indices[nnz], values[nnz] */
int tr_route_build(const int32_t* indptr, const int32_t* indices, const float* values,
                   int32_t n_rows, const tr_route_params* params, tr_route** out);
/* Table idx in the reference's return order (0..28); `count` is in elements. */
int tr_route_table(const tr_route* r, int idx, const void** data, int64_t* count);
/* The whole router on the device (sm_100a integer kernels, one CTA per
 * window): profile, dense-TC funnel, 2:4 units, max-degree matching, 2:4
 * groups, CUDA long / short parts, TC and mma.sp packing — the 29 tables of
 * tr_route_build, equal to them item for item for the same parameters, from
 * a device CSR whose rows are sorted by column (indptr / indices / values on
 * the device).  The tables stay on the device (one allocation the route
 * holds until tr_route_free): tr_route_table_device gives their device
 * addresses; tr_route_table copies a table to the host on its first call
 * for that table (thread-safe) and returns the host copy.  Replaces
 * block_sptc_2to4_online (TR-source/Block/block_online.cpp:545-871), whose
 * tables the reference's operator uploads to the GPU before every use.
 * params.threads is ignored; tr_route_seconds is the device routing time. */
int tr_route_device(const int32_t* d_indptr, const int32_t* d_indices, const float* d_values,
                    int32_t n_rows, const tr_route_params* params, tr_route** out);
/* Device address and item count of table idx (0..28) of a tr_route_device
 * route (TR_ERR_UNSUPPORTED for host-built routes). */
int tr_route_table_device(const tr_route* r, int idx, const void** d_data, int64_t* count);
/* The router's dense-TC funnel on the device (sm_100a integer kernels:
 * bitonic sorts, warp-ballot compaction, shared atomics; one CTA per
 * window): from a device CSR with rows sorted by column, the TC tables
 * t_row_offset, t_block_offset, t_column, t_value, t_window_row, t_binary
 * exactly as tr_route_build makes them in exact mode (params.window must be
 * 16; the 2:4 and CUDA stages and t_atomic, which depends on the 2:4
 * matching, are not produced).  Replaces the first stage of
 * block_sptc_2to4_online (TR-source/Block/block_online.cpp:584-620, :215-253,
 * :444-540).  Read the tables with tr_route_table (indices 0-4, 6; the
 * others are empty). */
int tr_route_tc_device(const int32_t* d_indptr, const int32_t* d_indices, const float* d_values,
                       int32_t n_rows, const tr_route_params* params, tr_route** out);
/* The device router's dense-TC funnel for callers that cannot allocate GPU
 * memory — code running under a caller-owned memory pool or arena, a
 * framework's custom allocator, or any setting where a cudaMalloc /
 * cudaFree inside the library would synchronise the device or break the
 * caller's memory accounting.  It calls no cudaMalloc, cudaFree or other
 * allocating routine: the caller passes the inputs (device CSR, rows sorted
 * by column) and the output buffers with their capacities (cap_sub
 * sub-blocks: t_column [cap_sub*8], t_binary [cap_sub*2], t_block_offset
 * [cap_sub+1]; cap_val values: t_value [cap_val]); the tables written equal
 * tr_route_tc_device's t_column, t_binary, t_block_offset and t_value, and
 * *n_sub_out / *n_val_out receive their sizes.  Its scratch (per-window
 * counts and offsets, status words: 1 MiB + 16 bytes) is one static device
 * array that every GPU loading the library holds until the process exits.
 * Nothing has to start at zero: each call clears the array's status words
 * itself, every count and offset is written before it is read, and the
 * output buffers are written, not accumulated into.
 * Limits, each refused with a clear error: at most 1,048,576 rows (65,536
 * windows), at most 2048 entries in any 16-row window (use
 * tr_route_tc_device beyond that), capacities large enough for the tables.
 * The first call on a device takes the array's device address and sets the
 * kernels' shared-memory limit.  All calls share the array: calls that
 * overlap on the GPU race (run them on one stream, one after another).  The
 * call waits for `stream` before returning (it reads four status words
 * back), so no call can be captured into a CUDA graph.  No counterpart in
 * the reference. */
int tr_route_tc_device_noalloc(const int32_t* d_indptr, const int32_t* d_indices,
                               const float* d_values, int32_t n_rows,
                               const tr_route_params* params, int32_t* t_column,
                               int64_t* t_binary, float* t_value, int32_t* t_block_offset,
                               int64_t cap_sub, int64_t cap_val, int64_t* n_sub_out,
                               int64_t* n_val_out, void* stream);
/* Seconds spent building the tables (the reference's 30th return). */
double tr_route_seconds(const tr_route* r);
void tr_route_free(tr_route* r);

/* ------------------------------------------------------------------------
 * 2:4 matching statistics: how well each window's columns pair into 2:4
 * groups (the reference's ablation extensions).  Host CSR in, counters out;
 * deterministic (each window's columns in column-id order); counters are
 * 64-bit.  Replaces
 *   TR_MATCH_SLIDING  matching_utils.match_2to4
 *                     (TR-source/Block/block_matching_window_para_dr.cpp:346-412)
 *   TR_MATCH_HASH     matching_utils_hash.match_2to4_hash
 *                     (TR-source/Block/block_matching_hash.cpp:373-420)
 *   TR_MATCH_BUCKET   matching_utils_bucket.match_2to4_bucket
 *                     (TR-source/Block/block_matching_bucket.cpp:430-480)
 *   TR_MATCH_ONLINE   the host restatement of matching_utils_online.match_2to4_online
 *                     (TR-source/Block/block_matching_online.cu:554-668): the
 *                     sliding variant's decisions on 16-row windows, 32 slots per
 *                     group; tr_match_2to4_online runs it on the GPU.
 * dense_threshold and t_max apply to TR_MATCH_SLIDING and TR_MATCH_ONLINE
 * (the others use their fixed constants).  Errors: window_size outside
 * [1, 64] (exactly 16 for TR_MATCH_ONLINE), dense_threshold < 1 (the
 * reference loops forever there), no rows or no columns.
 * ---------------------------------------------------------------------- */
enum { TR_MATCH_SLIDING = 0, TR_MATCH_HASH = 1, TR_MATCH_BUCKET = 2, TR_MATCH_ONLINE = 3 };

typedef struct tr_match_stats {
  int32_t total_rows, total_cols;   /* total_cols = largest column index + 1 */
  int64_t total_nnz;
  double sparsity;
  int32_t num_row_panels;           /* windows */
  int32_t reserved;
  int64_t num_groups;               /* 2:4 groups (num_sptc_groups of the sliding variant) */
  int64_t num_tc_blocks;            /* dense 16x8 blocks (sliding variant; 0 otherwise) */
  int64_t num_16x16_blocks;         /* groups packed four to a 16x16 block, per window */
  int64_t block_padding_groups;
  int64_t fine_fallback;            /* columns left unpaired */
  int64_t coarse_fallback;          /* columns of pairs left ungrouped */
  int64_t fake_zeros;               /* zero slots the groups carry */
  int64_t dense_to_tc_cols;         /* pool columns in dense blocks (sliding / online) */
  int64_t dense_to_sptc_cols;       /* pool columns in 2:4 fallback groups (sliding / online) */
} tr_match_stats;

int tr_match_2to4(const int32_t* indptr, const int32_t* indices, int32_t n_rows, int variant,
                  int32_t window_size, int32_t dense_threshold, int32_t t_max,
                  tr_match_stats* out);
/* TR_MATCH_ONLINE on the GPU (replaces matching_utils_online.match_2to4_online,
 * TR-source/Block/block_matching_online.cu:554-668): host CSR in; like the
 * reference's entry point it copies the matrix to the current device, runs
 * one CTA per 16-row window and waits for the result (this entry point
 * allocates device memory and synchronises).  Columns are taken in id order
 * (deterministic); windows with more than 2048 entries are counted on the
 * host by the same rules (the reference drops their columns past 2048).
 * window_size must be 16.  The result equals tr_match_2to4(TR_MATCH_ONLINE). */
int tr_match_2to4_online(const int32_t* indptr, const int32_t* indices, int32_t n_rows,
                         int32_t window_size, int32_t dense_threshold, int32_t t_max,
                         tr_match_stats* out);

/* ------------------------------------------------------------------------
 * Device plan: the routed operand laid out for the fused sm_100a kernel.
 * Built once per graph (on the host from route tables, uploaded), reused
 * by every forward / adjoint call.
 * ---------------------------------------------------------------------- */
typedef struct tr_plan tr_plan;

typedef struct tr_plan_info {
  int32_t n_rows, n_cols, n_windows;
  int64_t nnz;             /* entries the plan multiplies */
  int64_t tc_tiles;        /* 16x16 tensor-core tiles from the dense route */
  int64_t sptc_tiles;      /* 16x16 2:4 tiles from the SPTC route */
  int64_t residual_nnz;    /* CUDA-core entries */
  int64_t device_bytes;    /* plan footprint in HBM */
  int64_t promoted_tiles;  /* 16x16 tiles holding residual columns moved onto the tensor cores */
  int32_t row_scaled;      /* 1 if values are stored as FP16(v / row scale) */
  int32_t reordered;       /* 1 if the plan's rows were clustered before routing */
  int32_t engine;          /* TR_ENGINE_WINDOW or TR_ENGINE_BLOCK */
  int32_t n_blocks;        /* 128-row blocks (block engine) */
  int64_t chunks;          /* 16-column chunks = tensor-core MMAs per product (block engine) */
  int64_t n_edges;         /* edges (per-entry values) the plan addresses: A's CSR entries */
  int64_t slots;           /* block engine: used K slots = distinct (block, column) pairs
                              (slot layers included) = B rows gathered per product */
} tr_plan_info;

/* Host route tables (pointer + element count each), in the reference's
 * order; the pointers may be NULL when the count is 0. */
typedef struct tr_tables {
  const int32_t* t_row_offset;   int64_t n_t_row_offset;
  const int32_t* t_block_offset; int64_t n_t_block_offset;
  const int32_t* t_column;       int64_t n_t_column;
  const uint16_t* t_value;       int64_t n_t_value;       /* FP16 */
  const int32_t* t_window_row;   int64_t n_t_window_row;
  const int64_t* t_binary;       int64_t n_t_binary;
  const int32_t* c_row_offset;   int64_t n_c_row_offset;
  const int32_t* c_row;          int64_t n_c_row;
  const int32_t* c_column;       int64_t n_c_column;
  const uint16_t* c_value;       int64_t n_c_value;       /* FP16 */
  const int32_t* cs_row_offset;  int64_t n_cs_row_offset;
  const int32_t* cs_row;         int64_t n_cs_row;
  const int32_t* cs_column;      int64_t n_cs_column;
  const uint16_t* cs_value;      int64_t n_cs_value;      /* FP16 */
  const int32_t* s_tile_column;  int64_t n_s_tile_column; /* [tiles*16] */
  const uint32_t* s_packed_a;    int64_t n_s_packed_a;    /* [tiles*64] half2 words */
  const uint32_t* s_packed_meta; int64_t n_s_packed_meta; /* [tiles*8] */
  const int32_t* s_window_tile_offset; int64_t n_s_window_tile_offset; /* [windows+1] */
} tr_tables;

int tr_plan_from_tables(const tr_tables* t, int32_t n_rows, int32_t n_cols, int32_t window,
                        tr_plan** out);
/* Route a CSR with this library's own router (exact mode) and build the
 * plan in one step.  `values` are FP32 (rounded to FP16 in the plan). */
int tr_plan_from_csr(const int32_t* indptr, const int32_t* indices, const float* values,
                     int32_t n_rows, int32_t n_cols, const tr_route_params* params,
                     tr_plan** out);
/* Options of the native plan builder (tr_plan_build).  Zero-initialised
 * options give the same plan as tr_plan_from_csr. */
typedef struct tr_plan_opts {
  int32_t row_scale;       /* 1: per-row FP32 scale s_r = max|v| of the row; the
                              plan stores FP16(v / s_r) and the epilogue
                              multiplies by s_r (small GCN weights keep FP16
                              precision) */
  int32_t promote_min;     /* residual columns used by >= promote_min rows of a
                              16-row window are gathered once and multiplied on
                              the tensor cores (0: keep the CUDA-core residual) */
  int32_t transpose;       /* 1: plan for A^T (the adjoint dB = A^T dC); entry
                              indices still refer to A's CSR */
  int32_t reorder;         /* TR_REORDER_*: rows with shared columns are put into
                              the same windows before routing; results are
                              written to the original row positions */
  int32_t demote_below;    /* 2:4 tile columns holding fewer than demote_below
                              entries of their window go to the CUDA-core
                              residual (0 or 1: keep the router's 2:4 tiles) */
  const int32_t* row_order;  /* TR_REORDER_GIVEN: host array [rows of the
                              (transposed) matrix], plan row i = row_order[i],
                              a permutation (e.g. from tr_tca_order) */
  int32_t engine;          /* TR_ENGINE_WINDOW (0): the reference's three routes
                              over 16-row windows; TR_ENGINE_BLOCK: every entry
                              on the tensor cores over 128-row blocks, each
                              distinct column of a block gathered once (route
                              parameters, promote_min and demote_below do not
                              apply) */
} tr_plan_opts;

/* Plan engines (tr_plan_opts.engine).
 *   TR_ENGINE_WINDOW  the routed layout: dense-TC and 2:4 tiles of 16-row
 *                     windows on the tensor cores, the residual on CUDA cores
 *   TR_ENGINE_BLOCK   128-row blocks: the distinct columns of a block are
 *                     the K slots of 16-column chunks, one tcgen05.mma
 *                     (M = 128 rows, N = K features) per chunk with FP32
 *                     accumulation in TMEM; each row of B is gathered once
 *                     per block and each output row written once (bitwise
 *                     repeatable).  Pays off when rows that share columns
 *                     sit in the same block (reorder = TR_REORDER_LABEL on
 *                     community-structured graphs). */
enum { TR_ENGINE_WINDOW = 0, TR_ENGINE_BLOCK = 1 };

/* Row orders of tr_plan_opts.reorder:
 *   TR_REORDER_NONE     natural order
 *   TR_REORDER_LABEL    label propagation with a 256-row label cap
 *   TR_REORDER_TCA      the TCA clustering of tr_tca_order (default
 *                       parameters, host threads)
 *   TR_REORDER_GIVEN    the caller's permutation in row_order */
enum { TR_REORDER_NONE = 0, TR_REORDER_LABEL = 1, TR_REORDER_TCA = 2, TR_REORDER_GIVEN = 3 };

/* The row order TR_REORDER_LABEL would give a plan of A (transpose = 0) or
 * A^T (transpose = 1), alone: order[rows of that matrix], plan row i = row
 * order[i].  Passing it back as TR_REORDER_GIVEN builds the same plan as
 * TR_REORDER_LABEL, so callers that build several plans of one matrix (an
 * autotuner) compute it once.  Host CSR in; deterministic. */
int tr_label_order(const int32_t* indptr, const int32_t* indices, int32_t n_rows, int32_t n_cols,
                   int32_t transpose, int32_t* order);

/* TCA row clustering (replaces spmm/tr_csr_fp16/tr_tca_reorder.py:44-357,
 * apply_tca_reorder): MinHash-LSH (128 permutations, bands tuned for
 * lsh_threshold) proposes pairs of rows, pairs are merged most similar
 * (exact Jaccard of the column sets) first into clusters of at most `thres`
 * rows, and the clusters the same way into groups of at most `cluster_thres`
 * clusters.  Host CSR in; order[n_rows] out (new position -> old row, the
 * reference's reorder_id).  device = 1 runs the signatures and the Jaccard
 * similarities on the current GPU (same result); the bucket sort and the
 * clustering stay on the host.  Graphs with more than max_pairs candidate
 * pairs are refused (TR_ERR_UNSUPPORTED).  NULL params: the defaults below. */
typedef struct tr_tca_params {
  int32_t thres;           /* 16 */
  int32_t cluster_thres;   /* 128 */
  double lsh_threshold;    /* 0.2 */
  uint64_t seed;           /* 1 */
  int64_t max_pairs;       /* 2^25 */
  int32_t device;          /* 0 */
} tr_tca_params;
typedef struct tr_tca_stats {
  int32_t bands, rows_per_band;   /* LSH banding used */
  int64_t pairs1, clusters1;      /* candidate row pairs, row clusters */
  int64_t pairs2, clusters2;      /* candidate cluster pairs, final groups */
  double seconds[4];              /* wall time of: column sets + signatures,
                                     candidate pairs, Jaccard similarities,
                                     clustering (both levels together) */
} tr_tca_stats;
int tr_tca_order(const int32_t* indptr, const int32_t* indices, int32_t n_rows,
                 const tr_tca_params* params, int32_t* order, tr_tca_stats* stats);
/* The LSH banding tr_tca_order uses: b bands of r rows (b * r <= num_perm)
 * minimising 0.5 * (false-positive + false-negative) probability integrals
 * around the threshold. */
int tr_lsh_params(double threshold, int32_t num_perm, int32_t* bands, int32_t* rows);

/* Native plan builder: validate the CSR, optionally transpose and reorder it,
 * route it (params; mode TR_ROUTE_EXACT keeps every entry) and lay it out.
 * The plan records, for every CSR entry of A, where its value lives, so that
 * tr_plan_set_values can re-value it on the device.  No reference counterpart:
 * the reference re-routes on the host for every new value set. */
int tr_plan_build(const int32_t* indptr, const int32_t* indices, const float* values,
                  int32_t n_rows, int32_t n_cols, const tr_route_params* params,
                  const tr_plan_opts* opts, tr_plan** out);
/* The same builder, stopping before the upload: the host arrays of the plan
 * (for inspection and host-side tests; no device needed).  Arrays by index:
 * 0 win_tile, 1 win_split, 2 win_prom, 3 tile_col, 4 tile_a (FP16 bits),
 * 5 res_ptr, 6 res_col, 7 res_val (FP16 bits), 8 win_order, 9 row_scale
 * (FP32), 10 row_out, 11 val_slot, 12 edge_row, 13 res_edge; block layout:
 * 14 blk_chunk, 15 chunk_col, 16 chunk_ent, 17 ent_pos (uint16), 18 ent_val
 * (FP16 bits), 19 ent_src, 20 blk_order; `count` is in elements. */
typedef struct tr_host_plan tr_host_plan;
int tr_plan_build_host(const int32_t* indptr, const int32_t* indices, const float* values,
                       int32_t n_rows, int32_t n_cols, const tr_route_params* params,
                       const tr_plan_opts* opts, tr_host_plan** out);
int tr_host_plan_array(const tr_host_plan* h, int idx, const void** data, int64_t* count);
int tr_host_plan_upload(const tr_host_plan* h, tr_plan** out);
void tr_host_plan_free(tr_host_plan* h);
/* Plan files: a host plan written to disk once per graph so later runs skip
 * routing and layout (a plan cache; the reference routes on every call,
 * TR-source/spmm/tr_csr_fp16/mdataset2_online.py:100-153).  Versioned binary
 * with a checksum; the file is written beside `path` and renamed into place.
 * Loading refuses (with the reason) files that are not plan files, damaged
 * or truncated ones, other versions and arrays whose sizes or index ranges
 * are inconsistent.  Host only (no device needed); upload with
 * tr_host_plan_upload. */
int tr_host_plan_save(const tr_host_plan* h, const char* path);
int tr_host_plan_load(const char* path, tr_host_plan** out);
int tr_plan_info_get(const tr_plan* p, tr_plan_info* info);
void tr_plan_free(tr_plan* p);

/* ------------------------------------------------------------------------
 * Device compute (no allocation, no synchronisation).
 * ---------------------------------------------------------------------- */

/* Plain single-route CSR SpMM on CUDA cores (the baseline every routed
 * number is compared with).  device: indptr[m+1], indices[nnz],
 * values[nnz] FP16, b[n_cols*k] FP16, c[m*k] FP32 or FP16. */
int tr_spmm_csr(const int32_t* indptr, const int32_t* indices, const uint16_t* values,
                int32_t m, int32_t n_cols, int64_t nnz, const uint16_t* b, int32_t k,
                void* c, int c_dtype, void* stream);

/* Routed forward: C = A_plan · B.  route_mask restricts the routes computed
 * (for per-route timing; promoted tiles count as TR_ROUTE_CUDA); C rows of
 * the plan are fully overwritten.  For a plan built with opts.transpose this
 * is the adjoint dB = A^T · dC. */
int tr_spmm_routed(const tr_plan* p, const uint16_t* b, int32_t k, void* c, int c_dtype,
                   int route_mask, void* stream);

/* Replace the plan's values with new FP32 values of A's CSR entries (device
 * array of n_edges, in A's CSR order), recomputing the row scales of a
 * row-scaled plan.  Entries a compat plan does not multiply are ignored.
 * Used for learnable edge weights (the forward and the adjoint plan of the
 * same A take the same array). */
int tr_plan_set_values(tr_plan* p, const float* values, int64_t n_edges, void* stream);

/* Features per tensor-core launch of a block-engine plan (a multiple of 64
 * up to 256, the MMA's N; 0 = 256): a product of K features runs as
 * ceil(K / k_tile) launches, each gathering its feature slice of the same B
 * rows.  Tuned per graph and K by trspmm.autotune; no effect on window
 * plans. */
int tr_plan_set_k_tile(tr_plan* p, int32_t k_tile);

/* Bitwise-repeatable backward on a window plan (on != 0): the fused
 * adjoint + SDDMM adds the partial sums of rows cut by its segment
 * boundaries in a fixed order instead of by shared-memory atomics (about
 * 13 % slower on the headline graph).  Block-engine plans are always
 * repeatable. */
int tr_plan_set_deterministic(tr_plan* p, int32_t on);

/* Edge numbering.  Every per-entry array a plan reads or writes
 * (tr_plan_set_values' values, tr_adjoint_sddmm's dval) is indexed by edge
 * number; edges start numbered as A's CSR entries.
 *
 * tr_plan_entry_order writes order[q] = the edge at plan position q (device
 * array of n_edges; -1 where no edge sits), for plans whose entries form one
 * stream: block-engine plans and window plans without tensor-core tiles
 * (otherwise TR_ERR_UNSUPPORTED).  An all-residual adjoint plan's positions
 * are A^T's CSR order.
 *
 * tr_plan_renumber_edges gives A's edges new numbers: new_id[e] (device,
 * n_edges, a permutation — refused with TR_ERR_ARG otherwise) becomes the
 * number of the edge now numbered e.  Numbering both plans of one A by the
 * adjoint plan's entry order (new_id[order[q]] = q) makes the adjoint's value
 * upload and the fused backward's dval stores sequential.  Synchronises
 * `stream`; not capturable.  No reference counterpart: the reference keeps
 * no per-entry arrays on the device. */
int tr_plan_entry_order(const tr_plan* p, int32_t* order, void* stream);
int tr_plan_renumber_edges(tr_plan* p, const int32_t* new_id, int64_t n_edges, void* stream);

/* The backward of C = A(w) . B in one call: dB = A^T . dC through the
 * adjoint plan (built with opts.transpose), and dval = SDDMM(dC, B) on A's
 * pattern (a_indptr[a_rows+1], a_indices[nnz] on the device).  When the
 * adjoint plan holds every entry of A in its CUDA-core residual (a native
 * exact plan without tiles) and K <= 128, one kernel does both, gathering
 * each row of dC once for the two products; otherwise the routed adjoint and
 * the SDDMM run one after the other.  dc [a_rows, K] and b [n_cols, K] FP16,
 * db [n_cols, K] FP32 or FP16, dval [nnz] FP32.  No reference counterpart:
 * the reference has no backward. */
int tr_adjoint_sddmm(const tr_plan* adj, const int32_t* a_indptr, const int32_t* a_indices,
                     int32_t a_rows, int64_t nnz, const uint16_t* dc, const uint16_t* b, int32_t k,
                     void* db, int db_dtype, float* dval, void* stream);

/* Sampled dense-dense product on A's pattern (the gradient of the values):
 * out[e] = sum_f x[row(e), f] * y[indices[e], f] for every CSR entry e,
 * FP16 x [m, k] and y [n_cols, k], FP32 accumulation and output.  device:
 * indptr[m+1], indices[nnz], out[nnz]. */
int tr_sddmm_csr(const int32_t* indptr, const int32_t* indices, int32_t m, int32_t n_cols,
                 int64_t nnz, const uint16_t* x, const uint16_t* y, int32_t k, float* out,
                 void* stream);

/* FP32-feature route (replaces the reference's TF32 route for FP32
 * features, TR-source/SpMM/mGCNkernel.cu:2885-3031 and :3513-3674, which no
 * reference operator binds): C = A_plan . B with B [n_cols, k] FP32 on the
 * CUDA cores in FP32 -- the residual on the segment engine (4 features per
 * 16-byte load), the plan's tiles (dense TC, 2:4, promoted) by a CUDA-core
 * tile pass added to C.  A keeps the plan's precision (FP16 significand,
 * FP32 row scale when row-scaled, as precise as TF32); B is not rounded
 * (TF32 would keep 10 of its 23 fraction bits).  c [n_rows, k] FP32 or FP16,
 * every row overwritten; route_mask as in tr_spmm_routed (TR_ROUTE_ALL
 * bits).  K % 4 == 0 with 16-byte aligned b and c takes the vector kernels,
 * anything else a scalar kernel. */
int tr_spmm_routed_f32(const tr_plan* p, const float* b, int32_t k, void* c, int c_dtype,
                       int route_mask, void* stream);
/* tr_adjoint_sddmm with FP32 dc [a_rows, K] and b [n_cols, K]: one pass over
 * the adjoint plan for 16 < K <= 128 (K % 4 == 0) when the plan keeps every
 * entry in its residual; otherwise tr_spmm_routed_f32 then tr_sddmm_csr_f32. */
int tr_adjoint_sddmm_f32(const tr_plan* adj, const int32_t* a_indptr, const int32_t* a_indices,
                         int32_t a_rows, int64_t nnz, const float* dc, const float* b, int32_t k,
                         void* db, int db_dtype, float* dval, void* stream);
/* tr_sddmm_csr with FP32 x [m, k] and y [n_cols, k]. */
int tr_sddmm_csr_f32(const int32_t* indptr, const int32_t* indices, int32_t m, int32_t n_cols,
                     int64_t nnz, const float* x, const float* y, int32_t k, float* out,
                     void* stream);

/* ------------------------------------------------------------------------
 * Reference-compatible entry points (host tensors in, FP32 host out; device
 * memory allocated, copied and freed inside each call; `epoches` timed
 * launches averaged as the reference does).
 * ---------------------------------------------------------------------- */

/* Replaces Libra6SpMMOnline.forward_fp16_tcu_cuda_sptc_mma_parallel_online
 * (TR-source/SpMM/mGCN_online.cpp:760-800, returns :1130-1137).
 * ms_out[0..4] = total, tc, cuda_long, cuda_short, sptc (average per epoch). */
int tr_forward_fp16_tcu_cuda_sptc_mma_parallel_online(
    const int32_t* t_row_offset, int64_t n_t_row_offset,
    const int32_t* t_block_offset, int64_t n_t_block_offset,
    const int32_t* t_column, int64_t n_t_column,
    const uint16_t* t_value, int64_t n_t_value,
    const int32_t* t_window_row, int64_t n_t_window_row,
    const int32_t* t_atomic, int64_t n_t_atomic,
    const int64_t* t_binary, int64_t n_t_binary,
    const int32_t* c_row_offset, int64_t n_c_row_offset,
    const int32_t* c_row, int64_t n_c_row,
    const int32_t* c_atomic, int64_t n_c_atomic,
    const int32_t* c_column, int64_t n_c_column,
    const uint16_t* c_value, int64_t n_c_value,
    const int32_t* c_row_offset_short, int64_t n_c_row_offset_short,
    const int32_t* c_row_short, int64_t n_c_row_short,
    const int32_t* c_atomic_short, int64_t n_c_atomic_short,
    const int32_t* c_column_short, int64_t n_c_column_short,
    const uint16_t* c_value_short, int64_t n_c_value_short,
    const int32_t* s_column, int64_t n_s_column,
    const float* s_value, int64_t n_s_value,
    const int8_t* s_pos, int64_t n_s_pos,
    const int32_t* s_offsets, int64_t n_s_offsets,
    const int32_t* s_tile_window, int64_t n_s_tile_window,
    const int32_t* s_tile_column, int64_t n_s_tile_column,
    const int32_t* s_packed_a, int64_t n_s_packed_a,
    const int32_t* s_packed_meta, int64_t n_s_packed_meta,
    const int32_t* s_window_tile_offset, int64_t n_s_window_tile_offset,
    const uint16_t* rhs_matrix, int64_t n_rhs_matrix,
    int32_t parts_t, int32_t parts_c, int32_t partsize_c, int32_t parts_c_short,
    int32_t window, int32_t dimN, int32_t mOri, int32_t kOri, int32_t epoches,
    float* out, float* ms_out);

/* Replaces Libra6SpMMOnline.forward_fp16_sptc_online (mGCN_online.cpp:202-400):
 * the SPTC route alone from the unpacked group tables. */
int tr_forward_fp16_sptc_online(
    const int32_t* s_column, int64_t n_s_column,
    const float* s_value, int64_t n_s_value,
    const int8_t* s_pos, int64_t n_s_pos,
    const int32_t* s_window, int64_t n_s_window,
    const uint16_t* rhs_matrix, int64_t n_rhs_matrix,
    int32_t window, int32_t dimN, int32_t mOri, int32_t kOri, int32_t epoches,
    float* out, float* ms_out);

/* Replaces Libra6SpMMOnline.forward_fp16_sptc_mma_online (mGCN_online.cpp:404-652):
 * the SPTC route from the unpacked group tables plus per-window group offsets. */
int tr_forward_fp16_sptc_mma_online(
    const int32_t* s_column, int64_t n_s_column,
    const float* s_value, int64_t n_s_value,
    const int8_t* s_pos, int64_t n_s_pos,
    const int32_t* s_offsets, int64_t n_s_offsets,
    const uint16_t* rhs_matrix, int64_t n_rhs_matrix,
    int32_t window, int32_t dimN, int32_t mOri, int32_t kOri, int32_t epoches,
    float* out, float* ms_out);

/* Replaces Libra6SpMMOnline.forward_fp16_sptc_mma_packed_online
 * (mGCN_online.cpp:654-757): the SPTC route from the packed tiles. */
int tr_forward_fp16_sptc_mma_packed_online(
    const int32_t* s_tile_column, int64_t n_s_tile_column,
    const int32_t* s_packed_a, int64_t n_s_packed_a,
    const int32_t* s_packed_meta, int64_t n_s_packed_meta,
    const int32_t* s_window_tile_offset, int64_t n_s_window_tile_offset,
    const uint16_t* rhs_matrix, int64_t n_rhs_matrix,
    int32_t window, int32_t dimN, int32_t mOri, int32_t kOri, int32_t epoches,
    float* out, float* ms_out);

#ifdef __cplusplus
}
#endif
#endif /* TRSPMM_H */
