/*
 * holomap_cuda.h -- C ABI of libholomap_cuda.so, the B200 (sm_100a) exact kNN +
 * smooth-kNN engine for holomap, with the fuzzy simplicial set that follows
 * them (hm_fuzzy_graph*, src/fuzzy.rs:25-91, called at src/api.rs:149).
 *
 * The reference has no FFI on this path: its "operator API" is two
 * crate-private Rust calls made back to back by Holomap::fit_transform,
 *
 *     exact_knn(data: &[f32], n_features, k, metric) -> Knn     src/knn.rs:22
 *     smooth_knn(&knn.dists, k) -> SmoothKnn                     src/smooth_knn.rs:23
 *
 * called at src/api.rs:147-148 after the validation at src/api.rs:114-145.
 * Every entry point below replaces one or both of those calls and returns the
 * same arrays bit for bit: Knn{indices (u32), dists (f32)} row-major n x k
 * (src/knn.rs:13-19) and SmoothKnn{sigmas, rhos} (src/smooth_knn.rs:16-19).
 *
 * Conventions
 *   - Plain pointers and sizes only.  The caller allocates every output.
 *   - Return HM_OK (0) or a negative HM_ERR_* code; hm_last_error() gives a
 *     thread-local message.  Nothing aborts, nothing prints.
 *   - Preconditions: d >= 1, 1 <= k <= n, every input finite (the domain of
 *     exact_knn; fit_transform's validation at src/api.rs:114-145 is stricter,
 *     k >= 2 and n > k).  Violations return HM_ERR_INVALID; a non-finite input
 *     is reported with its first flat index, like HolomapError::NonFiniteInput
 *     (src/api.rs:36-43).
 *   - Host-pointer entry points are synchronous and thread-safe; they copy
 *     the input to the device once and the outputs back once.
 *   - Device-pointer entry points (suffix _device) are stream-ordered and
 *     asynchronous; `stream` is a cudaStream_t passed as void*.
 */
#ifndef HOLOMAP_CUDA_H
#define HOLOMAP_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HM_ABI_VERSION 1

#if defined(__GNUC__)
#define HM_API __attribute__((visibility("default")))
#else
#define HM_API
#endif

/* status codes */
#define HM_OK 0
#define HM_ERR_INVALID (-1)     /* argument outside the reference's preconditions */
#define HM_ERR_OOM (-2)         /* device or pinned allocation failed */
#define HM_ERR_CUDA (-3)        /* CUDA runtime / driver error */
#define HM_ERR_TIMEOUT (-4)     /* a bounded device wait gave up (the kernel returned early) */
#define HM_ERR_ADMISSION (-5)   /* serving: job larger than the context's memory budget */
#define HM_ERR_UNSUPPORTED (-6) /* valid input this build does not handle (message says why) */
#define HM_ERR_NOT_READY (-7)   /* serving: hm_poll / hm_wait on a job still in flight */

/* metric, the reference's Metric enum (src/metric.rs:8-15) plus one extension */
#define HM_METRIC_EUCLIDEAN 0
#define HM_METRIC_COSINE 1
#define HM_METRIC_MANHATTAN 2 /* extension: no reference metric (src/metric.rs:81) */

/* how the N x N distance bulk is evaluated; every path returns the same bytes */
#define HM_PATH_AUTO 0        /* autotuner table picks */
#define HM_PATH_PLAIN 1       /* exact binary64 SIMT over every pair */
#define HM_PATH_SCREEN_BF16 2 /* tcgen05 BF16 screen + exact rerank */
#define HM_PATH_SCREEN_TF32 3 /* tcgen05 TF32 screen + exact rerank */
#define HM_PATH_SCREEN_BF16X3 4 /* tcgen05 split-BF16 (hi*hi + hi*lo + lo*hi) screen + rerank */

/* Optional per-call statistics (pass NULL to skip). */
typedef struct hm_stats {
    int32_t path_used;           /* HM_PATH_* actually run */
    uint32_t col_splits;         /* plain path: column splits per row block */
    uint64_t candidates_total;   /* screened paths: candidates reranked exactly */
    uint32_t candidates_max_row; /* screened paths: most candidates in one row */
    uint32_t candidate_cap;      /* screened paths: per-row candidate capacity */
    uint64_t overflow_rows;      /* screened paths: rows sent to the exact path */
    uint64_t zero_rho_rows;      /* rows whose sigma floor used the global mean */
    double screen_band;          /* screened paths: largest keep band (distance units) */
    double device_ms;            /* device time of the call's kernels */
    uint64_t candidates_emitted; /* screened paths: candidates the screen wrote (before the
                                    final threshold) */
} hm_stats;

/* ----------------------------------------------------------------------------
 * Host-buffer entry points (synchronous)
 * ------------------------------------------------------------------------- */

/* Replaces exact_knn (src/knn.rs:22-55).  data: n x d row-major f32.
 * idx_out / dist_out: n x k.  Row i lists its k nearest points (itself
 * included, at distance exactly 0) ordered by (distance, index). */
HM_API int hm_knn(const float *data, uint64_t n, uint32_t d, uint32_t k, int metric,
           int path, uint32_t *idx_out, float *dist_out, hm_stats *stats);

/* Replaces smooth_knn (src/smooth_knn.rs:23-80).  dists: n x k, each row
 * ascending as exact_knn returns it.  sigma_out / rho_out: n. */
HM_API int hm_smooth_knn(const float *dists, uint64_t n, uint32_t k, float *sigma_out,
                  float *rho_out);

/* Replaces both calls of src/api.rs:147-148 with one device round trip. */
HM_API int hm_knn_smooth(const float *data, uint64_t n, uint32_t d, uint32_t k, int metric,
                  int path, uint32_t *idx_out, float *dist_out, float *sigma_out,
                  float *rho_out, hm_stats *stats);

/* ----------------------------------------------------------------------------
 * Device-pointer entry points (stream-ordered; same results as above)
 * ------------------------------------------------------------------------- */

/* Bytes of device scratch hm_knn_smooth_device needs for this problem. */
HM_API size_t hm_workspace_bytes(uint64_t n, uint32_t d, uint32_t k, int metric, int path);

/* Both stages on device memory.  d_sigma/d_rho may be NULL to skip
 * smooth-kNN.  d_workspace: hm_workspace_bytes(...) bytes, 256-byte aligned.
 * stats (optional) is filled only with what is known without a host sync
 * (path, splits, cap); counts need hm_stats_from_workspace after the stream
 * has been synchronised. */
HM_API int hm_knn_smooth_device(const float *d_data, uint64_t n, uint32_t d, uint32_t k,
                         int metric, int path, uint32_t *d_idx, float *d_dist,
                         float *d_sigma, float *d_rho, void *d_workspace,
                         size_t workspace_bytes, void *stream, hm_stats *stats);

/* Reads the counters a finished hm_knn_smooth_device call left in its
 * workspace (synchronous copy). */
HM_API int hm_stats_from_workspace(const void *d_workspace, uint64_t n, uint32_t d, uint32_t k,
                            int metric, int path, hm_stats *stats);

/* A row shard of exact_knn (src/knn.rs:22-55): query rows [row_begin,
 * row_end) against all n points, for splitting one dataset across GPUs (each
 * rank holds all points and computes its rows).  Row i of d_idx / d_dist
 * ((row_end - row_begin) x k) is point row_begin + i; indices refer to all n
 * points; the bytes equal rows [row_begin, row_end) of the whole graph.
 * smooth-kNN is not part of a shard (a rho == 0 row's sigma floor needs the
 * mean over all n*k distances): gather the shards' distances and run
 * hm_smooth_knn_device over all n rows. */
HM_API size_t hm_knn_rows_workspace_bytes(uint64_t n, uint32_t d, uint32_t k, int metric, int path,
                                          uint64_t row_begin, uint64_t row_end);
HM_API int hm_knn_rows_device(const float *d_data, uint64_t n, uint32_t d, uint32_t k, int metric,
                              int path, uint64_t row_begin, uint64_t row_end, uint32_t *d_idx,
                              float *d_dist, void *d_workspace, size_t workspace_bytes,
                              void *stream, hm_stats *stats);
/* Counters of a finished hm_knn_rows_device call (synchronous read). */
HM_API int hm_knn_rows_stats(const void *d_workspace, uint64_t n, uint32_t d, uint32_t k,
                             int metric, int path, uint64_t row_begin, uint64_t row_end,
                             hm_stats *stats);

/* smooth-kNN alone on device memory (src/smooth_knn.rs:23-80). d_workspace:
 * hm_smooth_workspace_bytes(n) bytes. */
HM_API size_t hm_smooth_workspace_bytes(uint64_t n);
HM_API int hm_smooth_knn_device(const float *d_dists, uint64_t n, uint32_t k, float *d_sigma,
                         float *d_rho, void *d_workspace, void *stream);
/* smooth-kNN of the rows [row_begin, row_end) of an n x k distance matrix,
 * for a row shard: d_sigma / d_rho receive (row_end - row_begin) values, the
 * same bits as rows [row_begin, row_end) of hm_smooth_knn_device over all n
 * rows (a rho == 0 row's floor is the mean of all n * k distances,
 * src/smooth_knn.rs:26, :70-74).  d_workspace: hm_smooth_workspace_bytes(n). */
HM_API int hm_smooth_knn_rows_device(const float *d_dists, uint64_t n, uint32_t k, uint64_t row_begin,
                                     uint64_t row_end, float *d_sigma, float *d_rho, void *d_workspace,
                                     void *stream);

/* The fuzzy simplicial set (replaces fuzzy_simplicial_set, src/fuzzy.rs:25-91):
 * the kNN graph (n x k indices and distances, each row's indices distinct, as
 * exact_knn returns them) and its calibration (sigma, rho) fused into the
 * symmetric membership graph W = A + A^T - A o A^T in binary32, as COO sorted
 * by (row, col) with zeros dropped; the same entries, in the same order, with
 * the same bits as the reference.  Every sigma must be non-negative, as
 * smooth-kNN returns it (the host entry point checks this and the index
 * bound).  Capacity of rows / cols / vals: 2 n k entries; *nnz receives the
 * count.  n k must stay below 2^31.
 *
 * hm_fuzzy_graph: host buffers in and out (one allocation, synchronous).
 * hm_fuzzy_graph_device: device pointers; d_nnz is a device uint64; the
 * workspace (hm_fuzzy_workspace_bytes, 256-byte aligned) holds the sort's
 * buffers; ordered on `stream`, nothing synchronised. */
HM_API size_t hm_fuzzy_workspace_bytes(uint64_t n, uint32_t k);
HM_API int hm_fuzzy_graph_device(const uint32_t *d_idx, const float *d_dist, const float *d_sigma,
                                 const float *d_rho, uint64_t n, uint32_t k, uint32_t *d_rows,
                                 uint32_t *d_cols, float *d_vals, uint64_t *d_nnz, void *d_workspace,
                                 size_t workspace_bytes, void *stream);
HM_API int hm_fuzzy_graph(const uint32_t *idx, const float *dist, const float *sigma, const float *rho,
                          uint64_t n, uint32_t k, uint32_t *rows_out, uint32_t *cols_out,
                          float *vals_out, uint64_t *nnz_out);
/* After hm_fuzzy_graph_device on `stream` (synchronous read of its workspace):
 * HM_ERR_INVALID if some index was not below n or a row repeated an index
 * (the kernels keep every access in bounds, but the output is then not the
 * fuzzy set of a kNN graph), else HM_OK.  hm_fuzzy_graph checks it itself. */
HM_API int hm_fuzzy_graph_status(const void *d_workspace, uint64_t n, uint32_t k, void *stream);

/* The spectral stage that follows the fuzzy graph (spectral_layout_single,
 * src/spectral.rs:70-83).
 *
 * hm_laplacian_device replaces Laplacian::new (src/sparse.rs:56-71, with
 * Csr::from_fuzzy :21-35): from the (row, col)-sorted COO of n points
 * (d_rows / d_cols / d_vals, nnz entries, as hm_fuzzy_graph writes it) it
 * writes the CSR offsets d_indptr (n + 1), the normalized weights d_svals
 * (nnz, S = D^-1/2 W D^-1/2) and d_degrees (n), bit for bit as the
 * reference; the column indices of the CSR are d_cols itself.
 * hm_laplacian_matvec_device replaces Laplacian::matvec (src/sparse.rs:78-84):
 * d_y = L d_x = d_x - S d_x, bit for bit.
 *
 * hm_eigenpairs_device replaces smallest_eigenpairs (src/eigen.rs:31-37)
 * with the Lanczos iteration of src/eigen.rs:95-223 at every n: the k
 * smallest eigenvalues of L (ascending, values_out) and unit eigenvectors
 * (vectors_out, column-major n x k, canonical sign), both HOST arrays.
 * *found_out = pairs locked (k unless 200 cycles ran out), *cycles_out (may
 * be NULL) = restart cycles run.  The eigenpairs agree with the reference to
 * its tolerances, not bit for bit (the tridiagonal step uses the implicit QL
 * method; the reference uses nalgebra), and are identical from run to run.
 * d_workspace: hm_eigenpairs_workspace_bytes(n, k), 256-byte aligned.
 * Synchronous (the iteration reads a few scalars back every step); 1 <= k <=
 * min(n, 1024).
 *
 * hm_spectral_eigenpairs: host COO in, eigenpairs out (one allocation). */
HM_API int hm_laplacian_device(const uint32_t *d_rows, const uint32_t *d_cols, const float *d_vals,
                               uint64_t n, uint64_t nnz, uint64_t *d_indptr, double *d_svals,
                               double *d_degrees, void *stream);
HM_API int hm_laplacian_matvec_device(const uint64_t *d_indptr, const uint32_t *d_cols,
                                      const double *d_svals, uint64_t n, const double *d_x,
                                      double *d_y, void *stream);
HM_API size_t hm_eigenpairs_workspace_bytes(uint64_t n, uint32_t k);
HM_API int hm_eigenpairs_device(const uint64_t *d_indptr, const uint32_t *d_cols,
                                const double *d_svals, uint64_t n, uint32_t k, void *d_workspace,
                                size_t workspace_bytes, void *stream, double *values_out,
                                double *vectors_out, uint32_t *found_out, uint32_t *cycles_out);
HM_API int hm_spectral_eigenpairs(const uint32_t *rows, const uint32_t *cols, const float *vals,
                                  uint64_t n, uint64_t nnz, uint32_t k, double *values_out,
                                  double *vectors_out, uint32_t *found_out, uint32_t *cycles_out);

/* ----------------------------------------------------------------------------
 * Batches: many independent problems of uneven n, d, k and metric in one
 * pass of the device pipeline (every kernel works on the whole batch; the
 * screened jobs of one operand format share one persistent screen launch).
 * No reference counterpart: the reference embeds one dataset per call; each
 * job is the same computation as exact_knn + smooth_knn on its own data.
 * ------------------------------------------------------------------------- */

/* One problem of a batch.  All pointers are device pointers; sigma_out /
 * rho_out NULL skips smooth-kNN for the job. */
typedef struct hm_job {
    const float *data;  /* n x d row-major */
    uint64_t n;
    uint32_t d, k;
    int32_t metric, path;
    uint32_t *idx_out;  /* n x k */
    float *dist_out;    /* n x k */
    float *sigma_out;   /* n (or NULL) */
    float *rho_out;     /* n (or NULL) */
} hm_job;

typedef struct hm_batch hm_batch; /* opaque plan of one batch */

/* Validate and lay out a batch (host only; no device work). */
HM_API int hm_batch_create(const hm_job *jobs, uint32_t njobs, hm_batch **out);
HM_API void hm_batch_destroy(hm_batch *batch);
/* Device scratch the batch needs. */
HM_API size_t hm_batch_workspace_bytes(const hm_batch *batch);
/* Attach the workspace (256-byte aligned) and write the batch's job tables
 * into it, ordered on `stream`. */
HM_API int hm_batch_bind(hm_batch *batch, void *d_workspace, size_t workspace_bytes, void *stream);
/* Enqueue the whole pipeline on `stream` (kernel launches only: no host
 * synchronisation, no allocation). */
HM_API int hm_batch_run(hm_batch *batch, void *stream);
/* Same work as hm_batch_run, through a CUDA graph that the first call
 * captures on `stream` and later calls replay with one launch. */
HM_API int hm_batch_graph_launch(hm_batch *batch, void *stream);
/* Counters of one job after the stream has finished (synchronous read).
 * Returns HM_ERR_INVALID when the job's data held a non-finite value. */
HM_API int hm_batch_job_stats(const hm_batch *batch, uint32_t job, hm_stats *stats);
/* The path the planner resolved for one job. */
HM_API int hm_batch_job_path(const hm_batch *batch, uint32_t job);

/* ----------------------------------------------------------------------------
 * Serving: a request loop on one device.  No reference counterpart (the
 * reference answers one fit_transform call at a time); each request is the
 * computation of src/api.rs:147-148 on its own data and returns the same
 * bytes alone or in any mix.
 *
 * A context owns a device arena of `memory_bytes`.  Submitted requests wait
 * in arrival order; a scheduler thread admits them while their device
 * footprint (points + outputs + pipeline scratch) fits the arena and a batch
 * slot is free, runs each admitted group as one batch on its own stream
 * (copy in, pipeline, copy out), and forms the next batch from whatever has
 * arrived as soon as a slot frees, so batches overlap on the device.
 * Requests whose footprint exceeds the arena fail with HM_ERR_ADMISSION.
 * ------------------------------------------------------------------------- */

typedef struct hm_ctx hm_ctx; /* opaque serving context */

typedef struct hm_ctx_config {
    uint64_t memory_bytes;   /* device arena; 0 = 3/4 of the device's free memory */
    uint32_t max_inflight;   /* batches on the device at once; 0 = 4 */
    uint32_t max_batch_jobs; /* requests per batch; 0 = 64 */
    double max_batch_work;   /* a batch closes once its sum of n*n*d passes this; 0 = 4e11 */
    double small_work;       /* requests with n*n*d at or below this are batched apart and run
                                on high-priority streams; 0 = 2e10 */
} hm_ctx_config;

/* What a finished (or pending) request reports. */
typedef struct hm_request_info {
    int32_t status;      /* HM_OK, HM_ERR_NOT_READY while queued/running, or its error */
    int32_t path_used;   /* HM_PATH_* the planner chose */
    uint64_t batch;      /* sequence number of the batch that ran it */
    uint32_t batch_jobs; /* requests in that batch */
    uint32_t reserved;
    double submit_ms;    /* steady-clock times since hm_ctx_create */
    double admit_ms;
    double done_ms;
    hm_stats stats;      /* the request's counters (device_ms is 0) */
} hm_request_info;

/* Start a context on the current device (starts the scheduler thread). */
HM_API int hm_ctx_create(const hm_ctx_config *config_or_null, hm_ctx **out);
/* Finish every submitted request, stop the scheduler and free the context. */
HM_API int hm_ctx_destroy(hm_ctx *ctx);
/* Queue one request.  In a request, data / idx_out / dist_out / sigma_out /
 * rho_out are HOST pointers (page-locked memory lets the copies overlap;
 * sigma_out / rho_out may be NULL) that must stay valid until the request
 * is finished.  Returns a ticket. */
HM_API int hm_submit(hm_ctx *ctx, const hm_job *request, uint64_t *ticket);
/* HM_OK when finished successfully, HM_ERR_NOT_READY while pending, else
 * the request's error.  info (optional) is filled in every case. */
HM_API int hm_poll(hm_ctx *ctx, uint64_t ticket, hm_request_info *info);
/* Block until the request finishes or timeout_ns passes (then HM_ERR_NOT_READY);
 * timeout_ns >= 2^62 (UINT64_MAX included) waits without a deadline. */
HM_API int hm_wait(hm_ctx *ctx, uint64_t ticket, uint64_t timeout_ns, hm_request_info *info);
/* Forget a finished ticket (its info is no longer kept). */
HM_API int hm_release(hm_ctx *ctx, uint64_t ticket);

typedef struct hm_ctx_totals {
    uint64_t submitted, finished, failed, batches;
    uint64_t arena_bytes, arena_peak_bytes; /* capacity and high-water mark */
    uint32_t max_batch_jobs_seen, max_inflight_seen;
} hm_ctx_totals;
HM_API int hm_ctx_totals_read(hm_ctx *ctx, hm_ctx_totals *totals);

/* ----------------------------------------------------------------------------
 * Allocation-free entry point.  No counterpart in the reference (its Rust
 * path allocates its Vecs freely); this exists for callers that cannot call
 * cudaMalloc: a plugin inside a host engine that has already reserved the
 * card's memory for its own allocator, or a latency-bound request loop that
 * must not call the allocator because cudaMalloc/cudaFree can block and
 * synchronise the device.
 * ------------------------------------------------------------------------- */

/* Size of the fixed device scratch array inside the library (64 MiB).  Every
 * GPU that loads the library holds it until the process exits. */
#define HM_NOALLOC_SCRATCH_BYTES (64ull << 20)

/* The same results as hm_knn_smooth_device on the plain path, with the
 * caller's device inputs and outputs and no allocation of any kind: scratch
 * comes from the library's static array.  Problems whose scratch
 * (hm_workspace_bytes(..., HM_PATH_PLAIN)) exceeds HM_NOALLOC_SCRATCH_BYTES
 * are rejected with HM_ERR_UNSUPPORTED.  The first call on a device (and in
 * each new CUDA context of it, e.g. after cudaDeviceReset) looks up the
 * array's device address: make it before any stream capture.  All calls share
 * the array: calls that overlap on the GPU race on it.  The call itself does
 * not wait for the device, so a non-finite input is reported by
 * hm_noalloc_stats, not by this return code. */
HM_API int hm_knn_smooth_noalloc(const float *d_data, uint64_t n, uint32_t d, uint32_t k,
                                 int metric, uint32_t *d_idx, float *d_dist, float *d_sigma,
                                 float *d_rho, void *stream);
HM_API size_t hm_noalloc_scratch_bytes(void);

/* The status and counters of the last hm_knn_smooth_noalloc call on the
 * current device, which stay in the static scratch: waits for the work queued
 * on `stream` (the stream that call used) and reads them into a host struct,
 * allocating nothing.  Returns HM_ERR_INVALID when that call's points held a
 * non-finite value (hm_last_error() names its first flat index), as the
 * workspace-taking entry points do, HM_ERR_TIMEOUT if a bounded device wait
 * gave up, else HM_OK; stats (optional) receives the counts.  The next call on
 * the device overwrites them, and calls that overlap on the GPU race on them.
 * No counterpart in the reference (see hm_knn_smooth_noalloc). */
HM_API int hm_noalloc_stats(void *stream, hm_stats *stats);

/* ----------------------------------------------------------------------------
 * Misc
 * ------------------------------------------------------------------------- */

/* Thread-local text of the last error on this thread ("" if none). */
HM_API const char *hm_last_error(void);

/* HM_ABI_VERSION of the loaded library. */
HM_API int hm_abi_version(void);

/* The path HM_PATH_AUTO resolves to for this problem: the choice of the
 * nearest grid point of the autotuner table, measured on a B200 by
 * holomap_b200/autotune.py (holomap_b200/autotune_table.json); plain where
 * no screen applies (manhattan, k > 64, d > 2048). */
HM_API int hm_autotune_path(uint64_t n, uint32_t d, uint32_t k, int metric);
/* The same for a job planned in a batch of several (hm_batch_*, the serving
 * context's batches): the table measured on batches of jobs of each shape,
 * where the screens' fixed per-call costs are shared. */
HM_API int hm_autotune_path_batched(uint64_t n, uint32_t d, uint32_t k, int metric);
/* Autotuner sweep hook (no reference counterpart): while seed_div is nonzero,
 * screened plans made on this thread sample 1/seed_div of the columns in the
 * screen's threshold pass instead of the table's fraction; 0 restores the
 * table.  The results do not depend on it, only the speed. */
HM_API int hm_tuning_override(int seed_div);
/* Sweep and test hook (no reference counterpart): the emission form of the
 * screened plans made on this thread.  mode = 0: the pass runs over every
 * column tile; mode = 1: the symmetric form wherever a job can take it (a
 * whole dataset of at least two column tiles: only the tiles on and above
 * the diagonal, each value also serving its column's row); mode = -1 (the
 * default): the autotuner table's choice.  Same results in every mode. */
HM_API int hm_tuning_symmetric(int mode);
/* Sweep and test hook (no reference counterpart): mode = 0: the emission pass
 * runs with one CTA per 128-row block; mode = 1: the 2-SM form (a cluster of
 * two CTAs sharing one 256-row MMA, each CTA loading half of every column
 * tile) wherever a group can take it; mode = -1 (the default): the
 * autotuner table's choice.  Same results in every mode. */
HM_API int hm_tuning_pair(int mode);
/* Test hook (no reference counterpart): with on = 0, jobs planned on this
 * thread with HM_PATH_AUTO carry no escalation copy.  By default a job the
 * autotuner sends to the BF16 or TF32 screen also carries a split-BF16 copy:
 * after the threshold pass the device compares each row's keep band with its
 * threshold, and when the coarse screen would keep a large share of the
 * dataset for more than a tenth of the rows (points in clusters far tighter
 * than its rounding), the copy screens the job instead.  Same results either
 * way; hm_stats.path_used then reports HM_PATH_SCREEN_BF16X3. */
HM_API int hm_tuning_escalation(int on);

/* ----------------------------------------------------------------------------
 * Instrumentation (no reference counterpart; the reference has no timers on
 * this path).  With timing enabled the library records a CUDA event pair, on
 * the launching stream, around every launch of each kernel class below.
 * ------------------------------------------------------------------------- */
#define HM_KCLASS_BULK 0   /* tensor-core screen (the screened paths' N x N bulk) */
#define HM_KCLASS_SELECT 1 /* split merge / exact rerank + select */
#define HM_KCLASS_SMOOTH 2 /* smooth-kNN calibration */
#define HM_KCLASS_PREP 3   /* input checks, binary64 copy, operand prep */
#define HM_KCLASS_EXACT 4  /* exact binary64 kernel (plain path and fallback rows) */
#define HM_KCLASS_COUNT 5

HM_API int hm_timing_enable(int on);
/* Sum of event-timed milliseconds and launch count of one class since the
 * last reset (synchronises the recorded events). */
HM_API int hm_timing_read(int kernel_class, double *total_ms, uint64_t *launches, int reset);
/* Kernels this library has launched since it was loaded (all classes). */
HM_API uint64_t hm_launch_count(void);
/* Measured binary64 throughput of the current device (round-to-nearest
 * multiplies and adds per second, the operations of the exact kernels): a
 * synchronous probe of a few milliseconds on a private stream, used as the
 * FP64 roofline.  Changes no device setting. */
HM_API int hm_measure_fp64_rate(double *ops_per_s);

/* Test hook: while set (non-NULL), screened runs on this thread also write
 * every screened value c^_ij into d_out[i * n + j] (n x n floats). */
HM_API int hm_debug_set_screen_dump(float *d_out);

/* Test hook (host only, no device): the tridiagonal eigensolver of the
 * Lanczos iteration on diagonal d[m] and off-diagonal e[m - 1]; vals_out[m]
 * (unordered) and vecs_out (m x m row-major, eigenvectors as columns). */
HM_API int hm_debug_tridiag_eigen(const double *d, const double *e, uint32_t m, double *vals_out,
                                  double *vecs_out);

#ifdef __cplusplus
}
#endif

#endif /* HOLOMAP_CUDA_H */
