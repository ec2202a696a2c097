// hm_internal.cuh -- shared declarations of libholomap_cuda.so.
//
// Numerical contract: every kernel that produces a returned value does so in
// exactly the reference's operation order with explicitly rounded intrinsics
// (__dadd_rn, __dmul_rn, __fadd_rn, ...), and the library is compiled with
// --fmad=false so that nothing is contracted into an FMA.  See the comments in
// each kernel file for the reference lines it follows.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "../../include/holomap_cuda.h"

namespace hm {

// ---------------------------------------------------------------- errors
// Thread-local message for hm_last_error(); returns `code` for chaining.
int set_error(int code, const char *fmt, ...);
void clear_error();

#define HM_CUDA_TRY(expr)                                                        \
    do {                                                                         \
        cudaError_t e_ = (expr);                                                 \
        if (e_ != cudaSuccess)                                                   \
            return ::hm::set_error(e_ == cudaErrorMemoryAllocation ? HM_ERR_OOM  \
                                                                   : HM_ERR_CUDA, \
                                   "%s: %s (%s:%d)", #expr, cudaGetErrorString(e_), \
                                   __FILE__, __LINE__);                          \
    } while (0)

#define HM_TRY(expr)              \
    do {                          \
        int rc_ = (expr);         \
        if (rc_ != HM_OK) return rc_; \
    } while (0)

inline size_t round_up(size_t x, size_t m) { return (x + m - 1) / m * m; }

// Sets a kernel's dynamic shared-memory limit once per device (the attribute
// call is kept off the per-launch path).
int ensure_dynamic_smem(const void *func, int bytes);
// Multiprocessor count of the current device (cached; 148 without a device).
int device_sm_count();

// ----------------------------------------------------------- instrumentation
// Every kernel launch calls count_launch(); ScopedKernelTimer records an
// event pair around the launches in its scope when timing is enabled.
void count_launch(uint64_t n = 1);
bool timing_enabled();
void timing_record(int kclass, cudaStream_t s, bool start);

struct ScopedKernelTimer {
    int cls;
    cudaStream_t s;
    bool on;
    ScopedKernelTimer(int c, cudaStream_t st) : cls(c), s(st), on(timing_enabled()) {
        if (on) timing_record(cls, s, true);
    }
    ~ScopedKernelTimer() {
        if (on) timing_record(cls, s, false);
    }
};

// -------------------------------------------------------- composite keys
// Every returned distance is +0.0 or positive (possibly +inf), so its binary32
// bit pattern orders like the value and the 64-bit key (bits << 32) | index
// orders exactly like the reference's (total_cmp(dist), index) sort
// (src/knn.rs:46-48).  ~0 is a sentinel larger than every real key.
constexpr uint64_t KEY_NONE = ~0ull;

__device__ __forceinline__ uint64_t make_key(float dist, uint32_t idx) {
    return ((uint64_t)__float_as_uint(dist) << 32) | (uint64_t)idx;
}
__device__ __forceinline__ float key_dist(uint64_t key) {
    return __uint_as_float((uint32_t)(key >> 32));
}
__device__ __forceinline__ uint32_t key_idx(uint64_t key) { return (uint32_t)key; }

__device__ __forceinline__ uint64_t shfl_u64(uint64_t v, int src) {
    uint32_t lo = __shfl_sync(0xffffffffu, (uint32_t)v, src);
    uint32_t hi = __shfl_sync(0xffffffffu, (uint32_t)(v >> 32), src);
    return ((uint64_t)hi << 32) | lo;
}
__device__ __forceinline__ uint64_t shfl_xor_u64(uint64_t v, int mask) {
    uint32_t lo = __shfl_xor_sync(0xffffffffu, (uint32_t)v, mask);
    uint32_t hi = __shfl_xor_sync(0xffffffffu, (uint32_t)(v >> 32), mask);
    return ((uint64_t)hi << 32) | lo;
}
__device__ __forceinline__ uint64_t shfl_up_u64(uint64_t v, int delta) {
    uint32_t lo = __shfl_up_sync(0xffffffffu, (uint32_t)v, delta);
    uint32_t hi = __shfl_up_sync(0xffffffffu, (uint32_t)(v >> 32), delta);
    return ((uint64_t)hi << 32) | lo;
}

// A sorted list of the KPL*32 smallest keys seen, spread over a warp: element
// e lives in lane (e % 32) of slot (e / 32).  `tau` is element k-1, the
// admission threshold (warp-uniform).  Insert is warp-collective and requires
// x < tau (so x lands inside the first k elements).
template <int KPL>
struct WarpTopK {
    uint64_t v[KPL];
    uint64_t tau;

    __device__ __forceinline__ void reset() {
#pragma unroll
        for (int q = 0; q < KPL; ++q) v[q] = KEY_NONE;
        tau = KEY_NONE;
    }

    __device__ __forceinline__ void refresh_tau(uint32_t k, int lane) {
        const uint32_t qk = (k - 1) >> 5, lk = (k - 1) & 31;
        uint64_t t = KEY_NONE;
#pragma unroll
        for (int q = 0; q < KPL; ++q)
            if ((uint32_t)q == qk) t = v[q];
        tau = shfl_u64(t, (int)lk);
    }

    __device__ __forceinline__ void insert(uint64_t x, uint32_t k, int lane) {
        int pos = 0;
#pragma unroll
        for (int q = 0; q < KPL; ++q) pos += __popc(__ballot_sync(0xffffffffu, v[q] < x));
        uint64_t carry = KEY_NONE;
#pragma unroll
        for (int q = 0; q < KPL; ++q) {
            uint64_t up = shfl_up_u64(v[q], 1);
            uint64_t last = shfl_u64(v[q], 31);
            if (lane == 0) up = carry;
            const int e = q * 32 + lane;
            v[q] = (e < pos) ? v[q] : (e == pos ? x : up);
            carry = last;
        }
        refresh_tau(k, lane);
    }

    // Offer one key per lane; all lanes' keys below tau are inserted.
    __device__ __forceinline__ void offer(uint64_t key, uint32_t k, int lane) {
        unsigned m = __ballot_sync(0xffffffffu, key < tau);
        while (m) {
            const int src = __ffs(m) - 1;
            const uint64_t x = shfl_u64(key, src);
            insert(x, k, lane);
            m &= m - 1;
            m &= __ballot_sync(0xffffffffu, key < tau);
        }
    }
};

// ------------------------------------------------------------- jobs
// Every kernel works on a table of jobs (independent kNN problems): a single
// call is a batch of one.  Rows of all jobs form one "all-rows" space (job j
// owns rows [arow0, arow0 + n)); screened jobs of one operand format also
// share a "group" row space (job j owns group rows [row0, row0 + n)).

// Device-written counters of one job.
struct JobCounters {
    uint32_t nonfinite_min;  // smallest flat index of a non-finite input, or ~0
    uint32_t zero_count;     // rows whose rho is 0 (global-mean sigma floor)
    uint32_t ovf_count;      // screened rows sent to the exact fallback
    uint32_t max_row;        // most candidates reranked in one row
    unsigned long long candidates;  // candidates reranked exactly
    unsigned long long emitted;     // candidates the screen wrote
    uint32_t band_max_bits;  // widest keep band (binary32 bits)
    uint32_t error_code;     // nonzero if a bounded wait gave up
    uint32_t escalate;       // 1: the job's screen was too coarse for its data; its
                             // split-BF16 copy produced the rows (see JobDev::gate)
    uint32_t escalate_rows;  // rows whose band exceeded the escalation share of tau1
    // screen prep maxima (non-negative doubles as bits): |u|, |e|, |r|,
    // |A row|, |B row|, |u|^2, largest centred |x - mu|^2; then zero rows
    unsigned long long maxb[8];
};

struct JobDev {
    // problem and caller buffers (device pointers)
    uint32_t n, d, k, metric, path;
    uint32_t arow0;  // first row in the all-rows space
    uint32_t q0, q1; // query rows [q0, q1): a row shard; every row is a column
    uint32_t rb0;    // first 128-row screen block of the query rows
    const float *x;
    uint32_t *idx;              // addressed as idx[row * k] for rows in [q0, q1)
    float *dist, *sigma, *rho;  // sigma / rho null: no smooth-kNN
    // exact path (and the screened path's fallback)
    double *x64;                 // n_pad x ldd binary64 copy
    double *rnorm;               // sqrt of the sequential sum of squares (cosine)
    uint32_t ldd, n_pad, splits, split_cols;
    uint64_t *partial;           // splits x n x k keys (splits > 1)
    // smooth-kNN
    double target;               // log2(k), host platform log2
    uint32_t *zero_rows;         // n
    // screened path
    uint32_t group, row0, unit0, kp1, k_stages, row_blocks, col_tiles, parts, part_tiles, cap;
    uint32_t seed_tiles;         // leading column tiles of each part in the threshold pass
    unsigned long long slot0;    // first threshold-pass list (tlists * parts lists per row)
    uint32_t tlists;             // threshold-pass lists per column part (its epilogue segments)
    unsigned long long topk0;    // first k-array entry: list l's is [topk0 + (l - slot0) * k, +k)
    // candidate lists of the emission pass: elists per row (two per column
    // part; with the symmetric emission one more, the row's column list, last)
    uint32_t elists, sym;        // sym: the emission pass covers the tiles on and above the diagonal
    unsigned long long eslot0;   // first candidate list of the job
    unsigned long long cand0;    // first candidate slot: list l holds [cand0 + (l - eslot0) * cap, +cap)
    float scale;                 // 1 (cosine) or 2 (euclidean)
    double *mu, *csum;           // euclidean column mean and its partial sums
    uint32_t csum_blocks, csum_rows;
    uint32_t *ovf_list;          // n (job-local rows)
    JobCounters *cnt;            // the job's working counters (screen prep maxima)
    JobCounters *out;            // where its reported counts go (the original's for a copy)
    // Escalation: a job screened in BF16 or TF32 may carry a split-BF16 copy
    // (a second job entry on the same points and outputs).  After its
    // threshold pass a kernel decides, from the rows' bands against their
    // thresholds, whether the coarse screen would keep most of the dataset;
    // then the copy runs and the original's remaining kernels step aside.
    // gate: the original's escalate flag (null: always active); the job runs
    // while *gate == gate_on (the original 0, the copy 1).
    const uint32_t *gate;
    uint32_t gate_on;
    uint32_t escalation;         // the original: 1 if it has a copy to hand over to
};

// Whether a job's kernels run: always, unless it takes part in an
// escalation and its side is not the one the flag selects.  The flag is
// written once, between launches (never while a kernel reading it runs).
__device__ __forceinline__ bool job_active(const JobDev &J) {
    return !J.gate || *(volatile const uint32_t *)J.gate == J.gate_on;
}

// Host-side decomposition of an all-rows / item / group index into its job:
// `starts` holds njobs + 1 ascending offsets.
__device__ __forceinline__ uint32_t find_job(const uint32_t *starts, uint32_t njobs, uint32_t idx) {
    uint32_t lo = 0, hi = njobs;  // starts[lo] <= idx < starts[hi]
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (starts[mid] <= idx) lo = mid; else hi = mid;
    }
    return lo;
}

int kpl_for_k(uint32_t k);  // 1, 2, 4, 8 or 0 if k > 256

// Rows of padded length K1 at most this take the packed operand kernel
// (several rows per warp); the group's plan records which kernels run.
uint32_t operand_short_k1();
// The autotuner table's path for a problem, (seed_div) the fraction
// 1/seed_div of the columns the screen's threshold pass samples, and whether
// its emission pass takes the symmetric form and the 2-SM form (unless
// hm_tuning_symmetric / hm_tuning_pair force either on this thread).
int autotune_choice(uint64_t n, uint32_t d, uint32_t k, int metric, uint32_t *seed_div, bool *symmetric,
                    bool *pair, bool batched);
// Whether jobs left to the autotuner on the BF16 or TF32 screen carry a
// split-BF16 escalation copy (hm_tuning_escalation).
bool tuning_escalation();

// ------------------------------------------------------------- plain path
constexpr int PL_BM = 32;     // rows per CTA (8 warps x 4 rows)
constexpr int PL_BN = 128;    // columns per tile (32 lanes x 4)
constexpr int PL_BK = 16;     // dimensions per shared-memory stage
constexpr int PL_THREADS = 256;
constexpr int PL_ROW_PAD = 128;  // binary64 copy is padded to this many rows

// Work table of the exact path: item i = (job, group of PL_BM rows, column
// split); or, in fallback mode, each job's overflow list strided over
// `per_job` CTAs.
struct PlainWork {
    const JobDev *jobs;
    uint32_t njobs;
    const uint2 *items;     // x = job, y = group << 6 | split
    uint32_t nitems;
    uint32_t kpl;           // WarpTopK width for the largest k
    uint32_t fallback;      // 1: rows come from the jobs' overflow lists
    uint32_t per_job;       // fallback: CTAs per job
    const uint32_t *fb_jobs;  // fallback: the jobs that may have overflow rows
    uint32_t fb_njobs;
};

// PREP_CHECK_AND_NORMS: zeroes the job counters, checks every input for
// finiteness and forms the cosine row norms (all rows of every job;
// row_starts / all_rows: the all-rows space).  PREP_X64_*: the binary64 copy
// of the points, only for exact-path jobs, or (fallback mode) only for
// screened jobs whose overflow count is nonzero.
int launch_prep_jobs(const JobDev *jobs, uint32_t njobs, const uint32_t *job_blocks,
                     uint32_t total_blocks, int mode, cudaStream_t s, const uint32_t *row_starts = nullptr,
                     uint32_t all_rows = 0);
enum { PREP_CHECK_AND_NORMS = 0, PREP_X64_EXACT = 1, PREP_X64_FALLBACK = 2 };

int launch_plain(const PlainWork &w, int metric, cudaStream_t s);
// merges split lists of every exact-path job with splits > 1
int launch_merge(const JobDev *jobs, uint32_t njobs, const uint32_t *row_starts, uint32_t rows,
                 uint32_t kpl, cudaStream_t s);

// ------------------------------------------------------------- smooth kNN
// Per row of every job with smooth-kNN outputs (row_starts: all-rows space);
// rows whose rho is 0 get their unfloored sigma and are listed for the
// job's global-mean floor.
int launch_smooth(const JobDev *jobs, uint32_t njobs, const uint32_t *row_starts, uint32_t rows,
                  uint32_t kmax, cudaStream_t s);
// Sequential binary64 mean of each job's n*k distances, applied as the floor
// of its listed rows; one block per job, idle when its list is empty.
int launch_mean_all_floor(const JobDev *jobs, uint32_t njobs, cudaStream_t s);

// batch internals used by the request loop: where a bound batch keeps its
// per-job counters in the workspace, and a job's stats/status from a host
// copy of its counters
size_t batch_counters_offset(const hm_batch *B);
int batch_job_result(const hm_batch *B, uint32_t job, const JobCounters &c, hm_stats *st);
// counters of a finished single-job call (workspace `ws`), read after the
// work queued on `s`; the status is the call's (HM_ERR_INVALID for a
// non-finite input, HM_ERR_TIMEOUT for a bounded wait that gave up)
int single_job_stats(const void *ws, uint64_t n, uint32_t d, uint32_t k, int metric, int path,
                     cudaStream_t s, hm_stats *stats);

}  // namespace hm
