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

// ------------------------------------------------------------- plain path
constexpr int PL_BM = 32;     // rows per CTA (8 warps x 4 rows)
constexpr int PL_BN = 128;    // columns per tile (32 lanes x 4)
constexpr int PL_BK = 16;     // dimensions per shared-memory stage
constexpr int PL_THREADS = 256;
constexpr int PL_ROW_PAD = 128;  // binary64 copy is padded to this many rows

struct PlainArgs {
    const double *x64;    // n_pad x ldd binary64 copy, zero padded
    const double *rnorm;  // cosine: sqrt(sequential sum x^2) per row
    uint32_t n, ldd, k;
    uint32_t split_cols;  // columns per split, multiple of PL_BN
    uint32_t row_begin;   // first query row handled by this launch
    uint32_t row_end;     // one past the last query row
    uint64_t *partial;    // [splits][rows][k] keys when splits > 1
    uint32_t *idx_out;    // [rows][k] (rows counted from row_begin)
    float *dist_out;
    // Row-list mode (exact fallback of the screened path): when row_list is
    // set, the query rows are row_list[0 .. *row_count) instead of
    // [row_begin, row_end), outputs are indexed by the row itself, splits
    // must be 1 and the grid strides over groups of PL_BM listed rows.
    const uint32_t *row_list;
    const uint32_t *row_count;
};

int kpl_for_k(uint32_t k);  // 1, 2, 4, 8 or 0 if k > 256

// X (n x d f32) -> zero-padded binary64 copy (skipped when x64 is null) and,
// for cosine, the row norms.
int launch_prep_plain(const float *x, uint32_t n, uint32_t d, uint32_t ldd, uint32_t n_pad,
                      int metric, double *x64, double *rnorm, cudaStream_t s);
// The binary64 copy alone; when `gate` is set it is built only if *gate != 0
// (the screened path's fallback rows).
int launch_prep_x64(const float *x, uint32_t n, uint32_t d, uint32_t ldd, uint32_t n_pad,
                    double *x64, const uint32_t *gate, cudaStream_t s);
int launch_plain_knn(const PlainArgs &a, int metric, uint32_t splits, cudaStream_t s);
// Row-list mode with a persistent grid (the list length lives on the device).
int launch_plain_knn_rows(const PlainArgs &a, int metric, cudaStream_t s);
int launch_merge_splits(const uint64_t *partial, uint32_t rows, uint32_t k, uint32_t splits,
                        uint32_t *idx_out, float *dist_out, cudaStream_t s);

// ------------------------------------------------------------- smooth kNN
// Per-row calibration; rows whose rho is 0 get their unfloored sigma and are
// listed in zero_rows[0..*zero_count) for the global-mean floor.
int launch_smooth_knn(const float *dists, uint32_t n, uint32_t k, double target,
                      float *sigma, float *rho, uint32_t *zero_count, uint32_t *zero_rows,
                      cudaStream_t s);
// Sequential binary64 mean over all n*k distances, applied as the floor of
// the listed rows; exits at once when the list is empty.
int launch_mean_all_floor(const float *dists, uint64_t total, const uint32_t *zero_count,
                          const uint32_t *zero_rows, float *sigma, cudaStream_t s);

}  // namespace hm
