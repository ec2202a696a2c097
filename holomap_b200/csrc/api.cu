// api.cu -- the extern "C" entry points of libholomap_cuda.so.
//
// Host side of the drop-in for src/api.rs:147-148 (exact_knn + smooth_knn).
// Validation mirrors src/api.rs:114-145; the device pipeline is
//   prep -> distance bulk (plain or screened) -> [split merge] -> smooth-kNN
//   -> global-mean floor for rows without a positive distance,
// all stream-ordered, with one host<->device round trip for the host-pointer
// entry points.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>

#include "hm_internal.cuh"
#include "screen.cuh"

namespace hm {

static thread_local std::string g_last_error;

int set_error(int code, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}

void clear_error() { g_last_error.clear(); }

// ------------------------------------------------------------ validation
static int validate_knn(const void *data, uint64_t n, uint32_t d, uint32_t k, int metric) {
    if (!data) return set_error(HM_ERR_INVALID, "data is NULL");
    if (d == 0 || n == 0)
        return set_error(HM_ERR_INVALID, "bad shape: n=%llu rows of n_features=%u",
                         (unsigned long long)n, d);
    // exact_knn's own domain is 1 <= k <= n (src/knn.rs:22-55 takes the first
    // k of n sorted entries); fit_transform narrows it to k >= 2 and n > k
    // (src/api.rs:123-141) before calling it.
    if (k < 1) return set_error(HM_ERR_INVALID, "n_neighbors must be >= 1");
    if (n < k)
        return set_error(HM_ERR_INVALID, "need at least n_neighbors=%u points, got %llu", k,
                         (unsigned long long)n);
    if (metric < HM_METRIC_EUCLIDEAN || metric > HM_METRIC_MANHATTAN)
        return set_error(HM_ERR_INVALID, "unknown metric %d", metric);
    if (n > 0xffffffffull)
        return set_error(HM_ERR_UNSUPPORTED, "n=%llu exceeds the u32 index range",
                         (unsigned long long)n);
    if (kpl_for_k(k) == 0)
        return set_error(HM_ERR_UNSUPPORTED, "k=%u exceeds the largest supported k (256)", k);
    return HM_OK;
}

// ------------------------------------------------------------- workspace
static size_t align256(size_t x) { return round_up(x, 256); }

struct Layout {
    int path = HM_PATH_PLAIN;
    uint32_t ldd = 0, n_pad = 0, splits = 1, split_cols = 0;
    size_t off_flags = 0;    // Flags
    size_t off_x64 = 0, off_rnorm = 0, off_partial = 0, off_zero_rows = 0;
    size_t off_screen = 0;   // screened path workspace
    ScreenLayout screen;
    size_t total = 0;
};

// Device-side counters left in the workspace for hm_stats_from_workspace.
struct Flags {
    uint32_t zero_count;
    uint32_t nonfinite_min;   // smallest flat index of a non-finite input, or ~0
    uint32_t pad[2];
    ScreenCounters screen;
};

static int resolve_path(uint64_t n, uint32_t d, uint32_t k, int metric, int path) {
    if (path == HM_PATH_AUTO) return hm_autotune_path(n, d, k, metric);
    return path;
}

static int plan(uint64_t n, uint32_t d, uint32_t k, int metric, int path, Layout &L) {
    L.path = resolve_path(n, d, k, metric, path);
    if (L.path < HM_PATH_PLAIN || L.path > HM_PATH_SCREEN_BF16X3)
        return set_error(HM_ERR_INVALID, "unknown path %d", path);
    if (L.path != HM_PATH_PLAIN && metric == HM_METRIC_MANHATTAN)
        return set_error(HM_ERR_UNSUPPORTED,
                         "manhattan has no inner-product form; use the plain path");
    L.ldd = (uint32_t)round_up(d, PL_BK);
    L.n_pad = (uint32_t)(round_up(n, PL_ROW_PAD) + PL_ROW_PAD);
    const uint32_t row_blocks = (uint32_t)((n + PL_BM - 1) / PL_BM);
    const uint32_t col_tiles = (uint32_t)((n + PL_BN - 1) / PL_BN);
    uint32_t splits = (1184 + row_blocks - 1) / row_blocks;  // ~4 CTAs per SM slot
    uint32_t max_splits = col_tiles / 2 ? col_tiles / 2 : 1;
    if (splits > max_splits) splits = max_splits;
    if (splits > 32) splits = 32;
    if (splits < 1) splits = 1;
    L.split_cols = (uint32_t)round_up((n + splits - 1) / splits, PL_BN);
    L.splits = (uint32_t)((n + L.split_cols - 1) / L.split_cols);

    size_t off = 0;
    L.off_flags = off;
    off = align256(off + sizeof(Flags));
    L.off_zero_rows = off;
    off = align256(off + n * sizeof(uint32_t));
    L.off_x64 = off;
    off = align256(off + (size_t)L.n_pad * L.ldd * sizeof(double));
    L.off_rnorm = off;
    off = align256(off + (size_t)L.n_pad * sizeof(double));
    L.off_partial = off;
    if (L.splits > 1) off = align256(off + (size_t)L.splits * n * k * sizeof(uint64_t));
    L.off_screen = off;
    if (L.path != HM_PATH_PLAIN) {
        HM_TRY(screen_plan(n, d, k, metric, L.path, L.screen));
        off = align256(off + L.screen.total);
    }
    L.total = off;
    return HM_OK;
}

// ------------------------------------------------------- device pipeline
__global__ void check_finite_kernel(const float *__restrict__ x, uint64_t total,
                                    uint32_t *__restrict__ first_bad) {
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < total;
         t += (uint64_t)gridDim.x * blockDim.x) {
        if (!isfinite(x[t])) atomicMin(first_bad, (uint32_t)(t < 0xfffffffeull ? t : 0xfffffffeull));
    }
}

__global__ void init_flags_kernel(Flags *f) {
    if (threadIdx.x == 0) {
        f->zero_count = 0;
        f->nonfinite_min = 0xffffffffu;
        f->screen = ScreenCounters{};
    }
}

static int run_knn(const float *d_data, uint64_t n, uint32_t d, uint32_t k, int metric,
                   const Layout &L, char *ws, uint32_t *d_idx, float *d_dist, cudaStream_t s) {
    Flags *flags = reinterpret_cast<Flags *>(ws + L.off_flags);
    {
        ScopedKernelTimer timer(HM_KCLASS_PREP, s);
        init_flags_kernel<<<1, 32, 0, s>>>(flags);
        HM_CUDA_TRY(cudaGetLastError());
        const uint64_t total = n * (uint64_t)d;
        int blocks = (int)((total + 255) / 256);
        if (blocks > 148 * 8) blocks = 148 * 8;
        check_finite_kernel<<<blocks, 256, 0, s>>>(d_data, total, &flags->nonfinite_min);
        HM_CUDA_TRY(cudaGetLastError());
        count_launch(2);
    }
    double *x64 = reinterpret_cast<double *>(ws + L.off_x64);
    double *rnorm = reinterpret_cast<double *>(ws + L.off_rnorm);
    // the screened path builds the binary64 copy only if its fallback needs it
    HM_TRY(launch_prep_plain(d_data, (uint32_t)n, d, L.ldd, L.n_pad, metric,
                             L.path == HM_PATH_PLAIN ? x64 : nullptr, rnorm, s));

    if (L.path == HM_PATH_PLAIN) {
        PlainArgs a{};
        a.x64 = x64;
        a.rnorm = rnorm;
        a.n = (uint32_t)n;
        a.ldd = L.ldd;
        a.k = k;
        a.split_cols = L.split_cols;
        a.row_begin = 0;
        a.row_end = (uint32_t)n;
        a.partial = L.splits > 1 ? reinterpret_cast<uint64_t *>(ws + L.off_partial) : nullptr;
        a.idx_out = d_idx;
        a.dist_out = d_dist;
        a.row_list = nullptr;
        a.row_count = nullptr;
        HM_TRY(launch_plain_knn(a, metric, L.splits, s));
        if (L.splits > 1)
            HM_TRY(launch_merge_splits(a.partial, (uint32_t)n, k, L.splits, d_idx, d_dist, s));
        return HM_OK;
    }
    ScreenRun r{};
    r.data = d_data;
    r.x64 = x64;
    r.rnorm = rnorm;
    r.n = (uint32_t)n;
    r.d = d;
    r.ldd = L.ldd;
    r.n_pad = L.n_pad;
    r.k = k;
    r.metric = metric;
    r.path = L.path;
    r.idx_out = d_idx;
    r.dist_out = d_dist;
    r.counters = &flags->screen;
    return screen_run(r, L.screen, ws + L.off_screen, s);
}

static int run_smooth(const float *d_dist, uint64_t n, uint32_t k, float *d_sigma, float *d_rho,
                      uint32_t *zero_count, uint32_t *zero_rows, cudaStream_t s) {
    const double target = std::log2((double)k);  // src/smooth_knn.rs:25 (platform log2)
    HM_TRY(launch_smooth_knn(d_dist, (uint32_t)n, k, target, d_sigma, d_rho, zero_count,
                             zero_rows, s));
    HM_TRY(launch_mean_all_floor(d_dist, n * (uint64_t)k, zero_count, zero_rows, d_sigma, s));
    return HM_OK;
}

// ---------------------------------------------- per-thread device context
struct ThreadCtx {
    int device = -1;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    ~ThreadCtx() {
        // streams/events die with the context at process exit; nothing to do
    }
};
static thread_local ThreadCtx g_ctx;

static int thread_ctx(ThreadCtx *&out) {
    int dev = 0;
    HM_CUDA_TRY(cudaGetDevice(&dev));
    if (g_ctx.device != dev || !g_ctx.stream) {
        HM_CUDA_TRY(cudaStreamCreateWithFlags(&g_ctx.stream, cudaStreamNonBlocking));
        HM_CUDA_TRY(cudaEventCreate(&g_ctx.ev0));
        HM_CUDA_TRY(cudaEventCreate(&g_ctx.ev1));
        // keep freed stream-ordered allocations cached in the device pool
        cudaMemPool_t pool;
        if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
            uint64_t threshold = ~0ull;
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &threshold);
        }
        g_ctx.device = dev;
    }
    out = &g_ctx;
    return HM_OK;
}

// RAII list of stream-ordered allocations, freed on every exit path.
struct Allocs {
    cudaStream_t s;
    void *p[8] = {};
    int count = 0;
    explicit Allocs(cudaStream_t st) : s(st) {}
    int get(void **out, size_t bytes) {
        cudaError_t e = cudaMallocAsync(out, bytes ? bytes : 256, s);
        if (e != cudaSuccess)
            return set_error(e == cudaErrorMemoryAllocation ? HM_ERR_OOM : HM_ERR_CUDA,
                             "cudaMallocAsync(%zu): %s", bytes, cudaGetErrorString(e));
        p[count++] = *out;
        return HM_OK;
    }
    ~Allocs() {
        for (int i = 0; i < count; ++i) cudaFreeAsync(p[i], s);
        cudaStreamSynchronize(s);
    }
};

static void fill_stats(hm_stats *st, const Layout &L, const Flags &f, uint64_t n) {
    if (!st) return;
    st->path_used = L.path;
    st->col_splits = L.splits;
    st->zero_rho_rows = f.zero_count;
    st->candidate_cap = L.path == HM_PATH_PLAIN ? 0 : L.screen.cap;
    st->candidates_total = f.screen.candidates;
    st->candidates_max_row = f.screen.max_row;
    st->overflow_rows = f.screen.overflow_rows;
    st->candidates_emitted = f.screen.emitted;
    float band = 0.f;
    memcpy(&band, &f.screen.band_max_bits, sizeof band);
    st->screen_band = L.path == HM_PATH_PLAIN ? 0.0 : (double)band;
    (void)n;
}

static int host_pipeline(const float *data, uint64_t n, uint32_t d, uint32_t k, int metric,
                         int path, uint32_t *idx_out, float *dist_out, float *sigma_out,
                         float *rho_out, hm_stats *stats) {
    HM_TRY(validate_knn(data, n, d, k, metric));
    if (!idx_out || !dist_out) return set_error(HM_ERR_INVALID, "output pointer is NULL");
    Layout L;
    HM_TRY(plan(n, d, k, metric, path, L));
    ThreadCtx *ctx;
    HM_TRY(thread_ctx(ctx));
    cudaStream_t s = ctx->stream;
    const bool smooth = sigma_out && rho_out;
    int rc = HM_OK;
    Flags flags{};
    {
        Allocs A(s);
        void *d_data, *d_idx, *d_dist, *d_sigma = nullptr, *d_rho = nullptr, *ws;
        HM_TRY(A.get(&d_data, n * d * sizeof(float)));
        HM_TRY(A.get(&d_idx, n * k * sizeof(uint32_t)));
        HM_TRY(A.get(&d_dist, n * k * sizeof(float)));
        if (smooth) {
            HM_TRY(A.get(&d_sigma, n * sizeof(float)));
            HM_TRY(A.get(&d_rho, n * sizeof(float)));
        }
        HM_TRY(A.get(&ws, L.total));
        HM_CUDA_TRY(cudaMemcpyAsync(d_data, data, n * d * sizeof(float), cudaMemcpyHostToDevice, s));
        HM_CUDA_TRY(cudaEventRecord(ctx->ev0, s));
        char *w = static_cast<char *>(ws);
        rc = run_knn(static_cast<float *>(d_data), n, d, k, metric, L, w,
                     static_cast<uint32_t *>(d_idx), static_cast<float *>(d_dist), s);
        if (rc == HM_OK && smooth) {
            Flags *f = reinterpret_cast<Flags *>(w + L.off_flags);
            rc = run_smooth(static_cast<float *>(d_dist), n, k, static_cast<float *>(d_sigma),
                            static_cast<float *>(d_rho), &f->zero_count,
                            reinterpret_cast<uint32_t *>(w + L.off_zero_rows), s);
        }
        if (rc != HM_OK) return rc;
        HM_CUDA_TRY(cudaEventRecord(ctx->ev1, s));
        HM_CUDA_TRY(cudaMemcpyAsync(idx_out, d_idx, n * k * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
        HM_CUDA_TRY(cudaMemcpyAsync(dist_out, d_dist, n * k * sizeof(float), cudaMemcpyDeviceToHost, s));
        if (smooth) {
            HM_CUDA_TRY(cudaMemcpyAsync(sigma_out, d_sigma, n * sizeof(float), cudaMemcpyDeviceToHost, s));
            HM_CUDA_TRY(cudaMemcpyAsync(rho_out, d_rho, n * sizeof(float), cudaMemcpyDeviceToHost, s));
        }
        HM_CUDA_TRY(cudaMemcpyAsync(&flags, w + L.off_flags, sizeof(Flags), cudaMemcpyDeviceToHost, s));
        HM_CUDA_TRY(cudaStreamSynchronize(s));
        if (stats) {
            float ms = 0.f;
            cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
            stats->device_ms = ms;
        }
    }
    if (flags.nonfinite_min != 0xffffffffu)
        return set_error(HM_ERR_INVALID, "data contains a non-finite value at index %u",
                         flags.nonfinite_min);
    if (flags.screen.error_code)
        return set_error(HM_ERR_TIMEOUT, "screen kernel gave up waiting (code %u)",
                         flags.screen.error_code);
    fill_stats(stats, L, flags, n);
    return HM_OK;
}

}  // namespace hm

using namespace hm;

extern "C" {

int hm_abi_version(void) { return HM_ABI_VERSION; }

const char *hm_last_error(void) { return g_last_error.c_str(); }

int hm_knn(const float *data, uint64_t n, uint32_t d, uint32_t k, int metric, int path,
           uint32_t *idx_out, float *dist_out, hm_stats *stats) {
    clear_error();
    return host_pipeline(data, n, d, k, metric, path, idx_out, dist_out, nullptr, nullptr,
                         stats);
}

int hm_knn_smooth(const float *data, uint64_t n, uint32_t d, uint32_t k, int metric, int path,
                  uint32_t *idx_out, float *dist_out, float *sigma_out, float *rho_out,
                  hm_stats *stats) {
    clear_error();
    if (!sigma_out || !rho_out) return set_error(HM_ERR_INVALID, "sigma/rho output is NULL");
    return host_pipeline(data, n, d, k, metric, path, idx_out, dist_out, sigma_out, rho_out,
                         stats);
}

size_t hm_smooth_workspace_bytes(uint64_t n) {
    return align256(sizeof(uint32_t) * 4) + align256(n * sizeof(uint32_t));
}

int hm_smooth_knn_device(const float *d_dists, uint64_t n, uint32_t k, float *d_sigma,
                         float *d_rho, void *d_workspace, void *stream) {
    clear_error();
    if (!d_dists || !d_sigma || !d_rho || !d_workspace)
        return set_error(HM_ERR_INVALID, "NULL pointer argument");
    if (n == 0 || k == 0) return set_error(HM_ERR_INVALID, "empty distance matrix");
    if (n > 0xffffffffull) return set_error(HM_ERR_UNSUPPORTED, "n exceeds the u32 range");
    char *w = static_cast<char *>(d_workspace);
    return run_smooth(d_dists, n, k, d_sigma, d_rho, reinterpret_cast<uint32_t *>(w),
                      reinterpret_cast<uint32_t *>(w + align256(sizeof(uint32_t) * 4)),
                      static_cast<cudaStream_t>(stream));
}

int hm_smooth_knn(const float *dists, uint64_t n, uint32_t k, float *sigma_out, float *rho_out) {
    clear_error();
    if (!dists || !sigma_out || !rho_out) return set_error(HM_ERR_INVALID, "NULL pointer argument");
    if (n == 0 || k == 0) return set_error(HM_ERR_INVALID, "empty distance matrix");
    ThreadCtx *ctx;
    HM_TRY(thread_ctx(ctx));
    cudaStream_t s = ctx->stream;
    Allocs A(s);
    void *d_dists, *d_sigma, *d_rho, *ws;
    HM_TRY(A.get(&d_dists, n * k * sizeof(float)));
    HM_TRY(A.get(&d_sigma, n * sizeof(float)));
    HM_TRY(A.get(&d_rho, n * sizeof(float)));
    HM_TRY(A.get(&ws, hm_smooth_workspace_bytes(n)));
    HM_CUDA_TRY(cudaMemcpyAsync(d_dists, dists, n * k * sizeof(float), cudaMemcpyHostToDevice, s));
    HM_TRY(hm_smooth_knn_device(static_cast<float *>(d_dists), n, k, static_cast<float *>(d_sigma),
                                static_cast<float *>(d_rho), ws, s));
    HM_CUDA_TRY(cudaMemcpyAsync(sigma_out, d_sigma, n * sizeof(float), cudaMemcpyDeviceToHost, s));
    HM_CUDA_TRY(cudaMemcpyAsync(rho_out, d_rho, n * sizeof(float), cudaMemcpyDeviceToHost, s));
    HM_CUDA_TRY(cudaStreamSynchronize(s));
    return HM_OK;
}

size_t hm_workspace_bytes(uint64_t n, uint32_t d, uint32_t k, int metric, int path) {
    clear_error();
    if (validate_knn((const void *)1, n, d, k, metric) != HM_OK) return 0;
    Layout L;
    if (plan(n, d, k, metric, path, L) != HM_OK) return 0;
    return L.total;
}

int hm_knn_smooth_device(const float *d_data, uint64_t n, uint32_t d, uint32_t k, int metric,
                         int path, uint32_t *d_idx, float *d_dist, float *d_sigma, float *d_rho,
                         void *d_workspace, size_t workspace_bytes, void *stream,
                         hm_stats *stats) {
    clear_error();
    HM_TRY(validate_knn(d_data, n, d, k, metric));
    if (!d_idx || !d_dist || !d_workspace)
        return set_error(HM_ERR_INVALID, "NULL pointer argument");
    Layout L;
    HM_TRY(plan(n, d, k, metric, path, L));
    if (workspace_bytes < L.total)
        return set_error(HM_ERR_INVALID, "workspace of %zu bytes is below the %zu needed",
                         workspace_bytes, L.total);
    if (reinterpret_cast<uintptr_t>(d_workspace) % 256)
        return set_error(HM_ERR_INVALID, "workspace must be 256-byte aligned");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    char *w = static_cast<char *>(d_workspace);
    HM_TRY(run_knn(d_data, n, d, k, metric, L, w, d_idx, d_dist, s));
    if (d_sigma && d_rho) {
        Flags *f = reinterpret_cast<Flags *>(w + L.off_flags);
        HM_TRY(run_smooth(d_dist, n, k, d_sigma, d_rho, &f->zero_count,
                          reinterpret_cast<uint32_t *>(w + L.off_zero_rows), s));
    }
    if (stats) {
        memset(stats, 0, sizeof *stats);
        stats->path_used = L.path;
        stats->col_splits = L.splits;
        stats->candidate_cap = L.path == HM_PATH_PLAIN ? 0 : L.screen.cap;
    }
    return HM_OK;
}

int hm_stats_from_workspace(const void *d_workspace, uint64_t n, uint32_t d, uint32_t k,
                            int metric, int path, hm_stats *stats) {
    clear_error();
    if (!d_workspace || !stats) return set_error(HM_ERR_INVALID, "NULL pointer argument");
    HM_TRY(validate_knn((const void *)1, n, d, k, metric));
    Layout L;
    HM_TRY(plan(n, d, k, metric, path, L));
    Flags f{};
    HM_CUDA_TRY(cudaMemcpy(&f, static_cast<const char *>(d_workspace) + L.off_flags, sizeof f,
                           cudaMemcpyDeviceToHost));
    memset(stats, 0, sizeof *stats);
    fill_stats(stats, L, f, n);
    if (f.nonfinite_min != 0xffffffffu)
        return set_error(HM_ERR_INVALID, "data contains a non-finite value at index %u",
                         f.nonfinite_min);
    return HM_OK;
}

}  // extern "C"
