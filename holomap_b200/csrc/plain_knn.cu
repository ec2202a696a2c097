// plain_knn.cu -- exact kNN over every pair, in the reference's own binary64
// arithmetic, with a warp-level select on (distance bits, index) keys.
//
// Reference: src/knn.rs:22-55 (row loop, self override :35-43, sort by
// (total_cmp(dist), index) and take k :46-52), src/metric.rs:42-53 (euclidean),
// src/metric.rs:58-70 (cosine).
//
// Each pair's distance is the same sequence of correctly rounded binary64
// operations the reference performs: per dimension f64(x) - f64(y), square,
// add to a running sum that starts at +0.0, in dimension order (euclidean), or
// dot += f64(x) * f64(y) (cosine, whose per-row norm sums are precomputed in
// the same order by prep), then sqrt / divide / cast.  Dimensions past d are
// zero in the padded copy and add an exact +0.0, which leaves a sum that is
// never -0.0 unchanged.
//
// Layout: a CTA owns 32 query rows (8 warps x 4 rows) and walks the columns of
// its split 128 at a time; every lane computes a 4x4 block of pairs (rows of
// its warp x columns lane + 32c).  A warp therefore holds all 128 candidate
// keys of its 4 rows for the tile and feeds them to a warp-distributed sorted
// top-k list (WarpTopK).  Column splits (grid.y) write partial lists that
// merge_splits combines.
#include <cuda_runtime.h>

#include "hm_internal.cuh"

namespace hm {

int kpl_for_k(uint32_t k) {
    if (k <= 32) return 1;
    if (k <= 64) return 2;
    if (k <= 128) return 4;
    if (k <= 256) return 8;
    return 0;
}

// ------------------------------------------------------------------ prep
__global__ void prep_plain_kernel(const float *__restrict__ x, uint32_t n, uint32_t d,
                                  uint32_t ldd, uint32_t n_pad, double *__restrict__ x64,
                                  const uint32_t *__restrict__ gate) {
    if (gate && *gate == 0) return;  // nothing needs the binary64 copy
    const size_t total = (size_t)n_pad * ldd;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total;
         t += (size_t)gridDim.x * blockDim.x) {
        const size_t r = t / ldd, c = t % ldd;
        x64[t] = (r < n && c < d) ? (double)x[r * d + c] : 0.0;
    }
}

// sqrt of the sequential binary64 sum of squares, as the cosine metric forms
// na / nb (src/metric.rs:61-66, :69).
__global__ void row_norm_kernel(const float *__restrict__ x, uint32_t n, uint32_t d,
                                uint32_t n_pad, double *__restrict__ rnorm) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n_pad) return;
    if (r >= n) {
        rnorm[r] = 0.0;
        return;
    }
    const float *row = x + (size_t)r * d;
    double s = 0.0;
    for (uint32_t c = 0; c < d; ++c) {
        const double v = (double)row[c];
        s = __dadd_rn(s, __dmul_rn(v, v));
    }
    rnorm[r] = __dsqrt_rn(s);
}

int launch_prep_x64(const float *x, uint32_t n, uint32_t d, uint32_t ldd, uint32_t n_pad,
                    double *x64, const uint32_t *gate, cudaStream_t s) {
    ScopedKernelTimer timer(HM_KCLASS_PREP, s);
    const size_t total = (size_t)n_pad * ldd;
    const int threads = 256;
    int blocks = (int)((total + threads - 1) / threads);
    if (blocks > 148 * 16) blocks = 148 * 16;
    prep_plain_kernel<<<blocks, threads, 0, s>>>(x, n, d, ldd, n_pad, x64, gate);
    HM_CUDA_TRY(cudaGetLastError());
    count_launch();
    return HM_OK;
}

int launch_prep_plain(const float *x, uint32_t n, uint32_t d, uint32_t ldd, uint32_t n_pad,
                      int metric, double *x64, double *rnorm, cudaStream_t s) {
    if (x64) HM_TRY(launch_prep_x64(x, n, d, ldd, n_pad, x64, nullptr, s));
    ScopedKernelTimer timer(HM_KCLASS_PREP, s);
    if (metric == HM_METRIC_COSINE) {
        row_norm_kernel<<<(n_pad + 127) / 128, 128, 0, s>>>(x, n, d, n_pad, rnorm);
        HM_CUDA_TRY(cudaGetLastError());
        count_launch();
    }
    return HM_OK;
}

// ------------------------------------------------------------ the kernel
template <int METRIC>
__device__ __forceinline__ double pair_step(double acc, double a, double b) {
    if (METRIC == HM_METRIC_EUCLIDEAN) {
        const double t = __dsub_rn(a, b);
        return __dadd_rn(acc, __dmul_rn(t, t));
    } else if (METRIC == HM_METRIC_COSINE) {
        return __dadd_rn(acc, __dmul_rn(a, b));
    } else {
        return __dadd_rn(acc, fabs(__dsub_rn(a, b)));
    }
}

// Final binary64 -> binary32 step of each metric.
template <int METRIC>
__device__ __forceinline__ float pair_finish(double acc, double rn_a, double rn_b) {
    if (METRIC == HM_METRIC_EUCLIDEAN) {
        return __double2float_rn(__dsqrt_rn(acc));
    } else if (METRIC == HM_METRIC_COSINE) {
        // (1 - dot / (sqrt(na) * sqrt(nb))).max(0.0) as f32; NaN (a zero
        // vector) and any value <= 0 give +0.0.
        const double den = __dmul_rn(rn_a, rn_b);
        const double q = __ddiv_rn(acc, den);
        const double r = __dsub_rn(1.0, q);
        return (r > 0.0) ? __double2float_rn(r) : 0.0f;
    } else {
        return __double2float_rn(acc);
    }
}

template <int METRIC, int KPL>
__global__ void __launch_bounds__(PL_THREADS, (KPL <= 2 ? 2 : 1))
    plain_knn_kernel(const PlainArgs a) {
    __shared__ double As[2][PL_BM][PL_BK + 1];
    __shared__ double Bs[2][PL_BN][PL_BK + 1];
    __shared__ uint32_t s_rows[PL_BM];

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t split = blockIdx.y;
    const uint32_t c_begin = split * a.split_cols;
    const uint32_t c_end = min(a.n, c_begin + a.split_cols);
    const uint32_t ldd = a.ldd;
    const bool listed = a.row_list != nullptr;
    const uint32_t n_groups =
        listed ? (*a.row_count + PL_BM - 1) / PL_BM : (a.row_end - a.row_begin + PL_BM - 1) / PL_BM;
    const uint32_t rows_total = a.row_end - a.row_begin;

    for (uint32_t grp = blockIdx.x; grp < n_groups; grp += (listed ? gridDim.x : n_groups)) {
        // the 32 query rows of this group (0xffffffff: none)
        if (tid < PL_BM) {
            uint32_t r;
            if (listed) {
                const uint32_t at = grp * PL_BM + tid;
                r = at < *a.row_count ? a.row_list[at] : 0xffffffffu;
            } else {
                r = a.row_begin + grp * PL_BM + tid;
                if (r >= a.row_end) r = 0xffffffffu;
            }
            s_rows[tid] = r;
        }
        __syncthreads();

        WarpTopK<KPL> top[4];
#pragma unroll
        for (int r = 0; r < 4; ++r) top[r].reset();
        uint32_t my_rows[4];
        double rn_a[4];
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            my_rows[r] = s_rows[warp * 4 + r];
            rn_a[r] = (METRIC == HM_METRIC_COSINE && my_rows[r] != 0xffffffffu)
                          ? a.rnorm[my_rows[r]] : 0.0;
        }

        // loads of one stage: A 32x16 (2 per thread), B 128x16 (8 per thread)
        auto load_stage = [&](int buf, uint32_t col0, uint32_t k0) {
#pragma unroll
            for (int p = 0; p < 2; ++p) {
                const int lin = tid + p * PL_THREADS;
                const int r = lin >> 4, c = lin & 15;
                const uint32_t ar = s_rows[r] == 0xffffffffu ? 0u : s_rows[r];
                const double *src = a.x64 + (size_t)ar * ldd + k0 + c;
                const uint32_t dst = (uint32_t)__cvta_generic_to_shared(&As[buf][r][c]);
                asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(dst), "l"(src));
            }
#pragma unroll
            for (int p = 0; p < 8; ++p) {
                const int lin = tid + p * PL_THREADS;
                const int r = lin >> 4, c = lin & 15;
                const double *src = a.x64 + (size_t)(col0 + r) * ldd + k0 + c;
                const uint32_t dst = (uint32_t)__cvta_generic_to_shared(&Bs[buf][r][c]);
                asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(dst), "l"(src));
            }
            asm volatile("cp.async.commit_group;\n" ::);
        };

        const uint32_t nk = ldd / PL_BK;
        for (uint32_t col0 = c_begin; col0 < c_end; col0 += PL_BN) {
            double acc[4][4];
#pragma unroll
            for (int r = 0; r < 4; ++r)
#pragma unroll
                for (int c = 0; c < 4; ++c) acc[r][c] = 0.0;

            load_stage(0, col0, 0);
            for (uint32_t kt = 0; kt < nk; ++kt) {
                const int buf = kt & 1;
                if (kt + 1 < nk) {
                    load_stage(buf ^ 1, col0, (kt + 1) * PL_BK);
                    asm volatile("cp.async.wait_group 1;\n" ::);
                } else {
                    asm volatile("cp.async.wait_group 0;\n" ::);
                }
                __syncthreads();
#pragma unroll
                for (int kk = 0; kk < PL_BK; ++kk) {
                    double av[4], bv[4];
#pragma unroll
                    for (int r = 0; r < 4; ++r) av[r] = As[buf][warp * 4 + r][kk];
#pragma unroll
                    for (int c = 0; c < 4; ++c) bv[c] = Bs[buf][lane + 32 * c][kk];
#pragma unroll
                    for (int r = 0; r < 4; ++r)
#pragma unroll
                        for (int c = 0; c < 4; ++c)
                            acc[r][c] = pair_step<METRIC>(acc[r][c], av[r], bv[c]);
                }
                __syncthreads();
            }

            // finish the 16 pairs and feed the keys to the rows' lists
            double rn_b[4];
#pragma unroll
            for (int c = 0; c < 4; ++c)
                rn_b[c] = (METRIC == HM_METRIC_COSINE) ? a.rnorm[col0 + lane + 32 * c] : 0.0;
#pragma unroll
            for (int r = 0; r < 4; ++r) {
#pragma unroll
                for (int c = 0; c < 4; ++c) {
                    const uint32_t col = col0 + lane + 32 * c;
                    float dist = pair_finish<METRIC>(acc[r][c], rn_a[r], rn_b[c]);
                    if (col == my_rows[r]) dist = 0.0f;  // src/knn.rs:38-39
                    const uint64_t key = (col < c_end) ? make_key(dist, col) : KEY_NONE;
                    top[r].offer(key, a.k, lane);
                }
            }
        }

        // write the first k elements of each valid row
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            const uint32_t row = my_rows[r];
            if (row == 0xffffffffu) continue;
            const size_t orow = listed ? row : row - a.row_begin;
#pragma unroll
            for (int q = 0; q < KPL; ++q) {
                const uint32_t e = q * 32 + lane;
                if (e >= a.k) continue;
                const uint64_t key = top[r].v[q];
                if (a.partial) {
                    a.partial[((size_t)split * rows_total + orow) * a.k + e] = key;
                } else {
                    a.idx_out[orow * a.k + e] = key_idx(key);
                    a.dist_out[orow * a.k + e] = key_dist(key);
                }
            }
        }
        __syncthreads();  // s_rows is rewritten by the next group
    }
}

template <int METRIC>
static int launch_plain_metric(const PlainArgs &a, uint32_t splits, cudaStream_t s,
                               uint32_t grid_x = 0) {
    const uint32_t rows = a.row_end - a.row_begin;
    dim3 grid(grid_x ? grid_x : (rows + PL_BM - 1) / PL_BM, splits);
    ScopedKernelTimer timer(HM_KCLASS_BULK, s);
    switch (kpl_for_k(a.k)) {
    case 1: plain_knn_kernel<METRIC, 1><<<grid, PL_THREADS, 0, s>>>(a); break;
    case 2: plain_knn_kernel<METRIC, 2><<<grid, PL_THREADS, 0, s>>>(a); break;
    case 4: plain_knn_kernel<METRIC, 4><<<grid, PL_THREADS, 0, s>>>(a); break;
    case 8: plain_knn_kernel<METRIC, 8><<<grid, PL_THREADS, 0, s>>>(a); break;
    default: return set_error(HM_ERR_UNSUPPORTED, "k=%u exceeds 256", a.k);
    }
    HM_CUDA_TRY(cudaGetLastError());
    count_launch();
    return HM_OK;
}

int launch_plain_knn_rows(const PlainArgs &a, int metric, cudaStream_t s) {
    PlainArgs b = a;
    b.partial = nullptr;
    b.split_cols = (uint32_t)round_up(a.n, PL_BN);
    b.row_begin = 0;
    b.row_end = a.n;
    // persistent grid: groups of listed rows are strided over 2 CTAs per SM
    const uint32_t groups = (a.n + PL_BM - 1) / PL_BM;
    const uint32_t ctas = groups < 296 ? groups : 296;
    switch (metric) {
    case HM_METRIC_EUCLIDEAN: return launch_plain_metric<HM_METRIC_EUCLIDEAN>(b, 1, s, ctas);
    case HM_METRIC_COSINE: return launch_plain_metric<HM_METRIC_COSINE>(b, 1, s, ctas);
    case HM_METRIC_MANHATTAN: return launch_plain_metric<HM_METRIC_MANHATTAN>(b, 1, s, ctas);
    default: return set_error(HM_ERR_INVALID, "unknown metric %d", metric);
    }
}

int launch_plain_knn(const PlainArgs &a, int metric, uint32_t splits, cudaStream_t s) {
    switch (metric) {
    case HM_METRIC_EUCLIDEAN: return launch_plain_metric<HM_METRIC_EUCLIDEAN>(a, splits, s);
    case HM_METRIC_COSINE: return launch_plain_metric<HM_METRIC_COSINE>(a, splits, s);
    case HM_METRIC_MANHATTAN: return launch_plain_metric<HM_METRIC_MANHATTAN>(a, splits, s);
    default: return set_error(HM_ERR_INVALID, "unknown metric %d", metric);
    }
}

// ------------------------------------------------------------ split merge
// One warp per row folds the `splits` sorted partial lists into one.
template <int KPL>
__global__ void __launch_bounds__(256) merge_splits_kernel(const uint64_t *__restrict__ partial,
                                                           uint32_t rows, uint32_t k,
                                                           uint32_t splits,
                                                           uint32_t *__restrict__ idx_out,
                                                           float *__restrict__ dist_out) {
    const int lane = threadIdx.x & 31;
    const uint32_t row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (row >= rows) return;
    WarpTopK<KPL> top;
#pragma unroll
    for (int q = 0; q < KPL; ++q) {
        const uint32_t e = q * 32 + lane;
        top.v[q] = (e < k) ? partial[(size_t)row * k + e] : KEY_NONE;
    }
    top.refresh_tau(k, lane);
    for (uint32_t sp = 1; sp < splits; ++sp) {
        const uint64_t *list = partial + ((size_t)sp * rows + row) * k;
        for (uint32_t e0 = 0; e0 < k; e0 += 32) {
            const uint64_t key = (e0 + lane < k) ? list[e0 + lane] : KEY_NONE;
            if (!__any_sync(0xffffffffu, key < top.tau)) break;  // lists are sorted
            top.offer(key, k, lane);
        }
    }
#pragma unroll
    for (int q = 0; q < KPL; ++q) {
        const uint32_t e = q * 32 + lane;
        if (e < k) {
            idx_out[(size_t)row * k + e] = key_idx(top.v[q]);
            dist_out[(size_t)row * k + e] = key_dist(top.v[q]);
        }
    }
}

int launch_merge_splits(const uint64_t *partial, uint32_t rows, uint32_t k, uint32_t splits,
                        uint32_t *idx_out, float *dist_out, cudaStream_t s) {
    const int blocks = (int)((rows + 7) / 8);
    ScopedKernelTimer timer(HM_KCLASS_SELECT, s);
    switch (kpl_for_k(k)) {
    case 1: merge_splits_kernel<1><<<blocks, 256, 0, s>>>(partial, rows, k, splits, idx_out, dist_out); break;
    case 2: merge_splits_kernel<2><<<blocks, 256, 0, s>>>(partial, rows, k, splits, idx_out, dist_out); break;
    case 4: merge_splits_kernel<4><<<blocks, 256, 0, s>>>(partial, rows, k, splits, idx_out, dist_out); break;
    case 8: merge_splits_kernel<8><<<blocks, 256, 0, s>>>(partial, rows, k, splits, idx_out, dist_out); break;
    default: return set_error(HM_ERR_UNSUPPORTED, "k=%u exceeds 256", k);
    }
    HM_CUDA_TRY(cudaGetLastError());
    count_launch();
    return HM_OK;
}

}  // namespace hm
