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
// Layout: a CTA owns 32 query rows of one job (8 warps x 4 rows) and walks the
// columns of its split 128 at a time; every lane computes a 4x4 block of pairs (rows of
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
__global__ void init_counters_kernel(JobDev *jobs, uint32_t njobs) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= njobs) return;
    JobCounters c{};
    c.nonfinite_min = 0xffffffffu;
    *jobs[j].cnt = c;
}

// Binary64 copies of the points (exact-path jobs, or screened jobs with rows
// for the exact fallback).  Blocks are dealt to jobs by `job_blocks` (prefix
// offsets); each job's blocks stride over that job's elements.
__global__ void __launch_bounds__(256) prep_jobs_kernel(const JobDev *__restrict__ jobs, uint32_t njobs,
                                                        const uint32_t *__restrict__ job_blocks,
                                                        int mode) {
    const uint32_t jb = find_job(job_blocks, njobs, blockIdx.x);
    const JobDev &J = jobs[jb];
    const uint32_t lb = blockIdx.x - job_blocks[jb];
    const uint32_t nb = job_blocks[jb + 1] - job_blocks[jb];
    const size_t stride = (size_t)nb * blockDim.x;
    const size_t t0 = (size_t)lb * blockDim.x + threadIdx.x;
    if (mode == PREP_X64_EXACT && J.path != HM_PATH_PLAIN) return;
    // (an escalated job's fallback rows come from its copy's rerank: the
    // original's row list and count, so no activity check here)
    if (mode == PREP_X64_FALLBACK && (J.path == HM_PATH_PLAIN || J.cnt->ovf_count == 0)) return;
    const size_t total = (size_t)J.n_pad * J.ldd;
    for (size_t t = t0; t < total; t += stride) {
        const size_t r = t / J.ldd, c = t % J.ldd;
        J.x64[t] = (r < J.n && c < J.d) ? (double)J.x[r * J.d + c] : 0.0;
    }
}

// Input check and cosine row norms, one warp per 32 consecutive rows of the
// all-rows space (rows of several jobs may share a warp).  The warp stages its
// rows 32 dimensions at a time through shared memory with coalesced 128-byte
// reads (one row per load instruction), and lane r then walks row r's chunk in
// dimension order: the sequential binary64 sum of squares of the cosine
// metric's na / nb (src/metric.rs:61-66, :69), whose square root is kept per
// row.  Every value read is also checked for finiteness (the smallest flat
// index of a non-finite value per job, as HolomapError::NonFiniteInput
// reports it, src/api.rs:36-43).
constexpr int NRM_WARPS = 8;
__global__ void __launch_bounds__(NRM_WARPS * 32) check_norms_kernel(const JobDev *__restrict__ jobs,
                                                                    uint32_t njobs,
                                                                    const uint32_t *__restrict__ row_starts,
                                                                    uint32_t rows) {
    __shared__ float tile[NRM_WARPS][32][33];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t ar0 = (blockIdx.x * NRM_WARPS + warp) * 32;
    if (ar0 >= rows) return;
    const uint32_t ar = ar0 + lane;
    const uint32_t jb = ar < rows ? (row_starts ? find_job(row_starts, njobs, ar) : 0u) : 0u;
    const JobDev &J = jobs[jb];
    // (an escalation copy's rows are its original's: checked there)
    const bool mine = ar < rows && job_active(J);
    const uint32_t row = mine ? ar - J.arow0 : 0u;
    const uint32_t d = mine ? J.d : 0u;
    const float *xrow = J.x + (size_t)row * d;
    const bool cos = mine && J.metric == HM_METRIC_COSINE;
    const uint32_t dmax = __reduce_max_sync(0xffffffffu, d);
    double acc = 0.0;
    for (uint32_t c0 = 0; c0 < dmax; c0 += 32) {
        // row i of the warp, dimension c0 + lane: coalesced per row; all 32
        // rows' loads are issued before any is used
        float v[32];
#pragma unroll
        for (int i = 0; i < 32; ++i) {
            const float *src = reinterpret_cast<const float *>(
                __shfl_sync(0xffffffffu, reinterpret_cast<uintptr_t>(xrow), i));
            const uint32_t di = __shfl_sync(0xffffffffu, d, i);
            v[i] = (c0 + lane < di) ? src[c0 + lane] : 0.0f;
        }
        uint32_t bad = 0;
#pragma unroll
        for (int i = 0; i < 32; ++i) bad |= isfinite(v[i]) ? 0u : (1u << i);
        bad = __reduce_or_sync(0xffffffffu, bad);
        while (bad) {  // rare: a non-finite value in one of the rows
            const int i = __ffs(bad) - 1;
            bad &= bad - 1;
            const uint32_t di = __shfl_sync(0xffffffffu, d, i);
            const uint32_t ri = __shfl_sync(0xffffffffu, row, i);
            const uint32_t ji = __shfl_sync(0xffffffffu, jb, i);
            float vi = 0.0f;
#pragma unroll
            for (int q = 0; q < 32; ++q) vi = (q == i) ? v[q] : vi;
            if (c0 + lane < di && !isfinite(vi))
                atomicMin(&jobs[ji].cnt->nonfinite_min,
                          (uint32_t)min((size_t)ri * di + c0 + lane, (size_t)0xfffffffeull));
        }
#pragma unroll
        for (int i = 0; i < 32; ++i) tile[warp][i][lane] = v[i];
        __syncwarp();
        if (cos) {
            const uint32_t tmax = min(32u, d - min(d, c0));
            for (uint32_t t = 0; t < tmax; ++t) {
                const double e = (double)tile[warp][lane][t];
                acc = __dadd_rn(acc, __dmul_rn(e, e));
            }
        }
        __syncwarp();
    }
    if (cos) J.rnorm[row] = __dsqrt_rn(acc);
    // the plain path reads the norms of its padding rows [n, n_pad): zeros
    if (cos && row == J.n - 1)
        for (uint32_t r = J.n; r < J.n_pad; ++r) J.rnorm[r] = 0.0;
}

int launch_prep_jobs(const JobDev *jobs, uint32_t njobs, const uint32_t *job_blocks,
                     uint32_t total_blocks, int mode, cudaStream_t s, const uint32_t *row_starts,
                     uint32_t all_rows) {
    ScopedKernelTimer timer(HM_KCLASS_PREP, s);
    if (mode == PREP_CHECK_AND_NORMS) {
        init_counters_kernel<<<(njobs + 127) / 128, 128, 0, s>>>(const_cast<JobDev *>(jobs), njobs);
        HM_CUDA_TRY(cudaGetLastError());
        const uint32_t warps = (all_rows + 31) / 32;
        check_norms_kernel<<<(warps + NRM_WARPS - 1) / NRM_WARPS, NRM_WARPS * 32, 0, s>>>(jobs, njobs, row_starts,
                                                                                        all_rows);
        HM_CUDA_TRY(cudaGetLastError());
        count_launch(2);
        return HM_OK;
    }
    prep_jobs_kernel<<<total_blocks, 256, 0, s>>>(jobs, njobs, job_blocks, mode);
    HM_CUDA_TRY(cudaGetLastError());
    count_launch();
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
__global__ void __launch_bounds__(PL_THREADS, (KPL <= 2 ? 2 : 1)) plain_knn_kernel(const PlainWork w) {
    __shared__ double As[2][PL_BM][PL_BK + 1];
    __shared__ double Bs[2][PL_BN][PL_BK + 1];
    __shared__ uint32_t s_rows[PL_BM];

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    uint32_t jb, first_grp, grp_stride, n_groups, split = 0;
    if (!w.fallback) {
        const uint2 it = w.items[blockIdx.x];
        jb = it.x;
        first_grp = it.y >> 6;
        split = it.y & 63u;
        grp_stride = 1;
        n_groups = first_grp + 1;
    } else {
        jb = w.fb_jobs[blockIdx.x / w.per_job];
        first_grp = blockIdx.x % w.per_job;
        grp_stride = w.per_job;
        n_groups = (w.jobs[jb].cnt->ovf_count + PL_BM - 1) / PL_BM;
    }
    const JobDev &J = w.jobs[jb];
    const uint32_t c_begin = split * J.split_cols;
    const uint32_t c_end = min(J.n, c_begin + J.split_cols);
    const uint32_t ldd = J.ldd;

    for (uint32_t grp = first_grp; grp < n_groups; grp += grp_stride) {
        // the 32 query rows of this group (0xffffffff: none)
        if (tid < PL_BM) {
            uint32_t r;
            if (w.fallback) {
                const uint32_t at = grp * PL_BM + tid;
                r = at < J.cnt->ovf_count ? J.ovf_list[at] : 0xffffffffu;
            } else {
                r = grp * PL_BM + tid;
                if (r < J.q0 || r >= J.q1) r = 0xffffffffu;
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
            rn_a[r] = (METRIC == HM_METRIC_COSINE && my_rows[r] != 0xffffffffu) ? J.rnorm[my_rows[r]] : 0.0;
        }

        // loads of one stage: A 32x16 (2 per thread), B 128x16 (8 per thread)
        auto load_stage = [&](int buf, uint32_t col0, uint32_t k0) {
#pragma unroll
            for (int p = 0; p < 2; ++p) {
                const int lin = tid + p * PL_THREADS;
                const int r = lin >> 4, c = lin & 15;
                const uint32_t ar = s_rows[r] == 0xffffffffu ? 0u : s_rows[r];
                const double *src = J.x64 + (size_t)ar * ldd + k0 + c;
                const uint32_t dst = (uint32_t)__cvta_generic_to_shared(&As[buf][r][c]);
                asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(dst), "l"(src));
            }
#pragma unroll
            for (int p = 0; p < 8; ++p) {
                const int lin = tid + p * PL_THREADS;
                const int r = lin >> 4, c = lin & 15;
                const double *src = J.x64 + (size_t)(col0 + r) * ldd + k0 + c;
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
                rn_b[c] = (METRIC == HM_METRIC_COSINE) ? J.rnorm[col0 + lane + 32 * c] : 0.0;
#pragma unroll
            for (int r = 0; r < 4; ++r) {
#pragma unroll
                for (int c = 0; c < 4; ++c) {
                    const uint32_t col = col0 + lane + 32 * c;
                    float dist = pair_finish<METRIC>(acc[r][c], rn_a[r], rn_b[c]);
                    if (col == my_rows[r]) dist = 0.0f;  // src/knn.rs:38-39
                    const uint64_t key = (col < c_end) ? make_key(dist, col) : KEY_NONE;
                    top[r].offer(key, J.k, lane);
                }
            }
        }

        // write the first k elements of each valid row
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            const uint32_t row = my_rows[r];
            if (row == 0xffffffffu) continue;
#pragma unroll
            for (int q = 0; q < KPL; ++q) {
                const uint32_t e = q * 32 + lane;
                if (e >= J.k) continue;
                const uint64_t key = top[r].v[q];
                if (J.splits > 1 && !w.fallback) {
                    J.partial[((size_t)split * J.n + row) * J.k + e] = key;
                } else {
                    J.idx[(size_t)row * J.k + e] = key_idx(key);
                    J.dist[(size_t)row * J.k + e] = key_dist(key);
                }
            }
        }
        __syncthreads();  // s_rows is rewritten by the next group
    }
}

template <int METRIC>
static int launch_plain_metric(const PlainWork &w, uint32_t grid, cudaStream_t s) {
    switch (w.kpl) {
    case 1: plain_knn_kernel<METRIC, 1><<<grid, PL_THREADS, 0, s>>>(w); break;
    case 2: plain_knn_kernel<METRIC, 2><<<grid, PL_THREADS, 0, s>>>(w); break;
    case 4: plain_knn_kernel<METRIC, 4><<<grid, PL_THREADS, 0, s>>>(w); break;
    case 8: plain_knn_kernel<METRIC, 8><<<grid, PL_THREADS, 0, s>>>(w); break;
    default: return set_error(HM_ERR_UNSUPPORTED, "select width %u", w.kpl);
    }
    HM_CUDA_TRY(cudaGetLastError());
    count_launch();
    return HM_OK;
}

// One launch per metric present (the arithmetic is a template parameter);
// `w` describes that metric's items or fallback jobs.
int launch_plain(const PlainWork &w, int metric, cudaStream_t s) {
    const uint32_t grid = w.fallback ? w.fb_njobs * w.per_job : w.nitems;
    if (grid == 0) return HM_OK;
    ScopedKernelTimer timer(HM_KCLASS_EXACT, s);
    switch (metric) {
    case HM_METRIC_EUCLIDEAN: return launch_plain_metric<HM_METRIC_EUCLIDEAN>(w, grid, s);
    case HM_METRIC_COSINE: return launch_plain_metric<HM_METRIC_COSINE>(w, grid, s);
    case HM_METRIC_MANHATTAN: return launch_plain_metric<HM_METRIC_MANHATTAN>(w, grid, s);
    default: return set_error(HM_ERR_INVALID, "unknown metric %d", metric);
    }
}

// ------------------------------------------------------------ split merge
// One warp per row of an exact-path job with splits > 1 folds its split lists.
template <int KPL>
__global__ void __launch_bounds__(256) merge_splits_kernel(const JobDev *__restrict__ jobs, uint32_t njobs,
                                                           const uint32_t *__restrict__ row_starts,
                                                           uint32_t rows) {
    const int lane = threadIdx.x & 31;
    const uint32_t ar = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (ar >= rows) return;
    const uint32_t jb = row_starts ? find_job(row_starts, njobs, ar) : 0;
    const JobDev &J = jobs[jb];
    if (J.path != HM_PATH_PLAIN || J.splits <= 1) return;
    const uint32_t row = ar - J.arow0, k = J.k;
    if (row < J.q0 || row >= J.q1) return;
    WarpTopK<KPL> top;
#pragma unroll
    for (int q = 0; q < KPL; ++q) {
        const uint32_t e = q * 32 + lane;
        top.v[q] = (e < k) ? J.partial[(size_t)row * k + e] : KEY_NONE;
    }
    top.refresh_tau(k, lane);
    for (uint32_t sp = 1; sp < J.splits; ++sp) {
        const uint64_t *list = J.partial + ((size_t)sp * J.n + row) * k;
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
            J.idx[(size_t)row * k + e] = key_idx(top.v[q]);
            J.dist[(size_t)row * k + e] = key_dist(top.v[q]);
        }
    }
}

int launch_merge(const JobDev *jobs, uint32_t njobs, const uint32_t *row_starts, uint32_t rows,
                 uint32_t kpl, cudaStream_t s) {
    const int blocks = (int)((rows + 7) / 8);
    ScopedKernelTimer timer(HM_KCLASS_SELECT, s);
    switch (kpl) {
    case 1: merge_splits_kernel<1><<<blocks, 256, 0, s>>>(jobs, njobs, row_starts, rows); break;
    case 2: merge_splits_kernel<2><<<blocks, 256, 0, s>>>(jobs, njobs, row_starts, rows); break;
    case 4: merge_splits_kernel<4><<<blocks, 256, 0, s>>>(jobs, njobs, row_starts, rows); break;
    case 8: merge_splits_kernel<8><<<blocks, 256, 0, s>>>(jobs, njobs, row_starts, rows); break;
    default: return set_error(HM_ERR_UNSUPPORTED, "select width %u", kpl);
    }
    HM_CUDA_TRY(cudaGetLastError());
    count_launch();
    return HM_OK;
}

}  // namespace hm
