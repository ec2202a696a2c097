// smooth_knn.cu -- smooth-kNN calibration (rho, sigma) on the device.
//
// Reference: src/smooth_knn.rs:23-80 (per-row rho, 64-step binary32 bisection,
// MIN_K_DIST_SCALE floors), mean at :82-84, and libm::expf reached through
// src/fmath.rs:119-122.
//
// Rows of jobs with k <= 32 take four lanes each (smooth_knn_quad_kernel: the
// row in registers, exp terms in parallel, the adds in the reference's order),
// or one thread each when the rows alone fill the device
// (smooth_knn_row_kernel).  Larger k: one warp per
// row (of any job).  Lanes evaluate the row's exp terms in parallel; the
// binary32 partial sum is then formed in the reference's order (j = 1, 2, ...,
// k-1, each add rounded) by broadcasting the terms, so every lane holds the
// same psum and all control flow is warp-uniform.  All arithmetic uses
// explicitly rounded intrinsics and the file is compiled without FMA
// contraction or flush-to-zero.
#include <cuda_runtime.h>

#include "hm_internal.cuh"
#include "libm_expf.cuh"

namespace hm {

// One warp per row of the all-rows space; the row's values are read per
// 32-element chunk from global memory (L1 resident after the first pass).
__global__ void __launch_bounds__(256) smooth_knn_kernel(const JobDev *__restrict__ jobs, uint32_t njobs,
                                                         const uint32_t *__restrict__ row_starts,
                                                         uint32_t rows) {
    const int lane = threadIdx.x & 31;
    const uint32_t ar = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (ar >= rows) return;
    const JobDev &J = jobs[row_starts ? find_job(row_starts, njobs, ar) : 0];
    if (!J.sigma || !J.rho || J.k <= 32) return;  // k <= 32: the row kernels
    const uint32_t row = ar - J.arow0, k = J.k;
    const double target = J.target;
    const float *v = J.dist + (size_t)row * k;
    const uint32_t chunks = (k + 31) / 32;

    // rho: first positive distance in row order, else 0 (src/smooth_knn.rs:35)
    float rh = 0.0f;
    for (uint32_t ch = 0; ch < chunks; ++ch) {
        const uint32_t j = ch * 32 + lane;
        const float x = (j < k) ? v[j] : 0.0f;
        const unsigned m = __ballot_sync(0xffffffffu, x > 0.0f);
        if (m) {
            rh = __shfl_sync(0xffffffffu, x, __ffs(m) - 1);
            break;
        }
    }

    // bisection, binary32 state, hi seeded at f32::MAX (src/smooth_knn.rs:39-65)
    const float f32max = __uint_as_float(0x7f7fffffu);
    float lo = 0.0f, hi = f32max, mid = 1.0f;
    for (int it = 0; it < 64; ++it) {
        float psum = 0.0f;
        for (uint32_t ch = 0; ch < chunks; ++ch) {
            const uint32_t j = ch * 32 + lane;
            float term = 0.0f;
            if (j >= 1 && j < k) {
                const float dd = __fsub_rn(v[j], rh);
                term = (dd > 0.0f) ? expf_libm(-__fdiv_rn(dd, mid)) : 1.0f;
            }
            const uint32_t j_lo = (ch == 0) ? 1u : 0u;
            const uint32_t j_hi = min(32u, k - ch * 32);
            for (uint32_t l = j_lo; l < j_hi; ++l)
                psum = __fadd_rn(psum, __shfl_sync(0xffffffffu, term, (int)l));
        }
        const double ps = (double)psum;
        if (fabs(__dsub_rn(ps, target)) < 1e-5) break;
        if (ps > target) {
            hi = mid;
            mid = __fdiv_rn(__fadd_rn(lo, hi), 2.0f);
        } else {
            lo = mid;
            if (hi >= f32max)
                mid = __fmul_rn(mid, 2.0f);
            else
                mid = __fdiv_rn(__fadd_rn(lo, hi), 2.0f);
        }
    }

    float sg = mid;
    if (rh > 0.0f) {
        // floor = 1e-3 * mean(row), mean = f32(sequential f64 sum / k)
        double s = 0.0;
        for (uint32_t ch = 0; ch < chunks; ++ch) {
            const uint32_t j = ch * 32 + lane;
            const float x = (j < k) ? v[j] : 0.0f;
            const uint32_t j_hi = min(32u, k - ch * 32);
            for (uint32_t l = 0; l < j_hi; ++l)
                s = __dadd_rn(s, (double)__shfl_sync(0xffffffffu, x, (int)l));
        }
        const float mean_row = __double2float_rn(__ddiv_rn(s, (double)k));
        const float floor_v = __fmul_rn(1e-3f, mean_row);
        if (sg < floor_v) sg = floor_v;
    } else if (lane == 0) {
        // floored later with the job's global mean (mean_all_floor_kernel)
        const uint32_t slot = atomicAdd(&J.cnt->zero_count, 1u);
        J.zero_rows[slot] = row;
    }
    if (lane == 0) {
        J.sigma[row] = sg;
        J.rho[row] = rh;
    }
}

// One thread per row for k <= KC: the row stays in registers and the whole
// calibration is the reference's sequential loop, with no shuffles.  Rows of
// jobs with k > KC are left to smooth_knn_kernel.
// k <= KC (16 or 32), many rows: one thread per row, the row in registers and
// the reference's loop as written.
template <int KC>
__global__ void __launch_bounds__(128) smooth_knn_row_kernel(const JobDev *__restrict__ jobs, uint32_t njobs,
                                                             const uint32_t *__restrict__ row_starts,
                                                             uint32_t rows) {
    const uint32_t ar = blockIdx.x * blockDim.x + threadIdx.x;
    if (ar >= rows) return;
    const JobDev &J = jobs[row_starts ? find_job(row_starts, njobs, ar) : 0];
    if (!J.sigma || !J.rho || J.k > KC) return;
    const uint32_t row = ar - J.arow0, k = J.k;
    const double target = J.target;
    const float *src = J.dist + (size_t)row * k;
    float v[KC];
#pragma unroll
    for (int j = 0; j < KC; ++j) v[j] = (j < (int)k) ? src[j] : 0.0f;

    // rho: first positive distance in row order, else 0 (src/smooth_knn.rs:35)
    float rh = 0.0f;
    bool found = false;
#pragma unroll
    for (int j = 0; j < KC; ++j) {
        if (!found && j < (int)k && v[j] > 0.0f) {
            rh = v[j];
            found = true;
        }
    }
    // bisection, binary32 state, hi seeded at f32::MAX (src/smooth_knn.rs:39-65)
    const float f32max = __uint_as_float(0x7f7fffffu);
    float lo = 0.0f, hi = f32max, mid = 1.0f;
    for (int it = 0; it < 64; ++it) {
        float psum = 0.0f;
#pragma unroll
        for (int j = 1; j < KC; ++j) {
            if (j < (int)k) {
                const float dd = __fsub_rn(v[j], rh);
                psum = __fadd_rn(psum, (dd > 0.0f) ? expf_libm(-__fdiv_rn(dd, mid)) : 1.0f);
            }
        }
        const double ps = (double)psum;
        if (fabs(__dsub_rn(ps, target)) < 1e-5) break;
        if (ps > target) {
            hi = mid;
            mid = __fdiv_rn(__fadd_rn(lo, hi), 2.0f);
        } else {
            lo = mid;
            if (hi >= f32max)
                mid = __fmul_rn(mid, 2.0f);
            else
                mid = __fdiv_rn(__fadd_rn(lo, hi), 2.0f);
        }
    }
    float sg = mid;
    if (rh > 0.0f) {
        // floor = 1e-3 * mean(row), mean = f32(sequential f64 sum / k)
        double s = 0.0;
#pragma unroll
        for (int j = 0; j < KC; ++j)
            if (j < (int)k) s = __dadd_rn(s, (double)v[j]);
        const float floor_v = __fmul_rn(1e-3f, __double2float_rn(__ddiv_rn(s, (double)k)));
        if (sg < floor_v) sg = floor_v;
    } else {
        // floored later with the job's global mean (mean_all_floor_kernel)
        const uint32_t slot = atomicAdd(&J.cnt->zero_count, 1u);
        J.zero_rows[slot] = row;
    }
    J.sigma[row] = sg;
    J.rho[row] = rh;
}

// k <= KC (16 or 32): four lanes per row.  Lane q of a row holds the row's
// values j = 4 i + q and evaluates their exp terms; every lane then forms the
// binary32 partial sum in the reference's order (j = 1, ..., k - 1, each add
// rounded) from the four lanes' terms, so the four lanes hold the same psum
// and take the same branches (shuffles stay within the row's lanes).
template <int KC>
__global__ void __launch_bounds__(128) smooth_knn_quad_kernel(const JobDev *__restrict__ jobs, uint32_t njobs,
                                                              const uint32_t *__restrict__ row_starts,
                                                              uint32_t rows) {
    constexpr int NV = KC / 4;
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t ar = tid >> 2, q = tid & 3;
    if (ar >= rows) return;  // the row's four lanes leave together
    const JobDev &J = jobs[row_starts ? find_job(row_starts, njobs, ar) : 0];
    if (!J.sigma || !J.rho || J.k > KC) return;
    const unsigned gmask = 0xfu << (threadIdx.x & 28u);
    const uint32_t row = ar - J.arow0, k = J.k;
    const double target = J.target;
    const float *src = J.dist + (size_t)row * k;
    float v[NV];
#pragma unroll
    for (int i = 0; i < NV; ++i) {
        const uint32_t j = 4 * i + q;
        v[i] = j < k ? src[j] : 0.0f;
    }
    // value j of the row, from the lane that holds it
    auto at = [&](int j) { return __shfl_sync(gmask, v[j >> 2], j & 3, 4); };

    // rho: first positive distance in row order, else 0 (src/smooth_knn.rs:35)
    float rh = 0.0f;
#pragma unroll
    for (int j = 0; j < KC; ++j) {
        const float x = at(j);
        if (rh == 0.0f && j < (int)k && x > 0.0f) rh = x;
    }
    // bisection, binary32 state, hi seeded at f32::MAX (src/smooth_knn.rs:39-65)
    const float f32max = __uint_as_float(0x7f7fffffu);
    float lo = 0.0f, hi = f32max, mid = 1.0f;
    for (int it = 0; it < 64; ++it) {
        float term[NV];
#pragma unroll
        for (int i = 0; i < NV; ++i) {
            const float dd = __fsub_rn(v[i], rh);
            term[i] = (dd > 0.0f) ? expf_libm(-__fdiv_rn(dd, mid)) : 1.0f;
        }
        float psum = 0.0f;
#pragma unroll
        for (int j = 1; j < KC; ++j) {
            const float t = __shfl_sync(gmask, term[j >> 2], j & 3, 4);
            if (j < (int)k) psum = __fadd_rn(psum, t);
        }
        const double ps = (double)psum;
        if (fabs(__dsub_rn(ps, target)) < 1e-5) break;
        if (ps > target) {
            hi = mid;
            mid = __fdiv_rn(__fadd_rn(lo, hi), 2.0f);
        } else {
            lo = mid;
            if (hi >= f32max)
                mid = __fmul_rn(mid, 2.0f);
            else
                mid = __fdiv_rn(__fadd_rn(lo, hi), 2.0f);
        }
    }
    float sg = mid;
    if (rh > 0.0f) {
        // floor = 1e-3 * mean(row), mean = f32(sequential f64 sum / k)
        double s = 0.0;
#pragma unroll
        for (int j = 0; j < KC; ++j) {
            const float x = at(j);
            if (j < (int)k) s = __dadd_rn(s, (double)x);
        }
        const float floor_v = __fmul_rn(1e-3f, __double2float_rn(__ddiv_rn(s, (double)k)));
        if (sg < floor_v) sg = floor_v;
    } else if (q == 0) {
        // floored later with the job's global mean (mean_all_floor_kernel)
        const uint32_t slot = atomicAdd(&J.cnt->zero_count, 1u);
        J.zero_rows[slot] = row;
    }
    if (q == 0) {
        J.sigma[row] = sg;
        J.rho[row] = rh;
    }
}

int launch_smooth(const JobDev *jobs, uint32_t njobs, const uint32_t *row_starts, uint32_t rows,
                  uint32_t kmax, cudaStream_t s) {
    ScopedKernelTimer timer(HM_KCLASS_SMOOTH, s);
    // every job with k <= 32 (the kernel returns for rows of larger k)
    // four lanes per row unless the rows alone fill the device (then the
    // extra lanes' shuffles cost more than the shorter exp chains save)
    const bool quad = rows < (1u << 17);
    if (kmax <= 16) {
        if (quad)
            smooth_knn_quad_kernel<16><<<(rows + 31) / 32, 128, 0, s>>>(jobs, njobs, row_starts, rows);
        else
            smooth_knn_row_kernel<16><<<(rows + 127) / 128, 128, 0, s>>>(jobs, njobs, row_starts, rows);
    } else {
        if (quad)
            smooth_knn_quad_kernel<32><<<(rows + 31) / 32, 128, 0, s>>>(jobs, njobs, row_starts, rows);
        else
            smooth_knn_row_kernel<32><<<(rows + 127) / 128, 128, 0, s>>>(jobs, njobs, row_starts, rows);
    }
    HM_CUDA_TRY(cudaGetLastError());
    count_launch();
    if (kmax > 32) {  // rows of jobs with k > 32, one warp per row
        smooth_knn_kernel<<<(int)((rows + 7) / 8), 256, 0, s>>>(jobs, njobs, row_starts, rows);
        HM_CUDA_TRY(cudaGetLastError());
        count_launch();
    }
    return HM_OK;
}

// mean_all = f32(sequential binary64 sum of all n*k distances / (n*k))
// (src/smooth_knn.rs:26, :82-84).  The reference's order is one dependent
// chain, so one thread forms it; the other 255 threads of the job's block
// stage the next values through shared memory.  Idle when no row of the job
// had rho == 0.
__global__ void __launch_bounds__(256) mean_all_floor_kernel(const JobDev *__restrict__ jobs) {
    const JobDev &J = jobs[blockIdx.x];
    if (!J.sigma || !J.rho) return;
    const uint32_t cnt = J.cnt->zero_count;
    if (cnt == 0) return;
    __shared__ float stage[2][2048];
    __shared__ float floor_v;
    const float *dists = J.dist;
    const uint64_t total = (uint64_t)J.n * J.k;
    double s = 0.0;
    const uint64_t chunk = 2048;
    for (uint64_t base = 0; base < total; base += chunk) {
        const int buf = (int)((base / chunk) & 1);
        const uint64_t len = min(chunk, total - base);
        for (uint64_t t = threadIdx.x; t < len; t += blockDim.x) stage[buf][t] = dists[base + t];
        __syncthreads();
        if (threadIdx.x == 0)
            for (uint64_t t = 0; t < len; ++t) s = __dadd_rn(s, (double)stage[buf][t]);
        // the double buffer lets the next fill overlap the chain; the barrier
        // of the iteration after next protects reuse
    }
    if (threadIdx.x == 0) {
        const float mean_all = __double2float_rn(__ddiv_rn(s, (double)total));
        floor_v = __fmul_rn(1e-3f, mean_all);
    }
    __syncthreads();
    for (uint32_t t = threadIdx.x; t < cnt; t += blockDim.x) {
        const uint32_t row = J.zero_rows[t];
        if (J.sigma[row] < floor_v) J.sigma[row] = floor_v;
    }
}

int launch_mean_all_floor(const JobDev *jobs, uint32_t njobs, cudaStream_t s) {
    ScopedKernelTimer timer(HM_KCLASS_SMOOTH, s);
    mean_all_floor_kernel<<<njobs, 256, 0, s>>>(jobs);
    HM_CUDA_TRY(cudaGetLastError());
    count_launch();
    return HM_OK;
}

}  // namespace hm
