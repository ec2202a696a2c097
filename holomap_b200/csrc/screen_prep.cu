// screen_prep.cu -- operands and error terms of the tensor-core screen.
//
// For every row i the screen works on a real vector u_i whose inner products
// give the distance ordering exactly:
//   cosine     u_i = x_i / ||x_i||              (c = 1 - u_i.u_j)
//   euclidean  u_i = (x_i - mu) * 2^-s          (c = ||u_i||^2 + ||u_j||^2 - 2 u_i.u_j)
// with mu the column mean and 2^-s a power of two that brings the largest
// ||u_i|| into [0.5, 1) (exact scaling, so no overflow or underflow can arise
// in the screen's binary32 arithmetic).  u_i is formed in binary64, rounded
// to the tensor-core operand format (bf16, tf32, or a bf16 hi/lo split), and
// the exact rounding error of every row is measured in binary64.  The band
// kernel turns those measurements into each row's keep band 2E_i (the
// derivation is in screen.cuh).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "hm_internal.cuh"
#include "screen.cuh"

namespace hm {

constexpr double kFltMin = 1.1754943508222875e-38;  // 2^-126

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ void atomic_max_pos(unsigned long long *p, double v) {
    // non-negative doubles order like their bit patterns
    atomicMax(p, (unsigned long long)__double_as_longlong(v));
}

// Column sums of the rows in [blockIdx.x * rows_per, ...), binary64.
__global__ void colsum_partial_kernel(const float *__restrict__ x, uint32_t n, uint32_t d,
                                      uint32_t rows_per, double *__restrict__ partial) {
    const uint32_t r0 = blockIdx.x * rows_per;
    const uint32_t r1 = min(n, r0 + rows_per);
    for (uint32_t c = threadIdx.x; c < d; c += blockDim.x) {
        double s = 0.0;
        for (uint32_t r = r0; r < r1; ++r) s += (double)x[(size_t)r * d + c];
        partial[(size_t)blockIdx.x * d + c] = s;
    }
}

__global__ void colmean_kernel(const double *__restrict__ partial, uint32_t blocks, uint32_t n,
                               uint32_t d, double *__restrict__ mu) {
    for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < d; c += gridDim.x * blockDim.x) {
        double s = 0.0;
        for (uint32_t b = 0; b < blocks; ++b) s += partial[(size_t)b * d + c];
        mu[c] = s / (double)n;
    }
}

// Largest ||x_i - mu||^2 (euclidean), for the power-of-two scale.
__global__ void centred_norm_max_kernel(const float *__restrict__ x, uint32_t n, uint32_t d,
                                        const double *__restrict__ mu,
                                        unsigned long long *__restrict__ maxbits) {
    const int lane = threadIdx.x & 31;
    const uint32_t row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (row >= n) return;
    double s = 0.0;
    for (uint32_t t = lane; t < d; t += 32) {
        const double v = (double)x[(size_t)row * d + t] - mu[t];
        s += v * v;
    }
    s = warp_sum(s);
    if (lane == 0) atomic_max_pos(maxbits, s);
}

__device__ __forceinline__ double flush_tiny(double v) { return fabs(v) < kFltMin ? 0.0 : v; }

__device__ __forceinline__ uint16_t to_bf16_bits(double v, double *rounded) {
    const __nv_bfloat16 h = __float2bfloat16_rn((float)v);
    double r = (double)__bfloat162float(h);
    if (fabs(r) < kFltMin) {
        *rounded = 0.0;
        return 0;
    }
    *rounded = r;
    return __bfloat16_as_ushort(h);
}

__device__ __forceinline__ uint32_t to_tf32_bits(double v, double *rounded) {
    uint32_t b;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(b) : "f"((float)v));
    double r = (double)__uint_as_float(b);
    if (fabs(r) < kFltMin) {
        *rounded = 0.0;
        return 0u;
    }
    *rounded = r;
    return b;
}

// One warp per row: operand row(s), binary64 error statistics, additive
// terms of the screen epilogue.
__global__ void __launch_bounds__(256) operand_kernel(const float *__restrict__ x,
                                                     const double *__restrict__ rnorm_ref,
                                                     uint32_t n, uint32_t d, uint32_t metric,
                                                     ScreenLayout L, char *__restrict__ ws) {
    const int lane = threadIdx.x & 31;
    const uint32_t row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (row >= n) return;
    const double *mu = reinterpret_cast<const double *>(ws + L.off_mu);
    unsigned long long *maxb = reinterpret_cast<unsigned long long *>(ws + L.off_max);
    RowStat *stats = reinterpret_cast<RowStat *>(ws + L.off_rowstat);
    float *rowterm = reinterpret_cast<float *>(ws + L.off_rowterm);
    float *colterm = reinterpret_cast<float *>(ws + L.off_colterm);
    uint8_t *force = reinterpret_cast<uint8_t *>(ws + L.off_force);

    double scale = 1.0;
    bool zero_row = false;
    if (metric == HM_METRIC_EUCLIDEAN) {
        const double m = sqrt(__longlong_as_double((long long)maxb[ROWSTAT_FIELDS]));
        if (m > 0.0) {
            int e;
            frexp(m, &e);  // m = f * 2^e, f in [0.5, 1)
            scale = ldexp(1.0, -e);
        }
    } else {
        const double rn = rnorm_ref[row];
        zero_row = !(rn > 0.0);
        scale = zero_row ? 0.0 : 1.0 / rn;
    }

    double uu = 0.0, ee = 0.0, rr = 0.0, aa = 0.0;
    const float *xr = x + (size_t)row * d;
    for (uint32_t t = lane; t < L.kp1; t += 32) {
        double u = 0.0;
        if (t < d) {
            u = (metric == HM_METRIC_EUCLIDEAN) ? ((double)xr[t] - mu[t]) * scale
                                                : (zero_row ? 0.0 : (double)xr[t] / rnorm_ref[row]);
        }
        uu += u * u;
        if (L.kind == SCREEN_KIND_TF32) {
            double r;
            const uint32_t b = to_tf32_bits(u, &r);
            reinterpret_cast<uint32_t *>(ws + L.off_a)[(size_t)row * L.kp + t] = b;
            ee += (r - u) * (r - u);
            aa += r * r;
        } else if (!L.split) {
            double r;
            const uint16_t b = to_bf16_bits(u, &r);
            reinterpret_cast<uint16_t *>(ws + L.off_a)[(size_t)row * L.kp + t] = b;
            ee += (r - u) * (r - u);
            aa += r * r;
        } else {
            double hi, lo;
            const uint16_t bh = to_bf16_bits(u, &hi);
            const uint16_t bl = to_bf16_bits(u - hi, &lo);
            const double res = (u - hi) - lo;
            uint16_t *A = reinterpret_cast<uint16_t *>(ws + L.off_a) + (size_t)row * L.kp;
            uint16_t *B = reinterpret_cast<uint16_t *>(ws + L.off_b) + (size_t)row * L.kp;
            A[t] = bh;
            A[L.kp1 + t] = bh;
            A[2 * L.kp1 + t] = bl;
            B[t] = bh;
            B[L.kp1 + t] = bl;
            B[2 * L.kp1 + t] = bh;
            ee += lo * lo;
            rr += res * res;
            aa += 2.0 * hi * hi + lo * lo;
        }
    }
    uu = warp_sum(uu);
    ee = warp_sum(ee);
    rr = warp_sum(rr);
    aa = warp_sum(aa);
    if (lane == 0) {
        RowStat st;
        st.unorm = sqrt(uu);
        st.enorm = sqrt(ee);
        st.rnorm = sqrt(rr);
        st.anorm = sqrt(aa);
        st.bnorm = st.anorm;  // both operand layouts have the same row norm
        st.sqnorm = uu;
        stats[row] = st;
        atomic_max_pos(&maxb[0], st.unorm);
        atomic_max_pos(&maxb[1], st.enorm);
        atomic_max_pos(&maxb[2], st.rnorm);
        atomic_max_pos(&maxb[3], st.anorm);
        atomic_max_pos(&maxb[4], st.bnorm);
        atomic_max_pos(&maxb[5], st.sqnorm);
        if (metric == HM_METRIC_EUCLIDEAN) {
            const float nsq = __double2float_rn(uu);
            rowterm[row] = nsq;
            colterm[row] = nsq;
        } else {
            colterm[row] = zero_row ? 0.0f : 1.0f;
        }
        force[row] = zero_row ? 1 : 0;
        // shared screen threshold of the row starts at +inf (order-preserving key)
        reinterpret_cast<uint32_t *>(ws + L.off_rowthr)[row] = 0xff800000u;
        if (zero_row) atomicAdd(&maxb[7], 1ull);
    }
}

// Keep band 2E_i per row (see screen.cuh for the terms).
__global__ void band_kernel(uint32_t n, uint32_t d, uint32_t metric, ScreenLayout L,
                            char *__restrict__ ws, uint32_t *__restrict__ band_max_bits) {
    const uint32_t row = blockIdx.x * blockDim.x + threadIdx.x;
    if (row >= n) return;
    const unsigned long long *maxb = reinterpret_cast<const unsigned long long *>(ws + L.off_max);
    const RowStat st = reinterpret_cast<const RowStat *>(ws + L.off_rowstat)[row];
    const double Umax = __longlong_as_double((long long)maxb[0]);
    const double Emax = __longlong_as_double((long long)maxb[1]);
    const double Rmax = __longlong_as_double((long long)maxb[2]);
    const double Bmax = __longlong_as_double((long long)maxb[4]);
    const double SQmax = __longlong_as_double((long long)maxb[5]);
    const double K = (double)L.kp;
    const double gam = K * 0x1p-22;  // fp32 accumulation, any summation order
    const double tiny = K * 0x1p-125;
    double eps;
    if (!L.split) {
        eps = st.enorm * Umax + st.unorm * Emax + st.enorm * Emax;
    } else {
        eps = st.enorm * Emax + st.rnorm * Umax + (st.unorm + st.rnorm) * Rmax;
    }
    eps += gam * st.anorm * Bmax + tiny;
    double E;
    if (metric == HM_METRIC_EUCLIDEAN)
        E = 2.0 * eps + (st.sqnorm + SQmax) * (0x1p-21 + (double)(d + 8) * 0x1p-50);
    else
        E = eps + 0x1p-21 + (double)(d + 8) * 0x1p-51;
    const double B = 2.0 * E * (1.0 + 0x1p-10);
    const float bf = __double2float_ru(B);
    reinterpret_cast<float *>(ws + L.off_band)[row] = bf;
    atomicMax(band_max_bits, __float_as_uint(bf));
}

int launch_screen_prep(const ScreenPrepArgs &a, cudaStream_t s) {
    ScopedKernelTimer timer(HM_KCLASS_PREP, s);
    const ScreenLayout &L = a.L;
    HM_CUDA_TRY(cudaMemsetAsync(a.ws + L.off_max, 0, 8 * sizeof(unsigned long long), s));
    HM_CUDA_TRY(cudaMemsetAsync(a.ws + L.off_colterm, 0, round_up(a.n, SC_BN) * sizeof(float), s));
    if (a.metric == HM_METRIC_EUCLIDEAN) {
        const uint32_t rows_per = (a.n + L.csum_blocks - 1) / L.csum_blocks;
        colsum_partial_kernel<<<L.csum_blocks, 128, 0, s>>>(
            a.x, a.n, a.d, rows_per, reinterpret_cast<double *>(a.ws + L.off_csum));
        colmean_kernel<<<(a.d + 127) / 128, 128, 0, s>>>(
            reinterpret_cast<double *>(a.ws + L.off_csum), L.csum_blocks, a.n, a.d,
            reinterpret_cast<double *>(a.ws + L.off_mu));
        centred_norm_max_kernel<<<(a.n + 7) / 8, 256, 0, s>>>(
            a.x, a.n, a.d, reinterpret_cast<double *>(a.ws + L.off_mu),
            reinterpret_cast<unsigned long long *>(a.ws + L.off_max) + ROWSTAT_FIELDS);
        HM_CUDA_TRY(cudaGetLastError());
        count_launch(3);
    }
    operand_kernel<<<(a.n + 7) / 8, 256, 0, s>>>(a.x, a.rnorm_ref, a.n, a.d, a.metric, L, a.ws);
    HM_CUDA_TRY(cudaGetLastError());
    count_launch();
    return HM_OK;
}

int launch_screen_band(uint32_t n, uint32_t d, int metric, const ScreenLayout &L, char *ws,
                       uint32_t *band_max_bits, cudaStream_t s) {
    ScopedKernelTimer timer(HM_KCLASS_PREP, s);
    band_kernel<<<(n + 255) / 256, 256, 0, s>>>(n, d, (uint32_t)metric, L, ws, band_max_bits);
    HM_CUDA_TRY(cudaGetLastError());
    count_launch();
    return HM_OK;
}

}  // namespace hm
