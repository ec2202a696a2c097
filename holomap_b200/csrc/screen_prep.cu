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

constexpr uint32_t CSUM_BLOCKS = 64;  // column-sum partial blocks per euclidean job

// Column sums of one slice of a job's rows, binary64 (block = job x slice).
__global__ void colsum_partial_kernel(const JobDev *__restrict__ jobs, const GroupDev *__restrict__ G) {
    const uint32_t g = blockIdx.x / CSUM_BLOCKS, b = blockIdx.x % CSUM_BLOCKS;
    const JobDev &J = jobs[G->job_ids[g]];
    if (J.metric != HM_METRIC_EUCLIDEAN || !job_active(J)) return;
    const uint32_t per = (J.n + CSUM_BLOCKS - 1) / CSUM_BLOCKS;
    const uint32_t r0 = b * per, r1 = min(J.n, r0 + per);
    for (uint32_t c = threadIdx.x; c < J.d; c += blockDim.x) {
        double s = 0.0;
        for (uint32_t r = r0; r < r1; ++r) s += (double)J.x[(size_t)r * J.d + c];
        J.csum[(size_t)b * J.d + c] = s;
    }
}

__global__ void colmean_kernel(const JobDev *__restrict__ jobs, const GroupDev *__restrict__ G) {
    const JobDev &J = jobs[G->job_ids[blockIdx.x]];
    if (J.metric != HM_METRIC_EUCLIDEAN || !job_active(J)) return;
    for (uint32_t c = threadIdx.x; c < J.d; c += blockDim.x) {
        double s = 0.0;
        for (uint32_t b = 0; b < CSUM_BLOCKS; ++b) s += J.csum[(size_t)b * J.d + c];
        J.mu[c] = s / (double)J.n;
    }
}

// Largest ||x_i - mu||^2 of each euclidean job, for its power-of-two scale.
// A block covers 32 group rows (one job: a job's rows start 32-aligned), a
// warp 4 of them; one atomic per block.
__global__ void __launch_bounds__(256) centred_norm_max_kernel(const JobDev *__restrict__ jobs,
                                                              const GroupDev *__restrict__ G) {
    __shared__ double s_max[8];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t gr0 = blockIdx.x * 32;
    const JobDev &J = jobs[G->job_ids[find_job(G->row_starts, G->njobs, gr0)]];
    if (J.metric != HM_METRIC_EUCLIDEAN || !job_active(J)) return;  // uniform over the block
    double m = 0.0;
    for (uint32_t r = 0; r < 4; ++r) {
        const uint32_t row = gr0 + warp * 4 + r - J.row0;
        if (row >= J.n) break;  // padding between jobs
        double s = 0.0;
        for (uint32_t t = lane; t < J.d; t += 32) {
            const double v = (double)J.x[(size_t)row * J.d + t] - J.mu[t];
            s += v * v;
        }
        m = fmax(m, warp_sum(s));
    }
    if (lane == 0) s_max[warp] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < 8; ++w) m = fmax(m, s_max[w]);
        atomic_max_pos(&J.cnt->maxb[6], m);
    }
}

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

// Operand rows come in two kernels by the padded row length K1 of their job:
// operand_kernel (K1 > OP_SHORT_K1) gives every row a warp, the warps striding
// over the rows; operand_packed_kernel (K1 <= OP_SHORT_K1) gives a row 8 or 16
// lanes, so a warp works on two or four short rows at once.  Both run a
// persistent grid of OP_BLOCKS_PER_SM blocks per SM; each skips the other's
// jobs.  A row's loads (up to 512 elements with 32 lanes; 256 in the split
// form) are all issued before its first store, so a row costs one memory
// round trip; a job's maxima are kept per warp (per row group) and written,
// one atomic each, when the warp's next rows belong to another job, or at
// its end.
constexpr uint32_t OP_WARPS = 8;
constexpr int OP_BLOCKS_PER_SM = 3;
constexpr uint32_t OP_SHORT_K1 = 64;
uint32_t operand_short_k1() { return OP_SHORT_K1; }
constexpr int OP_TF32 = 0, OP_BF16 = 1, OP_SPLIT = 2;
// elements per lane in flight (the split form's six stores per element need
// the registers of half of them)
__host__ __device__ constexpr uint32_t op_per_lane(int mode) { return mode == OP_SPLIT ? 8u : 16u; }

// Operand row(s), binary64 error statistics, additive terms of the screen
// epilogue, and the row's shared threshold.  Every lane accumulates its
// elements t = lane, lane + 32, ... in ascending order.
template <int MODE>  // OP_TF32, OP_BF16 or OP_SPLIT: the group's operand format
__global__ void __launch_bounds__(OP_WARPS * 32, OP_BLOCKS_PER_SM) operand_kernel(const JobDev *__restrict__ jobs,
                                                               const GroupDev *__restrict__ Gp) {
    // the warp's maxima live in shared memory (lane 0 alone updates them)
    __shared__ double s_wmax[OP_WARPS][6];
    __shared__ unsigned long long s_wzero[OP_WARPS];
    const GroupDev &G = *Gp;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double *wmax = s_wmax[warp];
    const JobDev *cur = nullptr;  // the job whose maxima the warp holds
    auto reset = [&]() {
        if (lane == 0) {
            for (int q = 0; q < 6; ++q) wmax[q] = 0.0;
            s_wzero[warp] = 0;
        }
    };
    auto flush = [&]() {
        if (cur != nullptr && lane == 0) {
            unsigned long long *maxb = cur->cnt->maxb;
            for (int q = 0; q < 6; ++q) atomic_max_pos(&maxb[q], wmax[q]);
            if (s_wzero[warp]) atomicAdd(&maxb[7], s_wzero[warp]);
        }
        reset();
        cur = nullptr;
    };
    reset();
    const uint32_t stride = gridDim.x * OP_WARPS;
    for (uint32_t gr = blockIdx.x * OP_WARPS + warp; gr < G.rows; gr += stride) {
        const JobDev &J = jobs[G.job_ids[find_job(G.row_starts, G.njobs, gr)]];
        if (!job_active(J) || J.kp1 <= OP_SHORT_K1) continue;  // inactive, or operand_packed_kernel's
        const uint32_t row = gr - J.row0;
        if (row >= J.n) {  // padding between jobs: zero operands (read only as masked rows/columns)
            for (uint32_t t = lane; t < G.kpmax; t += 32) {
                if (G.elem_bytes == 4) {
                    reinterpret_cast<uint32_t *>(G.opa)[(size_t)gr * G.kpmax + t] = 0u;
                } else {
                    reinterpret_cast<uint16_t *>(G.opa)[(size_t)gr * G.kpmax + t] = 0;
                    reinterpret_cast<uint16_t *>(G.opb)[(size_t)gr * G.kpmax + t] = 0;
                }
            }
            continue;
        }
        if (&J != cur) {
            flush();
            cur = &J;
        }

        const bool euc = J.metric == HM_METRIC_EUCLIDEAN;
        double scale = 1.0;
        bool zero_row = false;
        if (euc) {
            const double m = sqrt(__longlong_as_double((long long)J.cnt->maxb[6]));
            if (m > 0.0) {
                int e;
                frexp(m, &e);  // m = f * 2^e, f in [0.5, 1)
                scale = ldexp(1.0, -e);
            }
        } else {
            const double rn = J.rnorm[row];
            zero_row = !(rn > 0.0);
            scale = zero_row ? 0.0 : 1.0 / rn;
        }

        const size_t kp = G.kpmax;
        const uint32_t d = J.d, kp1 = J.kp1;
        double uu = 0.0, ee = 0.0, rr = 0.0, aa = 0.0;
        const float *xr = J.x + (size_t)row * d;
        // cosine rows are scaled by 1 / ||x|| (the operand u is whatever this
        // arithmetic forms: the band is measured from it)
        const double mul = scale;
        constexpr uint32_t PER_LANE = op_per_lane(MODE);
        for (uint32_t t0 = 0; t0 < kp1; t0 += 32 * PER_LANE) {
            float xs[PER_LANE];
#pragma unroll
            for (uint32_t q = 0; q < PER_LANE; ++q) {
                const uint32_t t = t0 + 32 * q + lane;
                xs[q] = t < d ? __ldg(xr + t) : 0.0f;
            }
#pragma unroll
            for (uint32_t q = 0; q < PER_LANE; ++q) {
                const uint32_t t = t0 + 32 * q + lane;
                if (t >= kp1) break;
                double u = 0.0;
                if (t < d) u = euc ? ((double)xs[q] - __ldg(J.mu + t)) * mul : (double)xs[q] * mul;
                uu += u * u;
                if (MODE == OP_TF32) {
                    double r;
                    const uint32_t b = to_tf32_bits(u, &r);
                    reinterpret_cast<uint32_t *>(G.opa)[(size_t)gr * kp + t] = b;
                    ee += (r - u) * (r - u);
                    aa += r * r;
                } else if (MODE == OP_BF16) {
                    double r;
                    const uint16_t b = to_bf16_bits(u, &r);
                    reinterpret_cast<uint16_t *>(G.opa)[(size_t)gr * kp + t] = b;
                    ee += (r - u) * (r - u);
                    aa += r * r;
                } else {
                    double hi, lo;
                    const uint16_t bh = to_bf16_bits(u, &hi);
                    const uint16_t bl = to_bf16_bits(u - hi, &lo);
                    const double res = (u - hi) - lo;
                    uint16_t *A = reinterpret_cast<uint16_t *>(G.opa) + (size_t)gr * kp;
                    uint16_t *B = reinterpret_cast<uint16_t *>(G.opb) + (size_t)gr * kp;
                    A[t] = bh;
                    A[kp1 + t] = bh;
                    A[2 * kp1 + t] = bl;
                    B[t] = bh;
                    B[kp1 + t] = bl;
                    B[2 * kp1 + t] = bh;
                    ee += lo * lo;
                    rr += res * res;
                    aa += 2.0 * hi * hi + lo * lo;
                }
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
            G.rowstat[gr] = st;
            wmax[0] = fmax(wmax[0], st.unorm);
            wmax[1] = fmax(wmax[1], st.enorm);
            wmax[2] = fmax(wmax[2], st.rnorm);
            wmax[3] = fmax(wmax[3], st.anorm);
            wmax[4] = fmax(wmax[4], st.bnorm);
            wmax[5] = fmax(wmax[5], st.sqnorm);
            if (euc) {
                const float nsq = __double2float_rn(uu);
                G.rowterm[gr] = nsq;
                G.colterm[gr] = nsq;
            } else {
                G.rowterm[gr] = 0.0f;
                G.colterm[gr] = zero_row ? 0.0f : 1.0f;
            }
            G.force[gr] = zero_row ? 1 : 0;
            if (zero_row) ++s_wzero[warp];
            G.rowthr[gr] = 0xff800000u;  // the row's shared threshold starts at +inf
        }
    }
    flush();
}

// The same for the jobs with K1 <= OP_SHORT_K1: the warps stride over tiles
// of OP_TILE consecutive group rows (a tile lies in one job, whose rows start
// 32-aligned), a row taking 16 lanes when K1 > 32, else 8.  Every lane
// accumulates its elements t = s, s + L, ... (s its place among the row's L
// lanes) in ascending order.
constexpr uint32_t OP_TILE = 4;  // rows per tile: the most a warp holds at once
template <int MODE>
__global__ void __launch_bounds__(OP_WARPS * 32, OP_BLOCKS_PER_SM)
    operand_packed_kernel(const JobDev *__restrict__ jobs, const GroupDev *__restrict__ Gp) {
    // the maxima of each of the warp's row groups (a group's first lane alone
    // updates them)
    __shared__ double s_wmax[OP_WARPS][OP_TILE][6];
    __shared__ unsigned long long s_wzero[OP_WARPS][OP_TILE];
    const GroupDev &G = *Gp;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const JobDev *cur = nullptr;  // the job whose maxima the warp holds
    auto reset = [&]() {
        if (lane < (int)OP_TILE) {
            for (int q = 0; q < 6; ++q) s_wmax[warp][lane][q] = 0.0;
            s_wzero[warp][lane] = 0;
        }
        __syncwarp();
    };
    auto flush = [&]() {
        __syncwarp();
        if (cur != nullptr && lane == 0) {
            unsigned long long *maxb = cur->cnt->maxb;
            for (int q = 0; q < 6; ++q) {
                double m = s_wmax[warp][0][q];
                for (uint32_t g = 1; g < OP_TILE; ++g) m = fmax(m, s_wmax[warp][g][q]);
                atomic_max_pos(&maxb[q], m);
            }
            unsigned long long z = 0;
            for (uint32_t g = 0; g < OP_TILE; ++g) z += s_wzero[warp][g];
            if (z) atomicAdd(&maxb[7], z);
        }
        __syncwarp();
        reset();
        cur = nullptr;
    };
    reset();
    constexpr uint32_t PER_LANE = OP_SHORT_K1 / 16;  // a row's elements per lane: one chunk
    const size_t kp = G.kpmax;
    const uint32_t tiles = (G.rows + OP_TILE - 1) / OP_TILE;
    const uint32_t stride = gridDim.x * OP_WARPS;
    for (uint32_t ti = blockIdx.x * OP_WARPS + warp; ti < tiles; ti += stride) {
        const uint32_t gr0 = ti * OP_TILE;
        const JobDev &J = jobs[G.job_ids[find_job(G.row_starts, G.njobs, gr0)]];
        // uniform over the warp (a tile is of one job); longer rows are operand_kernel's
        if (!job_active(J) || J.kp1 > OP_SHORT_K1) continue;
        if (&J != cur) {
            flush();
            cur = &J;
        }
        const uint32_t d = J.d, kp1 = J.kp1;
        // padding rows between jobs: zero operands (read only as masked rows/columns)
        for (uint32_t p = 0; p < OP_TILE; ++p) {
            const uint32_t gr = gr0 + p;
            if (gr < G.rows && gr - J.row0 >= J.n) {
                for (uint32_t t = lane; t < G.kpmax; t += 32) {
                    if (G.elem_bytes == 4) {
                        reinterpret_cast<uint32_t *>(G.opa)[(size_t)gr * G.kpmax + t] = 0u;
                    } else {
                        reinterpret_cast<uint16_t *>(G.opa)[(size_t)gr * G.kpmax + t] = 0;
                        reinterpret_cast<uint16_t *>(G.opb)[(size_t)gr * G.kpmax + t] = 0;
                    }
                }
            }
        }
        const bool euc = J.metric == HM_METRIC_EUCLIDEAN;
        const uint32_t lpr = kp1 > 32 ? 16u : 8u;  // lanes per row
        const uint32_t g = (uint32_t)lane / lpr, sl = (uint32_t)lane % lpr;
        for (uint32_t p0 = 0; p0 < OP_TILE; p0 += 32 / lpr) {
            const uint32_t gr = gr0 + p0 + g;
            const uint32_t row = gr - J.row0;
            const bool real = gr < G.rows && row < J.n;  // padding rows compute zeros, write nothing
            double scale = 1.0;
            bool zero_row = false;
            if (euc) {
                const double m = sqrt(__longlong_as_double((long long)J.cnt->maxb[6]));
                if (m > 0.0) {
                    int e;
                    frexp(m, &e);  // m = f * 2^e, f in [0.5, 1)
                    scale = ldexp(1.0, -e);
                }
            } else if (real) {
                const double rn = J.rnorm[row];
                zero_row = !(rn > 0.0);
                scale = zero_row ? 0.0 : 1.0 / rn;
            }
            double uu = 0.0, ee = 0.0, rr = 0.0, aa = 0.0;
            const float *xr = J.x + (size_t)(real ? row : 0u) * d;
            // cosine rows are scaled by 1 / ||x|| (the operand u is whatever this
            // arithmetic forms: the band is measured from it)
            const double mul = scale;
            for (uint32_t t0 = 0; t0 < kp1; t0 += lpr * PER_LANE) {
                float xs[PER_LANE];
#pragma unroll
                for (uint32_t q = 0; q < PER_LANE; ++q) {
                    const uint32_t t = t0 + lpr * q + sl;
                    xs[q] = (real && t < d) ? __ldg(xr + t) : 0.0f;
                }
#pragma unroll
                for (uint32_t q = 0; q < PER_LANE; ++q) {
                    const uint32_t t = t0 + lpr * q + sl;
                    if (t >= kp1) break;
                    double u = 0.0;
                    if (t < d) u = euc ? ((double)xs[q] - __ldg(J.mu + t)) * mul : (double)xs[q] * mul;
                    uu += u * u;
                    if (MODE == OP_TF32) {
                        double r;
                        const uint32_t b = to_tf32_bits(u, &r);
                        if (real) reinterpret_cast<uint32_t *>(G.opa)[(size_t)gr * kp + t] = b;
                        ee += (r - u) * (r - u);
                        aa += r * r;
                    } else if (MODE == OP_BF16) {
                        double r;
                        const uint16_t b = to_bf16_bits(u, &r);
                        if (real) reinterpret_cast<uint16_t *>(G.opa)[(size_t)gr * kp + t] = b;
                        ee += (r - u) * (r - u);
                        aa += r * r;
                    } else {
                        double hi, lo;
                        const uint16_t bh = to_bf16_bits(u, &hi);
                        const uint16_t bl = to_bf16_bits(u - hi, &lo);
                        const double res = (u - hi) - lo;
                        if (real) {
                            uint16_t *A = reinterpret_cast<uint16_t *>(G.opa) + (size_t)gr * kp;
                            uint16_t *B = reinterpret_cast<uint16_t *>(G.opb) + (size_t)gr * kp;
                            A[t] = bh;
                            A[kp1 + t] = bh;
                            A[2 * kp1 + t] = bl;
                            B[t] = bh;
                            B[kp1 + t] = bl;
                            B[2 * kp1 + t] = bh;
                        }
                        ee += lo * lo;
                        rr += res * res;
                        aa += 2.0 * hi * hi + lo * lo;
                    }
                }
            }
            // the row's sums over its lpr lanes (xor partners stay in the group)
#pragma unroll
            for (uint32_t o = 8; o > 0; o >>= 1) {
                if (o < lpr) {
                    uu += __shfl_xor_sync(0xffffffffu, uu, o);
                    ee += __shfl_xor_sync(0xffffffffu, ee, o);
                    rr += __shfl_xor_sync(0xffffffffu, rr, o);
                    aa += __shfl_xor_sync(0xffffffffu, aa, o);
                }
            }
            if (sl == 0 && real) {
                double *wmax = s_wmax[warp][p0 + g];
                RowStat st;
                st.unorm = sqrt(uu);
                st.enorm = sqrt(ee);
                st.rnorm = sqrt(rr);
                st.anorm = sqrt(aa);
                st.bnorm = st.anorm;  // both operand layouts have the same row norm
                st.sqnorm = uu;
                G.rowstat[gr] = st;
                wmax[0] = fmax(wmax[0], st.unorm);
                wmax[1] = fmax(wmax[1], st.enorm);
                wmax[2] = fmax(wmax[2], st.rnorm);
                wmax[3] = fmax(wmax[3], st.anorm);
                wmax[4] = fmax(wmax[4], st.bnorm);
                wmax[5] = fmax(wmax[5], st.sqnorm);
                if (euc) {
                    const float nsq = __double2float_rn(uu);
                    G.rowterm[gr] = nsq;
                    G.colterm[gr] = nsq;
                } else {
                    G.rowterm[gr] = 0.0f;
                    G.colterm[gr] = zero_row ? 0.0f : 1.0f;
                }
                G.force[gr] = zero_row ? 1 : 0;
                if (zero_row) ++s_wzero[warp][p0 + g];
                G.rowthr[gr] = 0xff800000u;  // the row's shared threshold starts at +inf
            }
        }
    }
    flush();
}

// Keep band of one row (binary32 bits, rounded up), written to G.band.
__device__ __forceinline__ uint32_t band_of_row(const JobDev &J, const GroupDev &G, uint32_t gr) {
    const unsigned long long *maxb = J.cnt->maxb;
    const RowStat st = G.rowstat[gr];
    const double Umax = __longlong_as_double((long long)maxb[0]);
    const double Emax = __longlong_as_double((long long)maxb[1]);
    const double Rmax = __longlong_as_double((long long)maxb[2]);
    const double Bmax = __longlong_as_double((long long)maxb[4]);
    const double SQmax = __longlong_as_double((long long)maxb[5]);
    const double K = (double)(G.split ? 3 * J.kp1 : J.kp1);
    const double gam = K * 0x1p-22;  // fp32 accumulation, any summation order
    const double tiny = K * 0x1p-125;
    double eps;
    if (!G.split) {
        eps = st.enorm * Umax + st.unorm * Emax + st.enorm * Emax;
    } else {
        eps = st.enorm * Emax + st.rnorm * Umax + (st.unorm + st.rnorm) * Rmax;
    }
    eps += gam * st.anorm * Bmax + tiny;
    double E;
    if (J.metric == HM_METRIC_EUCLIDEAN)
        E = 2.0 * eps + (st.sqnorm + SQmax) * (0x1p-21 + (double)(J.d + 8) * 0x1p-50);
    else
        E = eps + 0x1p-21 + (double)(J.d + 8) * 0x1p-51;
    const double B = 2.0 * E * (1.0 + 0x1p-10);
    const float bf = __double2float_ru(B);
    G.band[gr] = bf;
    return __float_as_uint(bf);
}

// Keep band 2E_i per row (see screen.cuh for the terms).
__global__ void band_kernel(const JobDev *__restrict__ jobs, const GroupDev *__restrict__ Gp) {
    const GroupDev &G = *Gp;
    // a warp's 32 group rows belong to one job (each job's rows start
    // 32-aligned; G.rows is a multiple of 32)
    const uint32_t gr = blockIdx.x * blockDim.x + threadIdx.x;
    if (gr - (threadIdx.x & 31) >= G.rows) return;  // whole warps
    const JobDev &J = jobs[G.job_ids[find_job(G.row_starts, G.njobs, gr)]];
    if (!job_active(J)) return;  // uniform over the warp (32 rows of one job)
    const bool real = gr < G.rows && gr - J.row0 < J.n;  // not padding between jobs
    uint32_t bits = 0;
    if (real) bits = band_of_row(J, G, gr);
    bits = __reduce_max_sync(0xffffffffu, bits);  // non-negative floats order like their bits
    if ((threadIdx.x & 31) == 0 && bits) atomicMax(&J.out->band_max_bits, bits);
}


int launch_screen_prep(const JobDev *jobs, const GroupDev &G, const GroupDev *Gd, cudaStream_t s) {
    ScopedKernelTimer timer(HM_KCLASS_PREP, s);
    HM_CUDA_TRY(cudaMemsetAsync(G.colterm, 0, round_up(G.rows, SC_BN) * sizeof(float) + SC_BN * sizeof(float), s));
    colsum_partial_kernel<<<G.njobs * CSUM_BLOCKS, 128, 0, s>>>(jobs, Gd);
    colmean_kernel<<<G.njobs, 128, 0, s>>>(jobs, Gd);
    // G.rows is a multiple of 32: 32 group rows per block
    centred_norm_max_kernel<<<G.rows / 32, 256, 0, s>>>(jobs, Gd);
    const uint32_t op_cap = (uint32_t)device_sm_count() * OP_BLOCKS_PER_SM;
    const uint32_t row_blocks = (G.rows + OP_WARPS - 1) / OP_WARPS;
    const uint32_t row_grid = row_blocks < op_cap ? row_blocks : op_cap;
    const uint32_t tile_blocks = (G.rows + OP_WARPS * OP_TILE - 1) / (OP_WARPS * OP_TILE);
    const uint32_t tile_grid = tile_blocks < op_cap ? tile_blocks : op_cap;
    auto both = [&](auto rows_kernel, auto packed_kernel) {
        if (G.any_long_rows) rows_kernel<<<row_grid, OP_WARPS * 32, 0, s>>>(jobs, Gd);
        if (G.any_short_rows) packed_kernel<<<tile_grid, OP_WARPS * 32, 0, s>>>(jobs, Gd);
    };
    if (G.kind == SCREEN_KIND_TF32)
        both(operand_kernel<OP_TF32>, operand_packed_kernel<OP_TF32>);
    else if (!G.split)
        both(operand_kernel<OP_BF16>, operand_packed_kernel<OP_BF16>);
    else
        both(operand_kernel<OP_SPLIT>, operand_packed_kernel<OP_SPLIT>);
    HM_CUDA_TRY(cudaGetLastError());
    count_launch(3 + (G.any_long_rows ? 1 : 0) + (G.any_short_rows ? 1 : 0));
    return HM_OK;
}

int launch_screen_band(const JobDev *jobs, const GroupDev &G, const GroupDev *Gd, cudaStream_t s) {
    ScopedKernelTimer timer(HM_KCLASS_PREP, s);
    band_kernel<<<(G.rows + 255) / 256, 256, 0, s>>>(jobs, Gd);
    HM_CUDA_TRY(cudaGetLastError());
    count_launch();
    return HM_OK;
}

}  // namespace hm
