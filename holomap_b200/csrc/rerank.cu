// rerank.cu -- the row threshold between the two screen passes, and the
// exact rerank of the screen's candidates.
//
// threshold: one warp per row merges the k smallest mini-chunk minima of the
// row's lists into tau1, the k-th smallest of their union.  Every mini-chunk
// minimum is a screened value of the row, so at least k screened values are
// <= tau1 and the row's k-th smallest screened value tau^ <= tau1.
//
// rerank: one warp per query row.  tau^ is recomputed exactly as the k-th
// smallest screened value among the emitted candidates (pass 1 emitted every
// column with c^ <= tau1 + band, which includes the k smallest); candidates
// with c^ <= tau^ + band are compacted into shared memory, and each lane then
// evaluates one candidate's distance exactly as the reference does
// (src/metric.rs:42-53 euclidean, :58-70 cosine: binary64, dimension order,
// no contraction, self forced to 0 as in src/knn.rs:38-39), feeding the
// (distance bits, index) keys to a warp top-k list.  Rows whose candidate list
// overflowed, or that the screen cannot bound (zero vectors under cosine), are
// appended to the overflow list for the exact plain path.
#include <cuda_runtime.h>

#include "hm_internal.cuh"
#include "screen.cuh"

namespace hm {

// One dimension of the reference's accumulation: euclidean (x - y)^2,
// cosine x * y, each operation rounded to nearest in binary64.
template <int METRIC>
__device__ __forceinline__ double step(double acc, double x, double y) {
    if (METRIC == HM_METRIC_EUCLIDEAN) {
        const double diff = __dsub_rn(x, y);
        return __dadd_rn(acc, __dmul_rn(diff, diff));
    }
    return __dadd_rn(acc, __dmul_rn(x, y));
}

// k-th smallest of a warp's `total` keys (at most 32 * NQ; lane l holds keys
// l, l + 32, ...; absent keys are ~0): the largest r with fewer than k keys
// below it, found bit by bit from the highest bit where the keys differ.
template <int NQ>
__device__ __forceinline__ uint32_t kth_key(const uint32_t (&ov)[NQ], uint32_t total, uint32_t k, int lane) {
    uint32_t mn = 0xffffffffu, mx = 0u;
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
        if ((uint32_t)(q * 32 + lane) < total) {
            mn = min(mn, ov[q]);
            mx = max(mx, ov[q]);
        }
    }
    mn = __reduce_min_sync(0xffffffffu, mn);
    mx = __reduce_max_sync(0xffffffffu, mx);
    if (mn == mx) return mn;
    const int top = 31 - __clz(mn ^ mx);
    uint32_t r = top == 31 ? 0u : (mn & ~((2u << top) - 1u));  // the keys' common high bits
    for (int b = top; b >= 0; --b) {
        const uint32_t t = r | (1u << b);
        uint32_t c = 0;
#pragma unroll
        for (int q = 0; q < NQ; ++q) c += ov[q] < t ? 1u : 0u;
        c = __reduce_add_sync(0xffffffffu, c);
        if (c < k) r = t;
    }
    return r;
}

// kth_key over keys key(e), e < total <= 512, with the register count
// chosen by the total
template <int NQ, typename KeyFn>
__device__ __forceinline__ uint32_t kth_load(KeyFn key, uint32_t total, uint32_t k, int lane) {
    uint32_t ov[NQ];
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
        const uint32_t e = q * 32 + lane;
        ov[q] = e < total ? key(e) : 0xffffffffu;
    }
    return kth_key<NQ>(ov, total, k, lane);
}

template <typename KeyFn>
__device__ __forceinline__ uint32_t kth_of(KeyFn key, uint32_t total, uint32_t k, int lane) {
    if (total <= 32) return kth_load<1>(key, total, k, lane);
    if (total <= 64) return kth_load<2>(key, total, k, lane);
    if (total <= 128) return kth_load<4>(key, total, k, lane);
    if (total <= 256) return kth_load<8>(key, total, k, lane);
    return kth_load<16>(key, total, k, lane);
}

constexpr int RR_WARPS = 8;
constexpr int RR_LIST = 256;  // compacted candidates per warp between flushes
constexpr int RR_CBUF = 512;  // emitted candidates a warp stages in shared memory

// One warp per group row; candidates are evaluated 32 at a time, one per lane.
template <int METRIC, int KPL>
__device__ __forceinline__ void rerank_row(const JobDev *__restrict__ jobs, const GroupDev *__restrict__ Gp,
                                           uint32_t dstride) {
    extern __shared__ double rr_smem[];
    const GroupDev &G = *Gp;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t gr = blockIdx.x * RR_WARPS + warp;
    if (gr >= G.rows) return;
    const JobDev &J = jobs[G.job_ids[find_job(G.row_starts, G.njobs, gr)]];
    if ((int)J.metric != METRIC) return;
    const uint32_t row = gr - J.row0;
    if (row < J.q0 || row >= J.q1) return;  // padding between jobs, rows of other shards
    const uint32_t k = J.k, d = J.d, lists = 2 * J.parts;
    const size_t l0 = list_index(J, row, 0);
    double *xi = rr_smem + (size_t)warp * dstride;
    uint32_t *list = reinterpret_cast<uint32_t *>(rr_smem + (size_t)RR_WARPS * dstride) + warp * RR_LIST;
    unsigned long long *cbuf = reinterpret_cast<unsigned long long *>(
                                   reinterpret_cast<uint32_t *>(rr_smem + (size_t)RR_WARPS * dstride) +
                                   RR_WARPS * RR_LIST) + warp * RR_CBUF;

    // overflow / unbounded rows go to the exact plain path
    bool ovf = G.force[gr] != 0;
    for (uint32_t p = 0; p < lists; ++p) ovf |= G.cand_cnt[l0 + p] > J.cap;
    if (ovf) {
        if (lane == 0) {
            const uint32_t at = atomicAdd(&J.cnt->ovf_count, 1u);
            J.ovf_list[at] = row;
        }
        return;
    }
    // Threshold: the exact k-th smallest screened value of the row, over the
    // emitted candidates (they include the row's k smallest).  Up to RR_CBUF
    // candidates are staged in shared memory and the k-th found by a bitwise
    // search on the order-preserving keys; longer rows use a warp top-k.
    uint32_t total = 0;
    for (uint32_t p = 0; p < lists; ++p) total += G.cand_cnt[l0 + p];
    const bool staged = total <= RR_CBUF;
    float tau = __int_as_float(0x7f800000);
    if (staged) {
        uint32_t base = 0;
        for (uint32_t p = 0; p < lists; ++p) {
            const uint32_t cnt = G.cand_cnt[l0 + p];
            const unsigned long long *cand = G.cand + J.cand0 + (l0 + p - J.slot0) * J.cap;
            for (uint32_t e = lane; e < cnt; e += 32) cbuf[base + e] = cand[e];
            base += cnt;
        }
        __syncwarp();
        if (total >= k)
            tau = unord32(kth_of([&](uint32_t e) { return ord32(__uint_as_float((uint32_t)(cbuf[e] >> 32))); },
                                 total, k, lane));
    } else {
        WarpTopK<KPL> sel;
        sel.reset();
        for (uint32_t p = 0; p < lists; ++p) {
            const uint32_t cnt = G.cand_cnt[l0 + p];
            const unsigned long long *cand = G.cand + J.cand0 + (l0 + p - J.slot0) * J.cap;
            for (uint32_t e0 = 0; e0 < cnt; e0 += 32) {
                uint64_t key = KEY_NONE;
                if (e0 + lane < cnt) {
                    const unsigned long long c = cand[e0 + lane];
                    key = ((uint64_t)ord32(__uint_as_float((uint32_t)(c >> 32))) << 32) | (uint32_t)c;
                }
                sel.offer(key, k, lane);
            }
        }
        if (sel.tau != KEY_NONE) tau = unord32((uint32_t)(sel.tau >> 32));
    }
    const float thr = __fadd_ru(tau, G.band[gr]);

    for (uint32_t t = lane; t < d; t += 32) xi[t] = (double)J.x[(size_t)row * d + t];
    __syncwarp();
    const double rn_i = (METRIC == HM_METRIC_COSINE) ? J.rnorm[row] : 0.0;

    WarpTopK<KPL> top;
    top.reset();
    uint32_t fill = 0, kept = 0;
    const unsigned lt_mask = (1u << lane) - 1u;

    // Each lane evaluates one candidate, reading that candidate's row with
    // 16-byte loads (4 dimensions, consumed in order) and the query row as
    // broadcast pairs from shared memory.
    auto flush = [&](uint32_t m) {
        for (uint32_t b = 0; b < m; b += 32) {
            const bool mine = b + lane < m;
            const uint32_t j = mine ? list[b + lane] : row;
            const float *xj = J.x + (size_t)j * d;
            double acc = 0.0;
            uint32_t t = 0;
            // 16-byte loads when every row starts 16-byte aligned (the caller's
            // pointer need only be 4-byte aligned)
            if ((d & 3u) == 0 && (reinterpret_cast<uintptr_t>(J.x) & 15u) == 0) {
                const float4 *xj4 = reinterpret_cast<const float4 *>(xj);
                const double2 *xi2 = reinterpret_cast<const double2 *>(xi);
#pragma unroll 4
                for (uint32_t q = 0; q < d / 4; ++q) {
                    const float4 y = __ldg(xj4 + q);
                    const double2 p0 = xi2[2 * q], p1 = xi2[2 * q + 1];
                    acc = step<METRIC>(acc, p0.x, (double)y.x);
                    acc = step<METRIC>(acc, p0.y, (double)y.y);
                    acc = step<METRIC>(acc, p1.x, (double)y.z);
                    acc = step<METRIC>(acc, p1.y, (double)y.w);
                }
                t = d;
            }
            for (; t < d; ++t) acc = step<METRIC>(acc, xi[t], (double)__ldg(xj + t));
            uint64_t key = KEY_NONE;
            if (mine) {
                float dist;
                if (j == row) {
                    dist = 0.0f;  // src/knn.rs:38-39
                } else if (METRIC == HM_METRIC_EUCLIDEAN) {
                    dist = __double2float_rn(__dsqrt_rn(acc));
                } else {
                    const double q = __ddiv_rn(acc, __dmul_rn(rn_i, J.rnorm[j]));
                    const double r = __dsub_rn(1.0, q);
                    dist = (r > 0.0) ? __double2float_rn(r) : 0.0f;
                }
                key = make_key(dist, j);
            }
            top.offer(key, k, lane);
        }
        __syncwarp();
    };

    // compaction of the candidates within tau + band, from the staged copy or
    // from the lists
    auto compact = [&](const unsigned long long *src, uint32_t cnt) {
        for (uint32_t e0 = 0; e0 < cnt; e0 += 32) {
            bool pass = false;
            uint32_t j = 0;
            if (e0 + lane < cnt) {
                const unsigned long long c = src[e0 + lane];
                const float cv = __uint_as_float((uint32_t)(c >> 32));
                j = (uint32_t)c;
                pass = !(cv > thr);
            }
            const unsigned m = __ballot_sync(0xffffffffu, pass);
            if (pass) list[fill + __popc(m & lt_mask)] = j;
            fill += __popc(m);
            kept += __popc(m);
            __syncwarp();
            if (fill > RR_LIST - 32) {
                flush(fill);
                fill = 0;
            }
        }
    };
    if (staged) {
        compact(cbuf, total);
    } else {
        for (uint32_t p = 0; p < lists; ++p)
            compact(G.cand + J.cand0 + (l0 + p - J.slot0) * J.cap, G.cand_cnt[l0 + p]);
    }
    flush(fill);

#pragma unroll
    for (int q = 0; q < KPL; ++q) {
        const uint32_t e = q * 32 + lane;
        if (e < k) {
            J.idx[(size_t)row * k + e] = key_idx(top.v[q]);
            J.dist[(size_t)row * k + e] = key_dist(top.v[q]);
        }
    }
    if (lane == 0) {
        atomicAdd(&J.cnt->candidates, (unsigned long long)kept);
        atomicMax(&J.cnt->max_row, kept);
    }
}

// tau1 of every row: the k-th smallest of the union of its lists' k smallest
// mini-chunk minima (an upper bound of the row's k-th screened value).
template <int KPL>
__global__ void __launch_bounds__(256) threshold_kernel(const JobDev *__restrict__ jobs,
                                                       const GroupDev *__restrict__ Gp) {
    const GroupDev &G = *Gp;
    const int lane = threadIdx.x & 31;
    const uint32_t gr = blockIdx.x * 8 + (threadIdx.x >> 5);
    if (gr >= G.rows) return;
    const JobDev &J = jobs[G.job_ids[find_job(G.row_starts, G.njobs, gr)]];
    const uint32_t row = gr - J.row0;
    if (row < J.q0 || row >= J.q1) return;
    const uint32_t k = J.k, lists = 2 * J.parts;
    const size_t l0 = list_index(J, row, 0);
    // the row's lists' arrays are contiguous: lists x k values
    const float *base = G.topk + J.topk0 + (l0 - J.slot0) * k;
    const uint32_t total = lists * k;
    if (total <= 256) {
        const uint32_t r = kth_of([&](uint32_t e) { return ord32(base[e]); }, total, k, lane);
        if (lane == 0) G.rowthr[gr] = r;
        return;
    }
    WarpTopK<KPL> sel;
    sel.reset();
    for (uint32_t p = 0; p < lists; ++p) {
        const float *kk = base + p * k;
        for (uint32_t e0 = 0; e0 < k; e0 += 32) {
            const uint64_t key = (e0 + lane < k) ? (((uint64_t)ord32(kk[e0 + lane]) << 32) | (p * k + e0 + lane))
                                                 : KEY_NONE;
            if (!__any_sync(0xffffffffu, key < sel.tau)) break;  // arrays are ascending
            sel.offer(key, k, lane);
        }
    }
    if (lane == 0) G.rowthr[gr] = sel.tau == KEY_NONE ? ord32(__int_as_float(0x7f800000)) : (uint32_t)(sel.tau >> 32);
}

int launch_screen_threshold(const JobDev *jobs, const GroupDev &G, const GroupDev *Gd, uint32_t kpl,
                            cudaStream_t s) {
    if (G.rows == 0) return HM_OK;
    ScopedKernelTimer timer(HM_KCLASS_SELECT, s);
    const int blocks = (int)((G.rows + 7) / 8);
    switch (kpl) {
    case 1: threshold_kernel<1><<<blocks, 256, 0, s>>>(jobs, Gd); break;
    case 2: threshold_kernel<2><<<blocks, 256, 0, s>>>(jobs, Gd); break;
    default: return set_error(HM_ERR_UNSUPPORTED, "threshold width %u", kpl);
    }
    HM_CUDA_TRY(cudaGetLastError());
    count_launch();
    return HM_OK;
}

// One launch covers both metrics of a group: each warp's row runs the
// instantiation of its job's metric.
template <int MASK, int KPL>
__global__ void __launch_bounds__(RR_WARPS * 32, 3) rerank_kernel(const JobDev *__restrict__ jobs,
                                                               const GroupDev *__restrict__ Gp,
                                                               uint32_t dstride) {
    if (MASK & (1 << HM_METRIC_EUCLIDEAN)) rerank_row<HM_METRIC_EUCLIDEAN, KPL>(jobs, Gp, dstride);
    if (MASK & (1 << HM_METRIC_COSINE)) rerank_row<HM_METRIC_COSINE, KPL>(jobs, Gp, dstride);
}

template <int MASK>
static int launch_metric(const JobDev *jobs, const GroupDev &G, const GroupDev *Gd, uint32_t kpl,
                         uint32_t dmax, cudaStream_t s) {
    const uint32_t dstride = (uint32_t)round_up(dmax, 4);
    const size_t smem = (size_t)RR_WARPS * dstride * sizeof(double) + RR_WARPS * RR_LIST * sizeof(uint32_t) +
                        (size_t)RR_WARPS * RR_CBUF * sizeof(unsigned long long);
    const int blocks = (int)((G.rows + RR_WARPS - 1) / RR_WARPS);
#define HM_RR_CASE(K)                                                                       \
    case K: {                                                                               \
        HM_TRY(ensure_dynamic_smem((const void *)rerank_kernel<MASK, K>, (int)smem));       \
        rerank_kernel<MASK, K><<<blocks, RR_WARPS * 32, smem, s>>>(jobs, Gd, dstride);      \
        break;                                                                              \
    }
    switch (kpl) {
        HM_RR_CASE(1)
        HM_RR_CASE(2)
    default: return set_error(HM_ERR_UNSUPPORTED, "rerank width %u", kpl);
    }
#undef HM_RR_CASE
    HM_CUDA_TRY(cudaGetLastError());
    count_launch();
    return HM_OK;
}

// one launch for the metrics present in the group
int launch_rerank(const JobDev *jobs, const GroupDev &G, const GroupDev *Gd, uint32_t kpl,
                  uint32_t dmax, int metric_mask, cudaStream_t s) {
    if (G.rows == 0) return HM_OK;
    ScopedKernelTimer timer(HM_KCLASS_SELECT, s);
    const int mask = metric_mask & ((1 << HM_METRIC_EUCLIDEAN) | (1 << HM_METRIC_COSINE));
    if (mask == 1) return launch_metric<1>(jobs, G, Gd, kpl, dmax, s);
    if (mask == 2) return launch_metric<2>(jobs, G, Gd, kpl, dmax, s);
    if (mask == 3) return launch_metric<3>(jobs, G, Gd, kpl, dmax, s);
    return HM_OK;
}

}  // namespace hm
