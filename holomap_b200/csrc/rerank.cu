// rerank.cu -- the row threshold between the two screen passes, and the
// exact rerank of the screen's candidates.
//
// threshold: one warp per row merges the k smallest mini-chunk minima of the
// row's lists into tau1, the k-th smallest of their union.  Every mini-chunk
// minimum is a screened value of the row, so at least k screened values are
// <= tau1 and the row's k-th smallest screened value tau^ <= tau1.
//
// rerank: one warp per 8 consecutive group rows (always of one job: each job's
// rows start 32-aligned in the group), in three phases.
//   1. select, per row: tau^ is recomputed exactly as the k-th smallest
//      screened value among the emitted candidates (the emission pass wrote
//      every column with c^ <= tau1 + band, which includes the k smallest),
//      and the candidates with c^ <= tau^ + band are compacted in place to the
//      front of the row's own list region.  Rows whose list overflowed, or that
//      the screen cannot bound (zero vectors under cosine), are appended to the
//      overflow list for the exact plain path.
//   2. exact distances: the survivors of the warp's rows are taken as one flat
//      sequence and processed 32 at a time (a slice never spans more than 4
//      rows), one candidate per lane.  The candidate rows are staged through
//      shared memory 32 dimensions at a time by cp.async with coalesced
//      128-byte reads (8 lanes per candidate row; a 3-stage pipeline), the
//      query rows' chunks beside them, converted once to binary64; each lane
//      then accumulates its pair exactly as the reference does
//      (src/metric.rs:42-53 euclidean, :58-70 cosine: binary64, dimension
//      order, no contraction; self forced to 0 as in src/knn.rs:38-39) and
//      overwrites its survivor's slot with the (distance bits, index) key.
//   3. select, per row: the k smallest keys of its survivors (the reference's
//      (total_cmp(dist), index) order, src/knn.rs:46-52) are the row's output.
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

constexpr int RR_ROWS = 8;        // group rows per warp
constexpr int RR_WARPS = 4;       // warps per block
constexpr int RR_CBUF = 512;      // emitted candidates a warp stages in shared memory
constexpr int RR_STAGES = 3;      // chunks in flight
constexpr int RR_CH = 32;         // dimensions per chunk
constexpr int RR_XJ_STRIDE = 36;  // floats per staged candidate chunk (144 B: 16-byte aligned rows
                                  // whose 16-byte reads by 32 lanes need the minimum 4 wavefronts)
constexpr int RR_QROWS = 4;       // query rows per slice
constexpr int RR_XI_STRIDE = 36;  // doubles per converted query-row chunk (rows 8 banks apart)

// Shared memory of one warp: the select phase's staging buffer and the exact
// phase's chunk pipeline are never live together.
struct RrWarpSmem {
    union {
        unsigned long long cbuf[RR_CBUF];
        struct {
            float xj[RR_STAGES][32][RR_XJ_STRIDE];
            float xi[RR_STAGES][RR_QROWS][32];
            double xid[RR_QROWS][RR_XI_STRIDE];
            uint32_t cj[32];
        } ex;
    };
};

__device__ __forceinline__ uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// global -> shared copies that zero-fill the bytes past src_bytes (0 reads nothing)
__device__ __forceinline__ void cp_async16(void *dst, const void *src, uint32_t src_bytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(smem_addr(dst)), "l"(src), "r"(src_bytes)
                 : "memory");
}
__device__ __forceinline__ void cp_async4(void *dst, const void *src, uint32_t src_bytes) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(smem_addr(dst)), "l"(src), "r"(src_bytes)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// The survivors of one row live at the front of its list region (the row's
// elists candidate lists are contiguous).
__device__ __forceinline__ unsigned long long *row_region(const JobDev &J, const GroupDev &G, uint32_t row) {
    return cand_slots(J, G, cand_list(J, row, 0));
}

// Capacity of a row's candidate list s: the symmetric emission's column list
// (s = elists - 2) takes the room of two lists.
__device__ __forceinline__ uint32_t list_cap(const JobDev &J, uint32_t s) {
    return (J.sym && s == J.elists - 2) ? 2 * J.cap : J.cap;
}

// Phase 1 for one row: returns the survivor count (0 for rows sent to the
// exact fallback).
template <int KPL>
__device__ __forceinline__ uint32_t select_row(const JobDev &J, const GroupDev &G, uint32_t gr, uint32_t row,
                                               RrWarpSmem &sm, int lane) {
    const uint32_t k = J.k, lists = J.elists;
    const size_t l0 = cand_list(J, row, 0);
    // overflow / unbounded rows go to the exact plain path
    bool ovf = G.force[gr] != 0;
    uint32_t total = 0;
    for (uint32_t p = lane; p < lists; p += 32) {
        const uint32_t c = G.cand_cnt[l0 + p];
        ovf |= c > list_cap(J, p);
        total += c;
    }
    ovf = __any_sync(0xffffffffu, ovf);
    total = __reduce_add_sync(0xffffffffu, total);
    if (ovf) {
        if (lane == 0) {
            const uint32_t at = atomicAdd(&J.cnt->ovf_count, 1u);
            J.ovf_list[at] = row;
        }
        return 0;
    }
    unsigned long long *region = row_region(J, G, row);
    // Threshold: the exact k-th smallest screened value of the row, over the
    // emitted candidates (they include the row's k smallest).  Up to RR_CBUF
    // candidates are staged in shared memory and the k-th found by a bitwise
    // search on the order-preserving keys; longer rows use a warp top-k.
    const bool staged = total <= RR_CBUF;
    float tau = __int_as_float(0x7f800000);
    if (staged) {
        uint32_t base = 0;
        for (uint32_t p = 0; p < lists; ++p) {
            const uint32_t cnt = G.cand_cnt[l0 + p];
            const unsigned long long *cand = region + (size_t)p * J.cap;
            for (uint32_t e = lane; e < cnt; e += 32) sm.cbuf[base + e] = cand[e];
            base += cnt;
        }
        __syncwarp();
        if (total >= k)
            tau = unord32(kth_of([&](uint32_t e) { return ord32(__uint_as_float((uint32_t)(sm.cbuf[e] >> 32))); },
                                 total, k, lane));
    } else {
        WarpTopK<KPL> sel;
        sel.reset();
        for (uint32_t p = 0; p < lists; ++p) {
            const uint32_t cnt = G.cand_cnt[l0 + p];
            const unsigned long long *cand = region + (size_t)p * J.cap;
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

    // Compaction of the candidates within tau^ + band to the front of the
    // region.  From the lists themselves this is in place and safe: a write
    // lands at most at (entries kept so far) + 31 <= (position of the chunk
    // being read) + 31, every entry of which is already in registers.
    const unsigned lt_mask = (1u << lane) - 1u;
    uint32_t fill = 0;
    auto compact = [&](const unsigned long long *src, uint32_t cnt) {
        for (uint32_t e0 = 0; e0 < cnt; e0 += 32) {
            bool pass = false;
            unsigned long long c = 0;
            if (e0 + lane < cnt) {
                c = src[e0 + lane];
                pass = !(__uint_as_float((uint32_t)(c >> 32)) > thr);
            }
            const unsigned m = __ballot_sync(0xffffffffu, pass);
            if (pass) region[fill + __popc(m & lt_mask)] = c;
            fill += __popc(m);
        }
    };
    if (staged) {
        compact(sm.cbuf, total);
    } else {
        for (uint32_t p = 0; p < lists; ++p) compact(region + (size_t)p * J.cap, G.cand_cnt[l0 + p]);
    }
    __syncwarp();
    return fill;
}

// Phase 2: exact distances of the flat survivor sequence of the warp's rows
// (group rows gr0 .. gr0 + 7; lane r < 8 holds row r's count in `cnt_l`).
template <int METRIC>
__device__ __forceinline__ void exact_pairs(const JobDev &J, const GroupDev &G, uint32_t gr0, uint32_t cnt_l,
                                            RrWarpSmem &sm, int lane) {
    const uint32_t d = J.d;
    const float *__restrict__ x = J.x;
    // inclusive / exclusive scans of the eight counts (lanes 0-7)
    uint32_t incl = lane < RR_ROWS ? cnt_l : 0u;
#pragma unroll
    for (int o = 1; o < RR_ROWS; o <<= 1) {
        const uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
    }
    const uint32_t excl = incl - (lane < RR_ROWS ? cnt_l : 0u);
    const uint32_t total = __shfl_sync(0xffffffffu, incl, RR_ROWS - 1);
    // 16-byte staging when every candidate chunk starts 16-byte aligned
    const bool vec = (d & 3u) == 0 && (reinterpret_cast<uintptr_t>(x) & 15u) == 0;
    const uint32_t nch = (d + RR_CH - 1) / RR_CH;

    for (uint32_t s = 0; s < total;) {
        // rows of the slice: the first is the row holding pair s; a slice
        // ends at 32 pairs, at the total, or where a fifth row would begin
        const uint32_t r_s = __popc(__ballot_sync(0xffffffffu, lane < RR_ROWS && incl <= s));
        uint32_t end = min(s + 32, total);
        if (r_s + RR_QROWS < RR_ROWS) end = min(end, __shfl_sync(0xffffffffu, excl, r_s + RR_QROWS));
        const uint32_t p = s + lane;
        const bool active = p < end;
        uint32_t ri = 0;  // the lane's row, relative to r_s
#pragma unroll
        for (uint32_t q = 1; q < RR_QROWS; ++q) {
            const uint32_t e = __shfl_sync(0xffffffffu, excl, min(r_s + q, (uint32_t)RR_ROWS - 1));
            if (r_s + q < RR_ROWS && p >= e) ri = q;
        }
        const uint32_t last = __shfl_sync(0xffffffffu, ri, min(end - s, 32u) - 1);
        const uint32_t nr = last + 1;  // query rows staged for this slice
        const uint32_t my_excl = __shfl_sync(0xffffffffu, excl, r_s + ri);
        const uint32_t row = gr0 + r_s + ri - J.row0;  // job-local
        // idle lanes (p >= end) may name a padding row: they read nothing
        unsigned long long *slot = row_region(J, G, row) + (p - my_excl);
        uint32_t j = 0;
        if (active) j = (uint32_t)*slot;
        const uint32_t j0 = __shfl_sync(0xffffffffu, j, 0);
        if (!active) j = j0;  // idle lanes stage a valid row (lane 0's)
        sm.ex.cj[lane] = j;
        __syncwarp();

        auto issue = [&](uint32_t c, uint32_t st) {
            const uint32_t dim0 = c * RR_CH;
            if (vec) {
                const uint32_t sub = (uint32_t)lane & 7u, dp = dim0 + 4 * sub;
                const uint32_t bytes = dp < d ? 16u : 0u;  // d % 4 == 0: a piece is all in or all out
#pragma unroll
                for (uint32_t i = 0; i < 8; ++i) {
                    const uint32_t cand = 4 * i + ((uint32_t)lane >> 3);
                    const float *src = x + (size_t)sm.ex.cj[cand] * d + (bytes ? dp : 0u);
                    cp_async16(&sm.ex.xj[st][cand][4 * sub], src, bytes);
                }
            } else {
                const uint32_t dp = dim0 + (uint32_t)lane;
                const uint32_t bytes = dp < d ? 4u : 0u;
                for (uint32_t cand = 0; cand < 32; ++cand) {
                    const float *src = x + (size_t)sm.ex.cj[cand] * d + (bytes ? dp : 0u);
                    cp_async4(&sm.ex.xj[st][cand][lane], src, bytes);
                }
            }
            const uint32_t dp = dim0 + (uint32_t)lane;
            const uint32_t bytes = dp < d ? 4u : 0u;
            for (uint32_t a = 0; a < nr; ++a) {
                const uint32_t qrow = gr0 + r_s + a - J.row0;
                cp_async4(&sm.ex.xi[st][a][lane], x + (size_t)qrow * d + (bytes ? dp : 0u), bytes);
            }
        };

        issue(0, 0);
        cp_async_commit();
        if (nch > 1) issue(1, 1);
        cp_async_commit();
        double acc = 0.0;
        for (uint32_t c = 0; c < nch; ++c) {
            if (c + 2 < nch) issue(c + 2, (c + 2) % RR_STAGES);
            cp_async_commit();  // possibly empty: keeps the group count uniform
            cp_async_wait<2>();
            __syncwarp();
            const uint32_t st = c % RR_STAGES;
            for (uint32_t a = 0; a < nr; ++a) sm.ex.xid[a][lane] = (double)sm.ex.xi[st][a][lane];
            __syncwarp();
            const double *xiv = sm.ex.xid[ri];
            const float *xjv = sm.ex.xj[st][lane];
            const uint32_t tmax = min((uint32_t)RR_CH, d - c * RR_CH);
            if (tmax == RR_CH) {
#pragma unroll
                for (int q = 0; q < RR_CH / 4; ++q) {
                    const float4 y = *reinterpret_cast<const float4 *>(xjv + 4 * q);
                    const double2 a0 = *reinterpret_cast<const double2 *>(xiv + 4 * q);
                    const double2 a1 = *reinterpret_cast<const double2 *>(xiv + 4 * q + 2);
                    acc = step<METRIC>(acc, a0.x, (double)y.x);
                    acc = step<METRIC>(acc, a0.y, (double)y.y);
                    acc = step<METRIC>(acc, a1.x, (double)y.z);
                    acc = step<METRIC>(acc, a1.y, (double)y.w);
                }
            } else {
                for (uint32_t t = 0; t < tmax; ++t) acc = step<METRIC>(acc, xiv[t], (double)xjv[t]);
            }
            __syncwarp();
        }
        if (active) {
            float dist;
            if (j == row) {
                dist = 0.0f;  // src/knn.rs:38-39
            } else if (METRIC == HM_METRIC_EUCLIDEAN) {
                dist = __double2float_rn(__dsqrt_rn(acc));
            } else {
                const double q = __ddiv_rn(acc, __dmul_rn(J.rnorm[row], J.rnorm[j]));
                const double r = __dsub_rn(1.0, q);
                dist = (r > 0.0) ? __double2float_rn(r) : 0.0f;
            }
            *slot = make_key(dist, j);
        }
        __syncwarp();
        s = end;
    }
}

template <int KPL>
__global__ void __launch_bounds__(RR_WARPS * 32) rerank_kernel(const JobDev *__restrict__ jobs,
                                                               const GroupDev *__restrict__ Gp) {
    extern __shared__ __align__(16) unsigned char rr_smem_raw[];
    const GroupDev &G = *Gp;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    RrWarpSmem &sm = reinterpret_cast<RrWarpSmem *>(rr_smem_raw)[warp];
    const uint32_t gr0 = (blockIdx.x * RR_WARPS + warp) * RR_ROWS;
    if (gr0 >= G.rows) return;
    // gr0 is 8-aligned and every job's rows start 32-aligned: the warp's
    // rows belong to one job (or are padding after it)
    const JobDev &J = jobs[G.job_ids[find_job(G.row_starts, G.njobs, gr0)]];
    uint32_t cnt_l = 0, kept = 0, kept_max = 0;
    for (uint32_t r = 0; r < RR_ROWS; ++r) {
        const uint32_t row = gr0 + r - J.row0;
        uint32_t c = 0;
        if (row < J.n && row >= J.q0 && row < J.q1) c = select_row<KPL>(J, G, gr0 + r, row, sm, lane);
        if ((uint32_t)lane == r) cnt_l = c;
        kept += c;
        kept_max = max(kept_max, c);
    }
    if (__any_sync(0xffffffffu, cnt_l != 0)) {
        if (J.metric == HM_METRIC_EUCLIDEAN)
            exact_pairs<HM_METRIC_EUCLIDEAN>(J, G, gr0, cnt_l, sm, lane);
        else
            exact_pairs<HM_METRIC_COSINE>(J, G, gr0, cnt_l, sm, lane);
    }
    // phase 3: each row's k smallest exact keys
    const uint32_t k = J.k;
    for (uint32_t r = 0; r < RR_ROWS; ++r) {
        const uint32_t c = __shfl_sync(0xffffffffu, cnt_l, r);
        if (c == 0) continue;
        const uint32_t row = gr0 + r - J.row0;
        const unsigned long long *keys = row_region(J, G, row);
        WarpTopK<KPL> top;
        top.reset();
        for (uint32_t e0 = 0; e0 < c; e0 += 32)
            top.offer(e0 + lane < c ? (uint64_t)keys[e0 + lane] : KEY_NONE, k, lane);
#pragma unroll
        for (int q = 0; q < KPL; ++q) {
            const uint32_t e = q * 32 + lane;
            if (e < k) {
                J.idx[(size_t)row * k + e] = key_idx(top.v[q]);
                J.dist[(size_t)row * k + e] = key_dist(top.v[q]);
            }
        }
    }
    if (lane == 0 && kept) {
        atomicAdd(&J.cnt->candidates, (unsigned long long)kept);
        atomicMax(&J.cnt->max_row, kept_max);
    }
}

// Symmetric emission: each row's emission limit tau1 + 2 band (rounded up)
// and its raw-product form v* for cosine rows, for the column-side tests of
// the tiles above the diagonal; rows that take no column-side candidates
// (padding, zero vectors under cosine, jobs without the symmetric form) get
// limits nothing passes.
__global__ void __launch_bounds__(256) emit_limits_kernel(const JobDev *__restrict__ jobs,
                                                         const GroupDev *__restrict__ Gp, uint32_t padded) {
    const GroupDev &G = *Gp;
    const uint32_t gr = blockIdx.x * blockDim.x + threadIdx.x;
    if (gr >= padded) return;
    const float INF = __int_as_float(0x7f800000);
    float lim = -INF, vs = INF;
    if (gr < G.rows) {
        const JobDev &J = jobs[G.job_ids[find_job(G.row_starts, G.njobs, gr)]];
        const uint32_t row = gr - J.row0;
        if (J.sym && row < J.n && !G.force[gr]) {
            const float b = G.band[gr];
            lim = __fadd_ru(__fadd_ru(unord32(G.rowthr[gr]), b), b);
            vs = !(lim < INF) ? -INF : __fsub_rd(__fsub_rd(1.0f, lim), fmaxf(fabsf(lim), 1.0f) * 0x1p-20f);
        }
    }
    G.ethr[gr] = lim;
    G.evstar[gr] = vs;
}

int launch_emit_limits(const JobDev *jobs, const GroupDev &G, const GroupDev *Gd, cudaStream_t s) {
    ScopedKernelTimer timer(HM_KCLASS_SELECT, s);
    const uint32_t padded = (uint32_t)(round_up(G.rows, SC_BN) + SC_BN);
    emit_limits_kernel<<<(padded + 255) / 256, 256, 0, s>>>(jobs, Gd, padded);
    HM_CUDA_TRY(cudaGetLastError());
    count_launch();
    return HM_OK;
}

// Symmetric emission: the column-side candidates the emission pass staged
// (per CTA: the column's group row, the raw product and the candidate row)
// move into the rows' column lists with their exact screened values
// c^_ji = rowterm_j + colterm_i - scale v, the arithmetic row j's own tiles
// use.  blockIdx.y is the staging CTA.
__global__ void __launch_bounds__(256) column_scatter_kernel(const JobDev *__restrict__ jobs,
                                                            const GroupDev *__restrict__ Gp) {
    const GroupDev &G = *Gp;
    const uint32_t c = blockIdx.y;
    const uint32_t cnt = min(G.stage_cnt[c], G.stage_cap);
    for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < cnt; e += gridDim.x * blockDim.x) {
        const size_t at = (size_t)c * G.stage_cap + e;
        const uint32_t gr = G.stage_row[at];
        const unsigned long long key = G.stage_key[at];
        const JobDev &J = jobs[G.job_ids[find_job(G.row_starts, G.njobs, gr)]];
        const uint32_t j = gr - J.row0, i = (uint32_t)key;
        const float v = __uint_as_float((uint32_t)(key >> 32));
        const float rt = J.metric == HM_METRIC_EUCLIDEAN ? G.colterm[gr] : 0.0f;
        const float c2 = __fsub_rn(__fadd_rn(rt, G.colterm[J.row0 + i]), __fmul_rn(J.scale, v));
        const size_t l = cand_list(J, j, J.elists - 2);
        const uint32_t slot = atomicAdd(&G.cand_cnt[l], 1u);
        if (slot < 2 * J.cap) cand_slots(J, G, l)[slot] = ((unsigned long long)__float_as_uint(c2) << 32) | i;
    }
}

int launch_column_scatter(const JobDev *jobs, const GroupDev &G, const GroupDev *Gd, uint32_t ctas,
                          cudaStream_t s) {
    if (ctas == 0) return HM_OK;
    ScopedKernelTimer timer(HM_KCLASS_SELECT, s);
    column_scatter_kernel<<<dim3(8, ctas), 256, 0, s>>>(jobs, Gd);
    HM_CUDA_TRY(cudaGetLastError());
    count_launch();
    return HM_OK;
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

// One launch covers every job of the group, both metrics.
int launch_rerank(const JobDev *jobs, const GroupDev &G, const GroupDev *Gd, uint32_t kpl, uint32_t,
                  int, cudaStream_t s) {
    if (G.rows == 0) return HM_OK;
    ScopedKernelTimer timer(HM_KCLASS_SELECT, s);
    const size_t smem = (size_t)RR_WARPS * sizeof(RrWarpSmem);
    const uint32_t warps = (G.rows + RR_ROWS - 1) / RR_ROWS;
    const int blocks = (int)((warps + RR_WARPS - 1) / RR_WARPS);
    switch (kpl) {
    case 1:
        HM_TRY(ensure_dynamic_smem((const void *)rerank_kernel<1>, (int)smem));
        rerank_kernel<1><<<blocks, RR_WARPS * 32, smem, s>>>(jobs, Gd);
        break;
    case 2:
        HM_TRY(ensure_dynamic_smem((const void *)rerank_kernel<2>, (int)smem));
        rerank_kernel<2><<<blocks, RR_WARPS * 32, smem, s>>>(jobs, Gd);
        break;
    default: return set_error(HM_ERR_UNSUPPORTED, "rerank width %u", kpl);
    }
    HM_CUDA_TRY(cudaGetLastError());
    count_launch();
    return HM_OK;
}

}  // namespace hm
