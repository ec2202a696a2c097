// rerank.cu -- the row threshold between the two screen passes, and the
// exact rerank of the screen's candidates.
//
// threshold: one warp per row merges the k smallest mini-chunk minima of the
// row's lists into tau1, the k-th smallest of their union rounded up to 2^-13
// of its binade.  Every mini-chunk minimum is a screened value of the row, so
// at least k screened values are <= tau1 and the row's k-th smallest screened
// value tau^ <= tau1.
//
// rerank: one warp per 8 consecutive group rows (always of one job: each job's
// rows start 32-aligned in the group), in three phases.
//   1. select, per row: tau^ is recomputed as the k-th smallest screened
//      value among the emitted candidates (the emission pass wrote every
//      column with c^ <= tau1 + band, which includes the k smallest), rounded
//      up to 2^-15 of its binade (a larger threshold keeps a superset), and
//      the candidates with c^ <= tau^ + band are compacted in place to the
//      front of the row's own list region.  Rows whose list overflowed, or that
//      the screen cannot bound (zero vectors under cosine), are appended to the
//      overflow list for the exact plain path.
//   2. exact distances: the survivors of the warp's rows are taken as one flat
//      sequence and processed 32 at a time (a slice never spans more than 4
//      rows), one candidate per lane.  The candidate rows are staged through
//      shared memory 32 dimensions at a time by cp.async with coalesced
//      128-byte reads (8 lanes per candidate row; a 2-stage pipeline), the
//      query rows' chunks beside them, converted once to binary64; each lane
//      then accumulates its pair exactly as the reference does
//      (src/metric.rs:42-53 euclidean, :58-70 cosine: binary64, dimension
//      order, no contraction; self forced to 0 as in src/knn.rs:38-39) and
//      overwrites its survivor's slot with the (distance bits, index) key.
//   3. select, per row: the k smallest keys of its survivors (the reference's
//      (total_cmp(dist), index) order, src/knn.rs:46-52) are the row's output.
#include <cuda_runtime.h>

#include "hm_internal.cuh"
#include "mbarrier.cuh"
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

// Upper bound of the k-th smallest of a warp's `total` keys (at most 32 * NQ;
// lane l holds keys l, l + 32, ...; absent keys are ~0) that is exact but for
// the key bits below `lo`: the largest r with fewer than k keys below it is
// found bit by bit from the highest bit where the keys differ down to bit lo,
// so r holds the k-th smallest key's bits from lo up; the bits below lo are
// returned as ones (capped at the largest key).  lo = 0 gives the k-th
// smallest itself.
template <int NQ>
__device__ __forceinline__ uint32_t kth_key(const uint32_t (&ov)[NQ], uint32_t total, uint32_t k, int lo,
                                            int lane) {
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
    for (int b = top; b >= lo; --b) {
        const uint32_t t = r | (1u << b);
        uint32_t c = 0;
#pragma unroll
        for (int q = 0; q < NQ; ++q) c += ov[q] < t ? 1u : 0u;
        c = __reduce_add_sync(0xffffffffu, c);
        if (c < k) r = t;
    }
    return min(r | ((1u << lo) - 1u), mx);
}

// kth_key over keys key(e), e < total <= 512, with the register count
// chosen by the total
template <int NQ, typename KeyFn>
__device__ __forceinline__ uint32_t kth_load(KeyFn key, uint32_t total, uint32_t k, int lo, int lane) {
    uint32_t ov[NQ];
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
        const uint32_t e = q * 32 + lane;
        ov[q] = e < total ? key(e) : 0xffffffffu;
    }
    return kth_key<NQ>(ov, total, k, lo, lane);
}

template <typename KeyFn>
__device__ __forceinline__ uint32_t kth_of(KeyFn key, uint32_t total, uint32_t k, int lo, int lane) {
    if (total <= 32) return kth_load<1>(key, total, k, lo, lane);
    if (total <= 64) return kth_load<2>(key, total, k, lo, lane);
    if (total <= 128) return kth_load<4>(key, total, k, lo, lane);
    if (total <= 256) return kth_load<8>(key, total, k, lo, lane);
    return kth_load<16>(key, total, k, lo, lane);
}

constexpr int RR_ROWS = 8;        // group rows per warp of the exact phase
constexpr int RR_WARPS = 4;       // warps per block of the exact phase
constexpr int RR_CBUF = 512;      // emitted candidates a warp stages in shared memory
constexpr int RS_WARPS = 8;       // rows (warps) per block of the select and top-k phases
constexpr int RR_STAGES = 2;      // chunks in flight (11.5 KB of shared memory per warp)
constexpr int RR_CH = 32;         // dimensions per chunk
constexpr int RR_XJ_STRIDE = 36;  // floats per staged candidate chunk (144 B: 16-byte aligned rows
                                  // whose 16-byte reads by 32 lanes need the minimum 4 wavefronts)
constexpr int RR_QROWS = 4;       // query rows per slice
constexpr int RR_XI_STRIDE = 36;  // doubles per converted query-row chunk (rows 8 banks apart)

// Shared memory of one warp of the exact phase: the chunk pipeline.
struct RrWarpSmem {
    struct {
        float xj[RR_STAGES][32][RR_XJ_STRIDE];
        float xi[RR_STAGES][RR_QROWS][32];
        double xid[RR_QROWS][RR_XI_STRIDE];
        uint32_t cj[32];
    } ex;
};

// Shared memory of one warp of the select phase: the row's emitted
// candidates and the radix-select histogram.
struct RsWarpSmem {
    unsigned long long cbuf[RR_CBUF];
    uint32_t hist[256];
    uint32_t loff[32];  // first staged position of each list
};

// global -> shared copies that zero-fill the bytes past src_bytes (0 reads nothing)
__device__ __forceinline__ void cp_async16(void *dst, const void *src, uint32_t src_bytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(smem_u32(dst)), "l"(src), "r"(src_bytes)
                 : "memory");
}
__device__ __forceinline__ void cp_async4(void *dst, const void *src, uint32_t src_bytes) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(smem_u32(dst)), "l"(src), "r"(src_bytes)
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

// Upper bound of the k-th smallest (1-based k <= total) of the order-
// preserving keys held in registers (lane l: keys l, l + 32, ...; NQ per
// lane), exact but for its lowest byte, which is returned as ones (capped at
// the largest key): a most-significant-byte-first radix select, each pass
// counting the keys that share the bytes chosen so far in 256 shared-memory
// bins, the bin holding the k-th fixing the next byte.  Bytes the keys all
// share are skipped, and so is the last byte: a threshold above the k-th
// smallest by less than 2^-15 of its binade only keeps a superset.
template <int NQ>
__device__ __forceinline__ uint32_t radix_kth(const uint32_t (&key)[NQ], uint32_t total, uint32_t k,
                                              uint32_t *hist, int lane) {
    uint32_t mn = 0xffffffffu, mx = 0u;
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
        if ((uint32_t)(q * 32 + lane) < total) {
            mn = min(mn, key[q]);
            mx = max(mx, key[q]);
        }
    }
    mn = __reduce_min_sync(0xffffffffu, mn);
    mx = __reduce_max_sync(0xffffffffu, mx);
    if (mn == mx) return mn;
    const int hb = (31 - __clz(mn ^ mx)) >> 3;  // highest byte where the keys differ
    uint32_t mask = hb == 3 ? 0u : ~((1u << (8 * hb + 8)) - 1u);
    uint32_t prefix = mn & mask, kk = k;
    for (int shift = 8 * hb; shift >= 8; shift -= 8) {
        for (int b = lane; b < 256; b += 32) hist[b] = 0u;
        __syncwarp();
#pragma unroll
        for (int q = 0; q < NQ; ++q)
            if ((uint32_t)(q * 32 + lane) < total && (key[q] & mask) == prefix)
                atomicAdd(&hist[(key[q] >> shift) & 255u], 1u);
        __syncwarp();
        // lane l holds bins [8 l, 8 l + 8): the bin where the count reaches kk
        uint32_t h[8], sum = 0;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            h[j] = hist[8 * lane + j];
            sum += h[j];
        }
        uint32_t incl = sum;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        const int owner = __ffs(__ballot_sync(0xffffffffu, incl >= kk)) - 1;
        uint32_t bin = 0, below = incl - sum;
        bool found = false;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            if (!found && below + h[j] >= kk) {
                bin = 8 * lane + j;
                found = true;
            } else if (!found) {
                below += h[j];
            }
        }
        bin = __shfl_sync(0xffffffffu, bin, owner);
        below = __shfl_sync(0xffffffffu, below, owner);
        kk -= below;
        prefix |= bin << shift;
        mask |= 255u << shift;
        __syncwarp();
    }
    return min(prefix | 0xffu, mx);
}

template <int NQ>
__device__ __forceinline__ uint32_t kth_staged(const unsigned long long *cbuf, uint32_t total, uint32_t k,
                                               uint32_t *hist, int lane) {
    uint32_t key[NQ];
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
        const uint32_t e = q * 32 + lane;
        key[q] = e < total ? ord32(__uint_as_float((uint32_t)(cbuf[e] >> 32))) : 0xffffffffu;
    }
    return radix_kth<NQ>(key, total, k, hist, lane);
}

// Select phase for one row: returns the survivor count (0 for rows sent to
// the exact fallback).
template <int KPL>
__device__ __forceinline__ uint32_t select_row(const JobDev &J, const GroupDev &G, uint32_t gr, uint32_t row,
                                               RsWarpSmem &sm, int lane) {
    const uint32_t k = J.k, lists = J.elists;
    const size_t l0 = cand_list(J, row, 0);
    // lane p < lists holds list p's count; overflow / unbounded rows go to
    // the exact plain path
    const uint32_t myc = (uint32_t)lane < lists ? G.cand_cnt[l0 + lane] : 0u;
    const bool ovf = __any_sync(0xffffffffu, G.force[gr] != 0 || ((uint32_t)lane < lists && myc > list_cap(J, lane)));
    if (ovf) {
        if (lane == 0) {
            const uint32_t at = atomicAdd(&J.out->ovf_count, 1u);
            J.ovf_list[at] = row;
        }
        return 0;
    }
    uint32_t incl = myc;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
    unsigned long long *region = row_region(J, G, row);
    // Threshold: the k-th smallest screened value of the row over the emitted
    // candidates (they include the row's k smallest).  Up to RR_CBUF
    // candidates are staged in shared memory (every list's chunk c loaded
    // before any is stored) and the k-th bounded from above by a radix select
    // (to its lowest key byte); longer rows use a warp top-k (exact).
    const bool staged = total <= RR_CBUF;
    float tau = __int_as_float(0x7f800000);
    if (staged) {
        // flat copy: staged position e lies in the last list whose first
        // position is <= e (an empty list shares its successor's first
        // position, so the search lands on the list that holds e)
        if ((uint32_t)lane < lists) sm.loff[lane] = incl - myc;
        __syncwarp();
        for (uint32_t e0 = 0; e0 < total; e0 += 128) {
            unsigned long long v[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const uint32_t e = e0 + 32 * u + lane;
                if (e < total) {
                    uint32_t lo = 0, hi = lists;
                    while (hi - lo > 1) {
                        const uint32_t mid = (lo + hi) >> 1;
                        if (sm.loff[mid] <= e) lo = mid; else hi = mid;
                    }
                    v[u] = region[(size_t)lo * J.cap + (e - sm.loff[lo])];
                }
            }
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const uint32_t e = e0 + 32 * u + lane;
                if (e < total) sm.cbuf[e] = v[u];
            }
        }
        __syncwarp();
        if (total >= k) {
            uint32_t r;
            if (total <= 128) r = kth_staged<4>(sm.cbuf, total, k, sm.hist, lane);
            else if (total <= 256) r = kth_staged<8>(sm.cbuf, total, k, sm.hist, lane);
            else r = kth_staged<16>(sm.cbuf, total, k, sm.hist, lane);
            tau = unord32(r);
        }
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

// Select phase: one warp per group row; the block's rows (8-aligned) belong
// to one job, whose counters take one update per block.
template <int KPL>
__global__ void __launch_bounds__(RS_WARPS * 32, 4) rr_select_kernel(const JobDev *__restrict__ jobs,
                                                                  const GroupDev *__restrict__ Gp) {
    extern __shared__ __align__(16) unsigned char rs_smem_raw[];
    __shared__ uint32_t s_kept[RS_WARPS];
    const GroupDev &G = *Gp;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    RsWarpSmem &sm = reinterpret_cast<RsWarpSmem *>(rs_smem_raw)[warp];
    const uint32_t gr = blockIdx.x * RS_WARPS + warp;
    const uint32_t g0 = blockIdx.x * RS_WARPS;
    const JobDev &J = jobs[G.job_ids[find_job(G.row_starts, G.njobs, g0 < G.rows ? g0 : 0u)]];
    uint32_t c = 0;
    if (gr < G.rows) {
        const uint32_t row = gr - J.row0;
        if (row < J.n && row >= J.q0 && row < J.q1 && job_active(J)) c = select_row<KPL>(J, G, gr, row, sm, lane);
        if (lane == 0) G.row_cnt[gr] = c;
    }
    if (lane == 0) s_kept[warp] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t sum = 0, mx = 0;
        for (int w = 0; w < RS_WARPS; ++w) {
            sum += s_kept[w];
            mx = max(mx, s_kept[w]);
        }
        if (sum) {
            atomicAdd(&J.out->candidates, (unsigned long long)sum);
            atomicMax(&J.out->max_row, mx);
        }
    }
}

// The (distance bits, index) key of pair (row, j) from its binary64
// accumulation: the reference's final step of each metric, the self pair
// forced to 0 (src/knn.rs:38-39).
template <int METRIC>
__device__ __forceinline__ unsigned long long pair_key(const JobDev &J, uint32_t row, uint32_t j, double acc) {
    float dist;
    if (j == row) {
        dist = 0.0f;
    } else if (METRIC == HM_METRIC_EUCLIDEAN) {
        dist = __double2float_rn(__dsqrt_rn(acc));
    } else {
        const double q = __ddiv_rn(acc, __dmul_rn(J.rnorm[row], J.rnorm[j]));
        const double r = __dsub_rn(1.0, q);
        dist = (r > 0.0) ? __double2float_rn(r) : 0.0f;
    }
    return make_key(dist, j);
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

        // the rows this lane copies from, fixed for the slice: candidate
        // 4 i + lane / 8 (16-byte pieces, vector path) and query row a
        const uint32_t sub = (uint32_t)lane & 7u;
        const float *cp[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) cp[i] = x + (size_t)sm.ex.cj[4 * i + ((uint32_t)lane >> 3)] * d + 4 * sub;
        const float *qp[RR_QROWS];
#pragma unroll
        for (int a = 0; a < RR_QROWS; ++a)
            qp[a] = x + (size_t)(gr0 + r_s + min((uint32_t)a, nr - 1) - J.row0) * d + lane;

        auto issue = [&](uint32_t c, uint32_t st) {
            const uint32_t dim0 = c * RR_CH;
            if (vec) {
                const bool in = dim0 + 4 * sub < d;  // d % 4 == 0: a piece is all in or all out
#pragma unroll
                for (int i = 0; i < 8; ++i) {
                    const uint32_t cand = 4 * i + ((uint32_t)lane >> 3);
                    cp_async16(&sm.ex.xj[st][cand][4 * sub], in ? cp[i] + dim0 : cp[i], in ? 16u : 0u);
                }
            } else {
                const uint32_t dp = dim0 + (uint32_t)lane;
                const uint32_t bytes = dp < d ? 4u : 0u;
                for (uint32_t cand = 0; cand < 32; ++cand) {
                    const float *src = x + (size_t)sm.ex.cj[cand] * d + (bytes ? dp : 0u);
                    cp_async4(&sm.ex.xj[st][cand][lane], src, bytes);
                }
            }
            const bool qin = dim0 + (uint32_t)lane < d;
#pragma unroll
            for (int a = 0; a < RR_QROWS; ++a)
                if ((uint32_t)a < nr) cp_async4(&sm.ex.xi[st][a][lane], qin ? qp[a] + dim0 : qp[a] - lane, qin ? 4u : 0u);
        };

        for (uint32_t c = 0; c + 1 < RR_STAGES; ++c) {
            if (c < nch) issue(c, c);
            cp_async_commit();
        }
        double acc = 0.0;
        for (uint32_t c = 0; c < nch; ++c) {
            if (c + RR_STAGES - 1 < nch) issue(c + RR_STAGES - 1, (c + RR_STAGES - 1) % RR_STAGES);
            cp_async_commit();  // possibly empty: keeps the group count uniform
            cp_async_wait<RR_STAGES - 1>();
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
        if (active) *slot = pair_key<METRIC>(J, row, j, acc);
        __syncwarp();
        s = end;
    }
}

// Exact phase: one warp per 8 consecutive group rows (always of one job:
// each job's rows start 32-aligned in the group).
__global__ void __launch_bounds__(RR_WARPS * 32) rr_exact_kernel(const JobDev *__restrict__ jobs,
                                                                 const GroupDev *__restrict__ Gp) {
    extern __shared__ __align__(16) unsigned char rr_smem_raw[];
    const GroupDev &G = *Gp;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    RrWarpSmem &sm = reinterpret_cast<RrWarpSmem *>(rr_smem_raw)[warp];
    const uint32_t gr0 = (blockIdx.x * RR_WARPS + warp) * RR_ROWS;
    if (gr0 >= G.rows) return;
    const JobDev &J = jobs[G.job_ids[find_job(G.row_starts, G.njobs, gr0)]];
    const uint32_t cnt_l = lane < RR_ROWS ? G.row_cnt[gr0 + lane] : 0u;
    if (!__any_sync(0xffffffffu, cnt_l != 0)) return;
    if (J.metric == HM_METRIC_EUCLIDEAN)
        exact_pairs<HM_METRIC_EUCLIDEAN>(J, G, gr0, cnt_l, sm, lane);
    else
        exact_pairs<HM_METRIC_COSINE>(J, G, gr0, cnt_l, sm, lane);
}

// Bitonic sort of 64 keys held two per lane (element lane and 32 + lane),
// ascending.
__device__ __forceinline__ void bitonic64(uint64_t &a, uint64_t &b, int lane) {
#pragma unroll
    for (int size = 2; size <= 64; size <<= 1) {
#pragma unroll
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            if (stride == 32) {
                const uint64_t lo = a < b ? a : b, hi = a < b ? b : a;
                a = lo;  // size 64: every pair ascending
                b = hi;
            } else {
                const bool lower = (lane & stride) == 0;
                const uint64_t pa = shfl_xor_u64(a, stride), pb = shfl_xor_u64(b, stride);
                const bool asc0 = (lane & size) == 0, asc1 = ((32 + lane) & size) == 0;
                a = (lower == asc0) ? (a < pa ? a : pa) : (a < pa ? pa : a);
                b = (lower == asc1) ? (b < pb ? b : pb) : (b < pb ? pb : b);
            }
        }
    }
}

// Top-k phase: one warp per group row; the k smallest exact keys of the
// row's survivors are its output.
template <int KPL>
__global__ void __launch_bounds__(RS_WARPS * 32) rr_topk_kernel(const JobDev *__restrict__ jobs,
                                                                const GroupDev *__restrict__ Gp) {
    const GroupDev &G = *Gp;
    const int lane = threadIdx.x & 31;
    const uint32_t gr = blockIdx.x * RS_WARPS + (threadIdx.x >> 5);
    if (gr >= G.rows) return;
    const uint32_t c = G.row_cnt[gr];
    if (c == 0) return;
    const JobDev &J = jobs[G.job_ids[find_job(G.row_starts, G.njobs, gr)]];
    const uint32_t row = gr - J.row0, k = J.k;
    const unsigned long long *keys = row_region(J, G, row);
    uint32_t *idx = J.idx + (size_t)row * k;
    float *dist = J.dist + (size_t)row * k;
    if (c <= 64) {
        uint64_t a = (uint32_t)lane < c ? (uint64_t)keys[lane] : KEY_NONE;
        uint64_t b = 32u + lane < c ? (uint64_t)keys[32 + lane] : KEY_NONE;
        bitonic64(a, b, lane);
        if ((uint32_t)lane < k) {
            idx[lane] = key_idx(a);
            dist[lane] = key_dist(a);
        }
        if (32u + lane < k) {
            idx[32 + lane] = key_idx(b);
            dist[32 + lane] = key_dist(b);
        }
        return;
    }
    WarpTopK<KPL> top;
    top.reset();
    for (uint32_t e0 = 0; e0 < c; e0 += 32) top.offer(e0 + lane < c ? (uint64_t)keys[e0 + lane] : KEY_NONE, k, lane);
#pragma unroll
    for (int q = 0; q < KPL; ++q) {
        const uint32_t e = q * 32 + lane;
        if (e < k) {
            idx[e] = key_idx(top.v[q]);
            dist[e] = key_dist(top.v[q]);
        }
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
// (per epilogue warp: the column's group row, the raw product and the
// candidate row) move into the rows' column lists with their exact screened
// values c^_ji = rowterm_j + colterm_i - scale v, the arithmetic row j's own
// tiles use.  blockIdx.y is the stage (CTA x SC_STAGE_SLOTS + warp).
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
constexpr int TAU1_LOW_BITS = 10;
template <int KPL>
__global__ void __launch_bounds__(256) threshold_kernel(const JobDev *__restrict__ jobs,
                                                       const GroupDev *__restrict__ Gp) {
    const GroupDev &G = *Gp;
    const int lane = threadIdx.x & 31;
    const uint32_t gr = blockIdx.x * 8 + (threadIdx.x >> 5);
    if (gr >= G.rows) return;
    const JobDev &J = jobs[G.job_ids[find_job(G.row_starts, G.njobs, gr)]];
    const uint32_t row = gr - J.row0;
    if (row < J.q0 || row >= J.q1 || !job_active(J)) return;
    const uint32_t k = J.k, lists = J.tlists * J.parts;
    const size_t l0 = list_index(J, row, 0);
    // the row's lists' arrays are contiguous: lists x k values
    const float *base = G.topk + J.topk0 + (l0 - J.slot0) * k;
    const uint32_t total = lists * k;
    if (total <= 256) {
        // tau1 is an upper bound in any case: resolving it to 2^-13 of its
        // binade (ten low key bits left as ones) emits no measurable extra
        // candidates and halves the bit loop
        const uint32_t r = kth_of([&](uint32_t e) { return ord32(base[e]); }, total, k, TAU1_LOW_BITS, lane);
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

// Escalation decision (jobs with a split-BF16 copy), after the threshold
// pass.  A row whose keep band exceeds half of its threshold tau1 (an upper
// bound of its k-th screened value) would keep a share of the dataset set by
// the screen's rounding, not by its neighbours; when more than a tenth of a
// job's rows do, the job hands over to its copy.  Both outcomes return the
// same bytes; the choice is only about time.
constexpr float ESC_BAND_SHARE = 0.5f;
constexpr uint32_t ESC_ROWS_DIV = 10;

__global__ void __launch_bounds__(256) escalate_count_kernel(const JobDev *__restrict__ jobs,
                                                             const GroupDev *__restrict__ Gp) {
    const GroupDev &G = *Gp;
    const uint32_t gr = blockIdx.x * blockDim.x + threadIdx.x;
    if (gr - (threadIdx.x & 31) >= G.rows) return;  // whole warps: 32 rows of one job
    const JobDev &J = jobs[G.job_ids[find_job(G.row_starts, G.njobs, gr - (threadIdx.x & 31))]];
    if (!J.escalation) return;
    const uint32_t row = gr - J.row0;
    bool wide = false;
    if (gr < G.rows && row < J.n && row >= J.q0 && row < J.q1 && !G.force[gr]) {
        const float tau1 = unord32(G.rowthr[gr]);
        wide = G.band[gr] > ESC_BAND_SHARE * tau1;
    }
    const uint32_t c = __popc(__ballot_sync(0xffffffffu, wide));
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(&J.cnt->escalate_rows, c);
}

__global__ void escalate_decide_kernel(const JobDev *__restrict__ jobs, const GroupDev *__restrict__ Gp) {
    const GroupDev &G = *Gp;
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= G.njobs) return;
    const JobDev &J = jobs[G.job_ids[t]];
    if (!J.escalation) return;
    if ((unsigned long long)J.cnt->escalate_rows * ESC_ROWS_DIV > (unsigned long long)(J.q1 - J.q0)) {
        J.cnt->escalate = 1;
        J.cnt->band_max_bits = 0;  // the copy reports its own band
    }
}

int launch_escalation(const JobDev *jobs, const GroupDev &G, const GroupDev *Gd, cudaStream_t s) {
    if (G.rows == 0) return HM_OK;
    ScopedKernelTimer timer(HM_KCLASS_SELECT, s);
    escalate_count_kernel<<<(G.rows + 255) / 256, 256, 0, s>>>(jobs, Gd);
    HM_CUDA_TRY(cudaGetLastError());
    count_launch();
    escalate_decide_kernel<<<(G.njobs + 127) / 128, 128, 0, s>>>(jobs, Gd);
    HM_CUDA_TRY(cudaGetLastError());
    count_launch();
    return HM_OK;
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

// Three launches cover every job of the group, both metrics: select (the
// exact tau^ and the survivors), exact distances, per-row top-k.
int launch_rerank(const JobDev *jobs, const GroupDev &G, const GroupDev *Gd, uint32_t kpl, uint32_t,
                  int, cudaStream_t s) {
    if (G.rows == 0) return HM_OK;
    if (kpl != 1 && kpl != 2) return set_error(HM_ERR_UNSUPPORTED, "rerank width %u", kpl);
    ScopedKernelTimer timer(HM_KCLASS_SELECT, s);
    const int rs_blocks = (int)((G.rows + RS_WARPS - 1) / RS_WARPS);
    const size_t rs_smem = (size_t)RS_WARPS * sizeof(RsWarpSmem);
    if (kpl == 1) {
        HM_TRY(ensure_dynamic_smem((const void *)rr_select_kernel<1>, (int)rs_smem));
        rr_select_kernel<1><<<rs_blocks, RS_WARPS * 32, rs_smem, s>>>(jobs, Gd);
    } else {
        HM_TRY(ensure_dynamic_smem((const void *)rr_select_kernel<2>, (int)rs_smem));
        rr_select_kernel<2><<<rs_blocks, RS_WARPS * 32, rs_smem, s>>>(jobs, Gd);
    }
    HM_CUDA_TRY(cudaGetLastError());
    const size_t ex_smem = (size_t)RR_WARPS * sizeof(RrWarpSmem);
    const uint32_t warps = (G.rows + RR_ROWS - 1) / RR_ROWS;
    HM_TRY(ensure_dynamic_smem((const void *)rr_exact_kernel, (int)ex_smem));
    rr_exact_kernel<<<(int)((warps + RR_WARPS - 1) / RR_WARPS), RR_WARPS * 32, ex_smem, s>>>(jobs, Gd);
    HM_CUDA_TRY(cudaGetLastError());
    if (kpl == 1)
        rr_topk_kernel<1><<<rs_blocks, RS_WARPS * 32, 0, s>>>(jobs, Gd);
    else
        rr_topk_kernel<2><<<rs_blocks, RS_WARPS * 32, 0, s>>>(jobs, Gd);
    HM_CUDA_TRY(cudaGetLastError());
    count_launch(3);
    return HM_OK;
}

}  // namespace hm
