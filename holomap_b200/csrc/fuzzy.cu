// fuzzy.cu -- the fuzzy simplicial set on the device (src/fuzzy.rs:25-91):
// the symmetrized membership graph that consumes the kNN graph and its
// calibration, as COO sorted by (row, col).
//
// Row r of the output is the sorted union of two lists: F_r, the columns of
// row r's own kNN list with a nonzero directed strength A[r][c], and R_r,
// the rows s whose lists hold r with A[s][r] nonzero.  Each is a set (the
// indices of a row are distinct), so
//
//   1. fuzzy_rows_kernel (one warp per row) computes the strengths (self
//      skipped; 1 when d - rho <= 0 or sigma == 0, else libm expf(-(d /
//      sigma)); zeros dropped), orders F_r by rank (the count of smaller
//      columns), and writes each entry's reverse copy as (key col, value e)
//      with e its position in the kNN arrays; dropped entries get the key n.
//   2. A stable radix sort of the reverse copies over the bits of n groups
//      them by column with ascending e, so each R_r comes out sorted by
//      source row (CUB onesweep).
//   3. fuzzy_merge_kernel (one warp per row) binary-searches every element
//      of F_r in R_r: it finds the partner strength A[c][r], forms the
//      binary32 t-conorm (v + vt) - v * vt in the reference's order
//      (src/fuzzy.rs:67-75), and places the element at j + lb - dups_below
//      (F elements below it, R elements below it, minus those counted in
//      both).  The row's entry count |F_r| + |R_r| - |F_r and R_r| goes
//      through an exclusive scan (CUB) to row offsets.
//   4. fuzzy_write_kernel writes the F elements at their places and every R
//      element without an F partner at u + lb_F - dups_below (the same rule
//      seen from the other list), with strength (0 + vt) - 0 * vt.
//
// Strengths lie in [0, 1] (or are NaN) when every sigma is non-negative, and
// then no fused value of a union coordinate is zero: fl(v * vt) <= min(v,
// vt) <= max(v, vt) <= fl(v + vt) with one of the inequalities strict, so
// the difference is positive.  The reference's zero filter after the fusion
// therefore drops nothing and the union size is the entry count.  Every
// step is a function of the inputs alone: the output is the reference's,
// entry for entry.
#include <cub/cub.cuh>
#include <cuda_runtime.h>

#include "hm_internal.cuh"
#include "libm_expf.cuh"

namespace hm {

constexpr unsigned FZ_FULL = 0xffffffffu;
// bits of the status word the rows kernel sets for inputs outside the
// precondition (each row's indices distinct and below n)
constexpr uint32_t FZ_BAD_INDEX = 1u, FZ_BAD_DUPLICATE = 2u;

__device__ __forceinline__ float tconorm(float v, float vt) {
    return __fsub_rn(__fadd_rn(v, vt), __fmul_rn(v, vt));
}

__global__ void __launch_bounds__(256) fuzzy_rows_kernel(
    const uint32_t *__restrict__ idx, const float *__restrict__ dist, const float *__restrict__ sigma,
    const float *__restrict__ rho, uint32_t n, uint32_t k, float *__restrict__ wdir, uint32_t *__restrict__ rkey,
    uint32_t *__restrict__ rval, uint32_t *__restrict__ fcol, float *__restrict__ fw,
    uint32_t *__restrict__ fcount, uint32_t *__restrict__ bad) {
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t r = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (r >= n) return;  // whole warps
    const uint64_t base = r * k;
    const float rh = rho[r], sg = sigma[r];
    uint32_t cnt = 0;
    for (uint32_t j0 = 0; j0 < k; j0 += 32) {
        const uint32_t j = j0 + lane;
        bool valid = false;
        if (j < k) {
            const uint32_t col = idx[base + j];
            float w = 0.0f;
            if (col >= n) {
                // outside the precondition: dropped (so every later index
                // stays in bounds) and reported through the status word
                atomicOr(bad, FZ_BAD_INDEX);
            } else if ((uint64_t)col != r) {
                const float d = __fsub_rn(dist[base + j], rh);
                w = (d <= 0.0f || sg == 0.0f) ? 1.0f : expf_libm(-__fdiv_rn(d, sg));
                valid = w != 0.0f;
            }
            wdir[base + j] = w;
            rkey[base + j] = valid ? col : n;
            rval[base + j] = (uint32_t)(base + j);
        }
        cnt += __popc(__ballot_sync(FZ_FULL, valid));
    }
    __syncwarp();
    // rank of each valid column among the row's valid columns (dropped
    // entries carry the key n, above every column).  Equal columns (outside
    // the precondition: exact_knn's indices are distinct) rank by position,
    // so every slot of the row's F list is still written, and are reported.
    for (uint32_t j0 = 0; j0 < k; j0 += 32) {
        const uint32_t j = j0 + lane;
        const uint32_t mine = j < k ? rkey[base + j] : n;
        uint32_t rank = 0;
        bool dup = false;
        for (uint32_t c0 = 0; c0 < k; c0 += 32) {
            const uint32_t other = c0 + lane < k ? rkey[base + c0 + lane] : n;
#pragma unroll
            for (int s = 0; s < 32; ++s) {
                const uint32_t o = __shfl_sync(FZ_FULL, other, s);
                const uint32_t pos = c0 + (uint32_t)s;
                rank += (o < mine || (o == mine && pos < j)) ? 1u : 0u;
                dup |= o == mine && pos != j;
            }
        }
        if (dup && mine < n) atomicOr(bad, FZ_BAD_DUPLICATE);
        if (mine < n) {
            fcol[base + rank] = mine;
            fw[base + rank] = wdir[base + j];
        }
    }
    if (lane == 0) fcount[r] = cnt;
}

// first position in [lo, hi) of the sorted array a whose value is >= x
__device__ __forceinline__ uint32_t lower_bound_u32(const uint32_t *__restrict__ a, uint32_t lo, uint32_t hi,
                                                    uint32_t x) {
    while (lo < hi) {
        const uint32_t mid = lo + ((hi - lo) >> 1);
        if (a[mid] < x) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

__global__ void __launch_bounds__(256) fuzzy_merge_kernel(
    const uint32_t *__restrict__ skey, const uint32_t *__restrict__ sval, const float *__restrict__ wdir,
    uint32_t entries, uint32_t n, uint32_t k, const uint32_t *__restrict__ fcol, float *__restrict__ fw,
    const uint32_t *__restrict__ fcount, uint32_t *__restrict__ fpos, uint32_t *__restrict__ dpre,
    uint32_t *__restrict__ rstart, uint32_t *__restrict__ rdups, uint32_t *__restrict__ count) {
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t r = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (r >= n) return;  // whole warps
    const uint64_t base = r * k;
    uint32_t b = 0;
    if (lane < 2) b = lower_bound_u32(skey, 0, entries, (uint32_t)r + lane);
    const uint32_t start = __shfl_sync(FZ_FULL, b, 0), end = __shfl_sync(FZ_FULL, b, 1);
    const uint32_t fc = fcount[r];
    uint32_t dups = 0;
    for (uint32_t j0 = 0; j0 < fc; j0 += 32) {
        const uint32_t j = j0 + lane;
        bool found = false;
        uint32_t lb = 0;
        float v = 0.0f, vt = 0.0f;
        if (j < fc) {
            const uint32_t f = fcol[base + j];
            // R_r is sorted by source row sval / k
            uint32_t lo = start, hi = end;
            while (lo < hi) {
                const uint32_t mid = lo + ((hi - lo) >> 1);
                if (sval[mid] / k < f) lo = mid + 1;
                else hi = mid;
            }
            found = lo < end && sval[lo] / k == f;
            lb = lo - start;
            v = fw[base + j];
            if (found) vt = wdir[sval[lo]];
        }
        const unsigned ball = __ballot_sync(FZ_FULL, found);
        const uint32_t before = dups + __popc(ball & ((1u << lane) - 1u));
        if (j < fc) {
            fpos[base + j] = j + lb - before;
            dpre[base + j] = before;
            fw[base + j] = tconorm(v, vt);
        }
        dups += __popc(ball);
    }
    if (lane == 0) {
        rstart[r] = start;
        rdups[r] = dups;
        count[r] = fc + (end - start) - dups;
    }
}

__global__ void __launch_bounds__(256) fuzzy_write_kernel(
    const uint32_t *__restrict__ skey, const uint32_t *__restrict__ sval, const float *__restrict__ wdir,
    uint32_t n, uint32_t k, const uint32_t *__restrict__ fcol, const float *__restrict__ fval,
    const uint32_t *__restrict__ fcount, const uint32_t *__restrict__ fpos, const uint32_t *__restrict__ dpre,
    const uint32_t *__restrict__ rstart, const uint32_t *__restrict__ rdups, const uint32_t *__restrict__ count,
    const uint32_t *__restrict__ off, uint32_t *__restrict__ rows, uint32_t *__restrict__ cols,
    float *__restrict__ vals, unsigned long long *__restrict__ nnz) {
    const uint64_t entries = (uint64_t)n * k;
    const uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p == 0) *nnz = (unsigned long long)off[n - 1] + count[n - 1];
    if (p < entries) {  // F element j of row r
        const uint32_t r = (uint32_t)(p / k), j = (uint32_t)(p - (uint64_t)r * k);
        if (j < fcount[r]) {
            const uint32_t q = off[r] + fpos[p];
            rows[q] = r;
            cols[q] = fcol[p];
            vals[q] = fval[p];
        }
    } else if (p < 2 * entries) {  // reverse copy t, an element of R_r
        const uint32_t t = (uint32_t)(p - entries);
        const uint32_t r = skey[t];
        if (r >= n) return;  // dropped entry
        const uint32_t e = sval[t];
        const uint32_t s = e / k;
        const uint64_t base = (uint64_t)r * k;
        const uint32_t fc = fcount[r];
        const uint32_t lbf = lower_bound_u32(fcol + base, 0, fc, s);
        if (lbf < fc && fcol[base + lbf] == s) return;  // written with its F partner
        // F elements below s that also lie in R_r
        const uint32_t dup_below = lbf < fc ? dpre[base + lbf] : rdups[r];
        const uint32_t q = off[r] + (t - rstart[r]) + lbf - dup_below;
        rows[q] = r;
        cols[q] = s;
        vals[q] = tconorm(0.0f, wdir[e]);
    }
}

// bits that hold every value 0..n (the key n marks a dropped entry)
static int key_bits(uint64_t n) {
    int b = 1;
    while (b < 32 && (1ull << b) <= n) ++b;
    return b;
}

// Workspace: the directed strengths, the reverse copies (double-buffered
// for the sort), the ordered F lists and their merge results, per-row
// counters, and CUB's temporary storage.
struct FuzzyLayout {
    size_t wdir, rk0, rk1, rv0, rv1, fcol, fw, fpos, dpre, fcount, rstart, rdups, count, off, bad, temp,
        temp_bytes, total;
};

static int fuzzy_layout(uint64_t n, uint32_t k, FuzzyLayout *L) {
    const uint64_t entries = n * k;
    if (n >= 0x7fffffffull || entries > 0x7fffffffull)
        return set_error(HM_ERR_UNSUPPORTED, "n k above 2^31 - 1 entries");
    size_t sort_bytes = 0, scan_bytes = 0;
    cub::DoubleBuffer<uint32_t> kb(nullptr, nullptr), vb(nullptr, nullptr);
    HM_CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, sort_bytes, kb, vb, (int)entries));
    HM_CUDA_TRY(cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, (uint32_t *)nullptr, (uint32_t *)nullptr,
                                              (int)n));
    size_t at = 0;
    auto take = [&](size_t bytes) {
        const size_t here = at;
        at = round_up(at + std::max<size_t>(bytes, 1), 256);
        return here;
    };
    const size_t e4 = entries * 4, n4 = n * 4;
    L->wdir = take(e4);
    L->rk0 = take(e4);
    L->rk1 = take(e4);
    L->rv0 = take(e4);
    L->rv1 = take(e4);
    L->fcol = take(e4);
    L->fw = take(e4);
    L->fpos = take(e4);
    L->dpre = take(e4);
    L->fcount = take(n4);
    L->rstart = take(n4);
    L->rdups = take(n4);
    L->count = take(n4);
    L->off = take(n4);
    L->bad = take(4);
    L->temp_bytes = std::max(sort_bytes, scan_bytes);
    L->temp = take(L->temp_bytes);
    L->total = at;
    return HM_OK;
}

}  // namespace hm

using namespace hm;

extern "C" {

size_t hm_fuzzy_workspace_bytes(uint64_t n, uint32_t k) {
    clear_error();
    if (n == 0 || k == 0) {
        set_error(HM_ERR_INVALID, "empty graph");
        return 0;
    }
    FuzzyLayout L;
    if (fuzzy_layout(n, k, &L) != HM_OK) return 0;
    return L.total;
}

int hm_fuzzy_graph_device(const uint32_t *d_idx, const float *d_dist, const float *d_sigma, const float *d_rho,
                          uint64_t n, uint32_t k, uint32_t *d_rows, uint32_t *d_cols, float *d_vals,
                          uint64_t *d_nnz, void *d_workspace, size_t workspace_bytes, void *stream) {
    clear_error();
    if (!d_idx || !d_dist || !d_sigma || !d_rho || !d_rows || !d_cols || !d_vals || !d_nnz || !d_workspace)
        return set_error(HM_ERR_INVALID, "NULL pointer argument");
    if (n == 0 || k == 0) return set_error(HM_ERR_INVALID, "empty graph");
    FuzzyLayout L;
    HM_TRY(fuzzy_layout(n, k, &L));
    if (workspace_bytes < L.total)
        return set_error(HM_ERR_INVALID, "workspace of %zu bytes is below the %zu needed", workspace_bytes, L.total);
    if (reinterpret_cast<uintptr_t>(d_workspace) % 256)
        return set_error(HM_ERR_INVALID, "workspace must be 256-byte aligned");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    char *ws = static_cast<char *>(d_workspace);
    auto u32 = [&](size_t o) { return reinterpret_cast<uint32_t *>(ws + o); };
    auto f32 = [&](size_t o) { return reinterpret_cast<float *>(ws + o); };
    const uint32_t nn = (uint32_t)n, entries = (uint32_t)(n * k);
    const unsigned warp_blocks = (unsigned)((n * 32 + 255) / 256);
    HM_CUDA_TRY(cudaMemsetAsync(ws + L.bad, 0, 4, s));
    fuzzy_rows_kernel<<<warp_blocks, 256, 0, s>>>(d_idx, d_dist, d_sigma, d_rho, nn, k, f32(L.wdir), u32(L.rk0),
                                                  u32(L.rv0), u32(L.fcol), f32(L.fw), u32(L.fcount),
                                                  u32(L.bad));
    HM_CUDA_TRY(cudaGetLastError());
    count_launch();
    cub::DoubleBuffer<uint32_t> kb(u32(L.rk0), u32(L.rk1)), vb(u32(L.rv0), u32(L.rv1));
    size_t temp_bytes = L.temp_bytes;
    HM_CUDA_TRY(cub::DeviceRadixSort::SortPairs(ws + L.temp, temp_bytes, kb, vb, (int)entries, 0, key_bits(n), s));
    count_launch();
    fuzzy_merge_kernel<<<warp_blocks, 256, 0, s>>>(kb.Current(), vb.Current(), f32(L.wdir), entries, nn, k,
                                                   u32(L.fcol), f32(L.fw), u32(L.fcount), u32(L.fpos), u32(L.dpre),
                                                   u32(L.rstart), u32(L.rdups), u32(L.count));
    HM_CUDA_TRY(cudaGetLastError());
    count_launch();
    temp_bytes = L.temp_bytes;
    HM_CUDA_TRY(cub::DeviceScan::ExclusiveSum(ws + L.temp, temp_bytes, u32(L.count), u32(L.off), (int)n, s));
    count_launch();
    fuzzy_write_kernel<<<(unsigned)((2ull * entries + 255) / 256), 256, 0, s>>>(
        kb.Current(), vb.Current(), f32(L.wdir), nn, k, u32(L.fcol), f32(L.fw), u32(L.fcount), u32(L.fpos),
        u32(L.dpre), u32(L.rstart), u32(L.rdups), u32(L.count), u32(L.off), d_rows, d_cols, d_vals,
        reinterpret_cast<unsigned long long *>(d_nnz));
    HM_CUDA_TRY(cudaGetLastError());
    count_launch();
    return HM_OK;
}

int hm_fuzzy_graph_status(const void *d_workspace, uint64_t n, uint32_t k, void *stream) {
    clear_error();
    if (!d_workspace) return set_error(HM_ERR_INVALID, "NULL pointer argument");
    FuzzyLayout L;
    HM_TRY(fuzzy_layout(n, k, &L));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    uint32_t bad = 0;
    HM_CUDA_TRY(cudaMemcpyAsync(&bad, static_cast<const char *>(d_workspace) + L.bad, 4,
                                cudaMemcpyDeviceToHost, s));
    HM_CUDA_TRY(cudaStreamSynchronize(s));
    if (bad & FZ_BAD_INDEX) return set_error(HM_ERR_INVALID, "a kNN index is not below n");
    if (bad & FZ_BAD_DUPLICATE) return set_error(HM_ERR_INVALID, "a row of the kNN graph repeats an index");
    return HM_OK;
}

int hm_fuzzy_graph(const uint32_t *idx, const float *dist, const float *sigma, const float *rho, uint64_t n,
                   uint32_t k, uint32_t *rows_out, uint32_t *cols_out, float *vals_out, uint64_t *nnz_out) {
    clear_error();
    if (!idx || !dist || !sigma || !rho || !rows_out || !cols_out || !vals_out || !nnz_out)
        return set_error(HM_ERR_INVALID, "NULL pointer argument");
    if (n == 0 || k == 0) return set_error(HM_ERR_INVALID, "empty graph");
    const uint64_t e = n * k, cap = 2 * e;
    for (uint64_t j = 0; j < e; ++j)
        if (idx[j] >= n) return set_error(HM_ERR_INVALID, "kNN index %u at entry %llu is not below n", idx[j],
                                          (unsigned long long)j);
    for (uint64_t i = 0; i < n; ++i)
        if (sigma[i] < 0.0f) return set_error(HM_ERR_INVALID, "sigma[%llu] is negative", (unsigned long long)i);
    FuzzyLayout L;
    HM_TRY(fuzzy_layout(n, k, &L));
    const size_t ws = L.total;
    // one device block: inputs, outputs, count, workspace (256-byte aligned parts)
    const size_t o_idx = 0, o_dist = round_up(o_idx + e * 4, 256), o_sig = round_up(o_dist + e * 4, 256);
    const size_t o_rho = round_up(o_sig + n * 4, 256), o_rows = round_up(o_rho + n * 4, 256);
    const size_t o_cols = round_up(o_rows + cap * 4, 256), o_vals = round_up(o_cols + cap * 4, 256);
    const size_t o_nnz = round_up(o_vals + cap * 4, 256), o_ws = round_up(o_nnz + 8, 256);
    char *d = nullptr;
    HM_CUDA_TRY(cudaMalloc(&d, o_ws + ws));
    int rc = HM_OK;
    uint64_t nnz = 0;
    do {
        cudaError_t err = cudaMemcpy(d + o_idx, idx, e * 4, cudaMemcpyHostToDevice);
        if (err == cudaSuccess) err = cudaMemcpy(d + o_dist, dist, e * 4, cudaMemcpyHostToDevice);
        if (err == cudaSuccess) err = cudaMemcpy(d + o_sig, sigma, n * 4, cudaMemcpyHostToDevice);
        if (err == cudaSuccess) err = cudaMemcpy(d + o_rho, rho, n * 4, cudaMemcpyHostToDevice);
        if (err != cudaSuccess) {
            rc = set_error(HM_ERR_CUDA, "copy in: %s", cudaGetErrorString(err));
            break;
        }
        rc = hm_fuzzy_graph_device(reinterpret_cast<uint32_t *>(d + o_idx), reinterpret_cast<float *>(d + o_dist),
                                   reinterpret_cast<float *>(d + o_sig), reinterpret_cast<float *>(d + o_rho), n, k,
                                   reinterpret_cast<uint32_t *>(d + o_rows), reinterpret_cast<uint32_t *>(d + o_cols),
                                   reinterpret_cast<float *>(d + o_vals), reinterpret_cast<uint64_t *>(d + o_nnz),
                                   d + o_ws, ws, nullptr);
        if (rc != HM_OK) break;
        rc = hm_fuzzy_graph_status(d + o_ws, n, k, nullptr);
        if (rc != HM_OK) break;
        err = cudaMemcpy(&nnz, d + o_nnz, 8, cudaMemcpyDeviceToHost);
        if (err == cudaSuccess) err = cudaMemcpy(rows_out, d + o_rows, nnz * 4, cudaMemcpyDeviceToHost);
        if (err == cudaSuccess) err = cudaMemcpy(cols_out, d + o_cols, nnz * 4, cudaMemcpyDeviceToHost);
        if (err == cudaSuccess) err = cudaMemcpy(vals_out, d + o_vals, nnz * 4, cudaMemcpyDeviceToHost);
        if (err != cudaSuccess) rc = set_error(HM_ERR_CUDA, "copy out: %s", cudaGetErrorString(err));
    } while (false);
    cudaFree(d);
    *nnz_out = nnz;
    return rc;
}

}  // extern "C"
