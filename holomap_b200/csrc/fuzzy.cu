// fuzzy.cu -- the fuzzy simplicial set on the device (src/fuzzy.rs:25-91):
// the symmetrized membership graph that consumes the kNN graph and its
// calibration, as COO sorted by (row, col).
//
// Directed strengths A[i][col] (self edges skipped; 1 when d - rho <= 0 or
// sigma == 0, else libm expf(-(d / sigma)); zeros dropped) are written twice:
// the forward entry (i, col) into the first half of one key array and the
// reverse entry (col, i) into the second half, keyed row << b | col with b
// the bit width of n - 1 (32-bit keys while 2b <= 32, that is n <= 65536,
// else 64-bit).  The weight's bits are the value, its sign bit (free: a
// weight is in (0, 1]) marking the reverse entry; absent entries carry the
// all-ones key, which no off-diagonal coordinate can equal.  One stable radix
// sort over the 2b key bits orders the entries by (row, col); a coordinate
// holds at most one forward and one reverse entry (each row's indices are
// distinct).  The first entry of every coordinate forms the binary32
// t-conorm (v + vt) - v * vt as the reference does (src/fuzzy.rs:67-75), and
// a scan compacts the nonzero results.  Every step is a function of the
// inputs alone: the output is the reference's, entry for entry.
#include <cub/cub.cuh>
#include <cuda_runtime.h>

#include "hm_internal.cuh"
#include "libm_expf.cuh"

namespace hm {

constexpr uint32_t FZ_REVERSE = 0x80000000u;

template <typename Key>
__global__ void fuzzy_directed_kernel(const uint32_t *__restrict__ idx, const float *__restrict__ dist,
                                      const float *__restrict__ sigma, const float *__restrict__ rho,
                                      uint64_t n, uint32_t k, uint32_t b, Key *__restrict__ keys,
                                      uint32_t *__restrict__ vals) {
    const uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t entries = n * k;
    if (e >= entries) return;
    const uint64_t i = e / k;
    const uint32_t col = idx[e];
    Key fk = ~Key(0), rk = ~Key(0);
    uint32_t vb = 0;
    if ((uint64_t)col != i) {
        const float d = __fsub_rn(dist[e], rho[i]);
        const float s = sigma[i];
        const float w = (d <= 0.0f || s == 0.0f) ? 1.0f : expf_libm(-__fdiv_rn(d, s));
        if (w != 0.0f) {
            fk = (Key(i) << b) | Key(col);
            rk = (Key(col) << b) | Key(i);
            vb = __float_as_uint(w);
        }
    }
    keys[e] = fk;
    keys[entries + e] = rk;
    vals[e] = vb;
    vals[entries + e] = vb | FZ_REVERSE;
}

// flag[p] = 1 for the first entry of each coordinate whose t-conorm is
// nonzero; its weight goes to w[p]
template <typename Key>
__global__ void fuzzy_fuse_kernel(const Key *__restrict__ keys, const uint32_t *__restrict__ vals, uint64_t total,
                                  uint32_t *__restrict__ flag, float *__restrict__ w) {
    const uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= total) return;
    const Key key = keys[p];
    uint32_t keep = 0;
    float out = 0.0f;
    if (key != ~Key(0) && (p == 0 || keys[p - 1] != key)) {
        float v = 0.0f, vt = 0.0f;
        const uint32_t a = vals[p];
        (a & FZ_REVERSE ? vt : v) = __uint_as_float(a & ~FZ_REVERSE);
        if (p + 1 < total && keys[p + 1] == key) {
            const uint32_t c = vals[p + 1];
            (c & FZ_REVERSE ? vt : v) = __uint_as_float(c & ~FZ_REVERSE);
        }
        out = __fsub_rn(__fadd_rn(v, vt), __fmul_rn(v, vt));
        keep = out != 0.0f ? 1u : 0u;
    }
    flag[p] = keep;
    w[p] = out;
}

template <typename Key>
__global__ void fuzzy_scatter_kernel(const Key *__restrict__ keys, const uint32_t *__restrict__ flag,
                                     const uint32_t *__restrict__ pos, const float *__restrict__ w, uint64_t total,
                                     uint32_t b, uint32_t *__restrict__ rows, uint32_t *__restrict__ cols,
                                     float *__restrict__ outv, unsigned long long *__restrict__ nnz) {
    const uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= total) return;
    if (flag[p]) {
        const Key key = keys[p];
        const uint32_t q = pos[p];
        rows[q] = (uint32_t)(key >> b);
        cols[q] = (uint32_t)(key & ((Key(1) << b) - 1));
        outv[q] = w[p];
    }
    if (p == total - 1) *nnz = (unsigned long long)pos[p] + flag[p];
}

// bit width of the largest index n - 1 (at least 1)
static uint32_t index_bits(uint64_t n) {
    uint32_t b = 1;
    while (b < 63 && (1ull << b) < n) ++b;
    return b;
}

// Workspace: keys and values (double-buffered for the sort), flags,
// positions, fused weights, and CUB's temporary storage.
struct FuzzyLayout {
    size_t keys0, keys1, vals0, vals1, flag, pos, w, temp, temp_bytes, total;
    uint32_t b;
    bool wide;  // 64-bit keys
};

template <typename Key>
static int fuzzy_temp_bytes(uint64_t total, size_t *bytes) {
    size_t sort_bytes = 0, scan_bytes = 0;
    cub::DoubleBuffer<Key> kb(nullptr, nullptr);
    cub::DoubleBuffer<uint32_t> vb(nullptr, nullptr);
    HM_CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, sort_bytes, kb, vb, (int)total));
    HM_CUDA_TRY(cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, (uint32_t *)nullptr, (uint32_t *)nullptr,
                                              (int)total));
    *bytes = std::max(sort_bytes, scan_bytes);
    return HM_OK;
}

static int fuzzy_layout(uint64_t n, uint32_t k, FuzzyLayout *L) {
    const uint64_t total = 2 * n * k;
    if (n > 0x7fffffffull || total >= 0x7fffffffull) return set_error(HM_ERR_UNSUPPORTED, "2 n k above 2^31 entries");
    L->b = index_bits(n);
    L->wide = 2 * L->b > 32;
    const size_t kbytes = L->wide ? 8 : 4;
    HM_TRY(L->wide ? fuzzy_temp_bytes<unsigned long long>(total, &L->temp_bytes)
                   : fuzzy_temp_bytes<uint32_t>(total, &L->temp_bytes));
    size_t off = 0;
    auto take = [&](size_t bytes) {
        const size_t at = off;
        off = round_up(off + std::max<size_t>(bytes, 1), 256);
        return at;
    };
    L->keys0 = take(total * kbytes);
    L->keys1 = take(total * kbytes);
    L->vals0 = take(total * 4);
    L->vals1 = take(total * 4);
    L->flag = take(total * 4);
    L->pos = take(total * 4);
    L->w = take(total * 4);
    L->temp = take(L->temp_bytes);
    L->total = off;
    return HM_OK;
}

template <typename Key>
static int fuzzy_run(const FuzzyLayout &L, const uint32_t *d_idx, const float *d_dist, const float *d_sigma,
                     const float *d_rho, uint64_t n, uint32_t k, uint32_t *d_rows, uint32_t *d_cols, float *d_vals,
                     unsigned long long *d_nnz, char *ws, cudaStream_t s) {
    auto *k0 = reinterpret_cast<Key *>(ws + L.keys0);
    auto *k1 = reinterpret_cast<Key *>(ws + L.keys1);
    auto *v0 = reinterpret_cast<uint32_t *>(ws + L.vals0);
    auto *v1 = reinterpret_cast<uint32_t *>(ws + L.vals1);
    auto *flag = reinterpret_cast<uint32_t *>(ws + L.flag);
    auto *pos = reinterpret_cast<uint32_t *>(ws + L.pos);
    auto *w = reinterpret_cast<float *>(ws + L.w);
    const uint64_t entries = n * k, total = 2 * entries;
    fuzzy_directed_kernel<Key><<<(unsigned)((entries + 255) / 256), 256, 0, s>>>(d_idx, d_dist, d_sigma, d_rho, n,
                                                                                 k, L.b, k0, v0);
    HM_CUDA_TRY(cudaGetLastError());
    count_launch();
    cub::DoubleBuffer<Key> kb(k0, k1);
    cub::DoubleBuffer<uint32_t> vb(v0, v1);
    size_t temp_bytes = L.temp_bytes;
    HM_CUDA_TRY(cub::DeviceRadixSort::SortPairs(ws + L.temp, temp_bytes, kb, vb, (int)total, 0, (int)(2 * L.b), s));
    count_launch();
    fuzzy_fuse_kernel<Key><<<(unsigned)((total + 255) / 256), 256, 0, s>>>(kb.Current(), vb.Current(), total, flag,
                                                                            w);
    HM_CUDA_TRY(cudaGetLastError());
    count_launch();
    temp_bytes = L.temp_bytes;
    HM_CUDA_TRY(cub::DeviceScan::ExclusiveSum(ws + L.temp, temp_bytes, flag, pos, (int)total, s));
    count_launch();
    fuzzy_scatter_kernel<Key><<<(unsigned)((total + 255) / 256), 256, 0, s>>>(kb.Current(), flag, pos, w, total, L.b,
                                                                               d_rows, d_cols, d_vals, d_nnz);
    HM_CUDA_TRY(cudaGetLastError());
    count_launch();
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
    auto *nnz = reinterpret_cast<unsigned long long *>(d_nnz);
    return L.wide ? fuzzy_run<unsigned long long>(L, d_idx, d_dist, d_sigma, d_rho, n, k, d_rows, d_cols, d_vals,
                                                  nnz, ws, s)
                  : fuzzy_run<uint32_t>(L, d_idx, d_dist, d_sigma, d_rho, n, k, d_rows, d_cols, d_vals, nnz, ws, s);
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
