// screen.cu -- plan and launch sequence of the screened path, and the
// autotuner table that picks a path per (n, d, k, metric).
//
//   screen prep   operands + binary64 error statistics (screen_prep.cu)
//   band          keep band 2E_i per row
//   screen gemm   tcgen05 U U^T + running top-k + candidate emission
//   rerank        exact distances of the survivors + select (rerank.cu)
//   fallback      plain exact kernel over the rows the screen could not bound
#include <cuda.h>
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>

#include "hm_internal.cuh"
#include "screen.cuh"

namespace hm {

static thread_local float *g_debug_dump = nullptr;

static size_t a256(size_t x) { return round_up(x, 256); }

static uint32_t pow2ceil(uint32_t v) {
    uint32_t p = 1;
    while (p < v) p <<= 1;
    return p;
}

static int sm_count() {
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) == cudaSuccess &&
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess && sms > 0)
        return sms;
    cudaGetLastError();  // no device here: plan for a B200
    return 148;
}

int screen_plan(uint64_t n, uint32_t d, uint32_t k, int metric, int path, ScreenLayout &L) {
    if (metric != HM_METRIC_EUCLIDEAN && metric != HM_METRIC_COSINE)
        return set_error(HM_ERR_UNSUPPORTED, "metric %d has no inner-product screen", metric);
    if (k > 64) return set_error(HM_ERR_UNSUPPORTED, "the screened path handles k <= 64 (k=%u)", k);
    if (d > 2048) return set_error(HM_ERR_UNSUPPORTED, "the screened path handles d <= 2048 (d=%u)", d);
    L = ScreenLayout{};
    switch (path) {
    case HM_PATH_SCREEN_BF16: L.kind = SCREEN_KIND_BF16; L.elem_bytes = 2; break;
    case HM_PATH_SCREEN_TF32: L.kind = SCREEN_KIND_TF32; L.elem_bytes = 4; break;
    case HM_PATH_SCREEN_BF16X3: L.kind = SCREEN_KIND_BF16; L.elem_bytes = 2; L.split = true; break;
    default: return set_error(HM_ERR_INVALID, "path %d is not a screened path", path);
    }
    L.kslice = SC_SLICE_BYTES / L.elem_bytes;
    L.kp1 = (uint32_t)round_up(d, L.kslice);
    L.kp = L.split ? 3 * L.kp1 : L.kp1;
    L.k_stages = L.kp / L.kslice;
    L.row_blocks = (uint32_t)((n + SC_BM - 1) / SC_BM);
    L.col_tiles = (uint32_t)((n + SC_BN - 1) / SC_BN);

    // column parts: balance the persistent grid (makespan in tiles) against
    // the extra emissions each part costs
    const uint32_t G = (uint32_t)sm_count();
    double best = 1e300;
    for (uint32_t S = 1; S <= 8 && S <= L.col_tiles; ++S) {
        const uint32_t pt = (L.col_tiles + S - 1) / S;
        const uint32_t parts = (L.col_tiles + pt - 1) / pt;
        const uint64_t units = (uint64_t)L.row_blocks * parts;
        const double makespan = (double)((units + G - 1) / G) * pt;
        const double cost = makespan * (1.0 + 0.03 * parts);
        if (cost < best - 1e-9) {
            best = cost;
            L.part_tiles = pt;
            L.parts = parts;
        }
    }
    L.units = L.row_blocks * L.parts;
    // each (row, part) has two candidate lists, one per epilogue half tile
    const double per_slot = (double)n / (2.0 * L.parts);
    const double expect = 1.5 * k * (2.0 + std::log(std::fmax(1.0, per_slot / k)));
    L.cap = pow2ceil((uint32_t)expect);
    if (L.cap < 128) L.cap = 128;
    if (L.cap > 4096) L.cap = 4096;
    L.kpl = k <= 32 ? 1 : 2;
    L.csum_blocks = (uint32_t)std::fmin(256.0, std::ceil((double)n / 64.0));

    size_t off = 0;
    L.off_a = off;
    off = a256(off + (size_t)n * L.kp * L.elem_bytes);
    L.off_b = L.off_a;
    if (L.split) {
        L.off_b = off;
        off = a256(off + (size_t)n * L.kp * L.elem_bytes);
    }
    L.off_csum = off;
    off = a256(off + (size_t)L.csum_blocks * d * sizeof(double));
    L.off_mu = off;
    off = a256(off + (size_t)d * sizeof(double));
    L.off_max = off;
    off = a256(off + 8 * sizeof(unsigned long long));
    L.off_rowstat = off;
    off = a256(off + (size_t)n * sizeof(RowStat));
    L.off_rowterm = off;
    off = a256(off + (size_t)n * sizeof(float));
    L.off_colterm = off;  // padded to whole tiles, zero past n
    off = a256(off + round_up(n, SC_BN) * sizeof(float));
    L.off_band = off;
    off = a256(off + (size_t)n * sizeof(float));
    L.off_force = off;
    off = a256(off + (size_t)n);
    L.off_cand = off;
    off = a256(off + (size_t)n * L.parts * 2 * L.cap * sizeof(unsigned long long));
    L.off_cnt = off;
    off = a256(off + (size_t)n * L.parts * 2 * sizeof(uint32_t));
    L.off_tau = off;
    off = a256(off + (size_t)n * L.parts * 2 * k * sizeof(float));
    L.off_ovf = off;
    off = a256(off + (size_t)n * sizeof(uint32_t));
    L.off_ovf_cnt = off;
    off = a256(off + sizeof(uint32_t));
    L.off_rowthr = off;
    off = a256(off + (size_t)n * sizeof(uint32_t));
    L.total = off;
    return HM_OK;
}

// ------------------------------------------------------------ tensor maps
typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *,
                                  const cuuint64_t *, const cuuint64_t *, const cuuint32_t *,
                                  const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static int encode_fn(EncodeTiledFn *out) {
    static std::once_flag once;
    static EncodeTiledFn fn = nullptr;
    static cudaError_t err = cudaSuccess;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        err = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q);
        if (err == cudaSuccess && q == cudaDriverEntryPointSuccess) fn = reinterpret_cast<EncodeTiledFn>(p);
    });
    if (!fn) return set_error(HM_ERR_CUDA, "cuTensorMapEncodeTiled unavailable (%s)", cudaGetErrorString(err));
    *out = fn;
    return HM_OK;
}

// 2-D map over an n x kp operand, box = one 128-byte K slice x `box_rows`
// rows, 128-byte swizzle; rows past n read as zeros.
static int make_map(CUtensorMap *m, void *base, uint64_t n, const ScreenLayout &L, uint32_t box_rows) {
    EncodeTiledFn enc;
    HM_TRY(encode_fn(&enc));
    const cuuint64_t dims[2] = {L.kp, n};
    const cuuint64_t strides[1] = {(cuuint64_t)L.kp * L.elem_bytes};
    const cuuint32_t box[2] = {L.kslice, box_rows};
    const cuuint32_t estr[2] = {1, 1};
    const CUresult r = enc(m, L.elem_bytes == 2 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32,
                           2, base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                           CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                           CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return set_error(HM_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    return HM_OK;
}

static uint32_t make_idesc(int kind) {
    const uint32_t fmt = kind == SCREEN_KIND_BF16 ? 1u : 2u;  // BF16 / TF32 operands
    return (1u << 4)                    // accumulator: F32
           | (fmt << 7) | (fmt << 10)   // A, B formats
           | (0u << 15) | (0u << 16)    // A, B K-major
           | ((uint32_t)(SC_BN >> 3) << 17) | ((uint32_t)(SC_BM >> 4) << 24);
}

int screen_run(const ScreenRun &r, const ScreenLayout &L, char *ws, cudaStream_t s) {
    ScreenPrepArgs pa{};
    pa.x = r.data;
    pa.rnorm_ref = r.rnorm;
    pa.n = r.n;
    pa.d = r.d;
    pa.metric = (uint32_t)r.metric;
    pa.L = L;
    pa.ws = ws;
    HM_TRY(launch_screen_prep(pa, s));
    HM_TRY(launch_screen_band(r.n, r.d, r.metric, L, ws, &r.counters->band_max_bits, s));

    CUtensorMap ta, tb;
    HM_TRY(make_map(&ta, ws + L.off_a, r.n, L, SC_BM));
    HM_TRY(make_map(&tb, ws + L.off_b, r.n, L, SC_BN));

    ScreenGemmArgs g{};
    g.n = r.n;
    g.k = r.k;
    g.k_stages = L.k_stages;
    g.col_tiles = L.col_tiles;
    g.parts = L.parts;
    g.part_tiles = L.part_tiles;
    g.units = L.units;
    g.cap = L.cap;
    g.scale = r.metric == HM_METRIC_EUCLIDEAN ? 2.0f : 1.0f;
    g.rowterm = r.metric == HM_METRIC_EUCLIDEAN ? reinterpret_cast<float *>(ws + L.off_rowterm) : nullptr;
    g.colterm = reinterpret_cast<float *>(ws + L.off_colterm);
    g.band = reinterpret_cast<float *>(ws + L.off_band);
    g.cand = reinterpret_cast<unsigned long long *>(ws + L.off_cand);
    g.cand_cnt = reinterpret_cast<uint32_t *>(ws + L.off_cnt);
    g.part_topk = reinterpret_cast<float *>(ws + L.off_tau);
    g.error_code = &r.counters->error_code;
    g.emitted = &r.counters->emitted;
    g.zero_rows = reinterpret_cast<unsigned long long *>(ws + L.off_max) + 7;
    g.rowthr = reinterpret_cast<uint32_t *>(ws + L.off_rowthr);
    g.dump = r.debug_dump ? r.debug_dump : g_debug_dump;
    g.idesc = make_idesc(L.kind);
    HM_TRY(launch_screen_gemm(g, L.kind, r.k <= 32 ? 32u : 64u, ta, tb, s));

    uint32_t *ovf_cnt = reinterpret_cast<uint32_t *>(ws + L.off_ovf_cnt);
    HM_CUDA_TRY(cudaMemsetAsync(ovf_cnt, 0, sizeof(uint32_t), s));
    RerankArgs ra{};
    ra.x = r.data;
    ra.rnorm = r.rnorm;
    ra.n = r.n;
    ra.d = r.d;
    ra.k = r.k;
    ra.parts = L.parts * 2;  // candidate lists per row
    ra.cap = L.cap;
    ra.cand = g.cand;
    ra.cand_cnt = g.cand_cnt;
    ra.part_topk = g.part_topk;
    ra.band = g.band;
    ra.force_exact = reinterpret_cast<uint8_t *>(ws + L.off_force);
    ra.ovf_list = reinterpret_cast<uint32_t *>(ws + L.off_ovf);
    ra.ovf_cnt = ovf_cnt;
    ra.idx_out = r.idx_out;
    ra.dist_out = r.dist_out;
    ra.counters = r.counters;
    HM_TRY(launch_rerank(ra, r.metric, L.kpl, s));

    // exact plain path for the rows the screen could not settle (its binary64
    // copy of the points is built only when such rows exist)
    HM_TRY(launch_prep_x64(r.data, r.n, r.d, r.ldd, r.n_pad, const_cast<double *>(r.x64), ovf_cnt, s));
    PlainArgs pl{};
    pl.x64 = r.x64;
    pl.rnorm = r.rnorm;
    pl.n = r.n;
    pl.ldd = r.ldd;
    pl.k = r.k;
    pl.idx_out = r.idx_out;
    pl.dist_out = r.dist_out;
    pl.row_list = ra.ovf_list;
    pl.row_count = ovf_cnt;
    HM_TRY(launch_plain_knn_rows(pl, r.metric, s));
    return HM_OK;
}

}  // namespace hm

using namespace hm;

extern "C" {

// Autotuner table: the path HM_PATH_AUTO takes.  Screened paths need an inner
// product form (euclidean, cosine), k <= 64 and d <= 2048; below a few
// thousand points the plain path's single pass is as fast as screen + rerank.
int hm_autotune_path(uint64_t n, uint32_t d, uint32_t k, int metric) {
    if (metric == HM_METRIC_MANHATTAN || k > 64 || d > 2048 || n < 4096) return HM_PATH_PLAIN;
    if (metric == HM_METRIC_COSINE) return HM_PATH_SCREEN_BF16;
    return HM_PATH_SCREEN_TF32;
}

int hm_debug_set_screen_dump(float *d_out) {
    g_debug_dump = d_out;
    return HM_OK;
}

}  // extern "C"
