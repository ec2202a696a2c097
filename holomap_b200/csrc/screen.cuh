// screen.cuh -- the screened distance bulk: a tcgen05 tensor-core similarity
// screen with a proven error band, followed by an exact rerank of the
// survivors in the reference's binary64 order.
//
// Keep rule (per query row i, in screened units c^ = the screen's estimate of
// the row's distance-like value: 1 - cos for cosine, the squared distance of
// the centred, power-of-two scaled data for euclidean):
//
//   E_i  >= max_j |c^_ij - w_ij|,  w_ij = the reference's returned distance
//           mapped into the same units (cosine: itself; euclidean: squared),
//   tau_i = the k-th smallest c^_ij,
//   keep j  iff  c^_ij <= tau_i + 2 E_i.
//
// At least k points have c^ <= tau_i, so the reference's k-th value is at
// most tau_i + E_i, and every member j of the reference's top k has
// c^_ij <= w_ij + E_i <= tau_i + 2 E_i: it is kept.  The exact rerank of the
// kept set therefore returns the reference's list bit for bit.  E_i bounds
// (a) the operand rounding (error vectors of the bf16/tf32 operands, through
// Cauchy-Schwarz), (b) the tensor-core fp32 accumulation, taken as K * 2^-22
// of sum |a_k b_k| because its internal order is undocumented, (c) the
// screen epilogue's binary32 roundings and (d) the reference's own rounding
// (binary64 accumulation and the final binary32 cast).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

namespace hm {

// Counters the screened path leaves in the workspace (device-written).
struct ScreenCounters {
    unsigned long long candidates;  // candidates reranked exactly, all rows
    uint32_t max_row;               // most candidates reranked in one row
    uint32_t overflow_rows;         // rows sent to the exact fallback
    uint32_t band_max_bits;         // widest keep band 2E_i (binary32 bits)
    uint32_t error_code;            // nonzero if a bounded wait gave up
    uint32_t pad;
    unsigned long long emitted;     // candidates the screen wrote, all rows
};

// Screen GEMM tile: 128 query rows (UMMA M) x 256 columns (UMMA N), 128-byte
// K slices (64 bf16 or 32 tf32 elements) per pipeline stage.
constexpr int SC_BM = 128;
constexpr int SC_BN = 256;
constexpr int SC_SLICE_BYTES = 128;
constexpr int SC_STAGES = 4;
constexpr int SC_EPI_WARPS = 8;  // two per TMEM lane quadrant, one per half tile
constexpr int SC_THREADS = 64 + 32 * SC_EPI_WARPS;  // warp 0 TMA, warp 1 MMA, warps 2-9 epilogue

enum ScreenKind { SCREEN_KIND_BF16 = 0, SCREEN_KIND_TF32 = 1 };

struct ScreenLayout {
    int kind = SCREEN_KIND_BF16;
    bool split = false;       // operand is [hi|hi|lo] x [hi|lo|hi]
    uint32_t elem_bytes = 2;  // operand element size
    uint32_t kslice = 64;     // elements per 128-byte slice
    uint32_t kp1 = 0;         // one copy of d, padded to kslice
    uint32_t kp = 0;          // operand row length (kp1 or 3*kp1)
    uint32_t k_stages = 0;    // kp / kslice
    uint32_t row_blocks = 0, col_tiles = 0, parts = 1, part_tiles = 0, units = 0;
    uint32_t cap = 0;         // candidate slots per (row, part)
    uint32_t kpl = 1;         // rerank select width (WarpTopK slots per lane)
    uint32_t csum_blocks = 0; // euclidean column-mean partial blocks
    size_t off_a = 0, off_b = 0, off_csum = 0, off_mu = 0, off_max = 0, off_rowstat = 0;
    size_t off_rowterm = 0, off_colterm = 0, off_band = 0, off_force = 0;
    size_t off_cand = 0, off_cnt = 0, off_tau = 0, off_ovf = 0, off_ovf_cnt = 0, off_rowthr = 0;
    size_t total = 0;
};

struct ScreenRun {
    const float *data;
    const double *x64;
    const double *rnorm;
    uint32_t n, d, ldd, n_pad, k;
    int metric, path;
    uint32_t *idx_out;
    float *dist_out;
    ScreenCounters *counters;
    float *debug_dump;  // optional n x n screened values (tests only)
};

int screen_plan(uint64_t n, uint32_t d, uint32_t k, int metric, int path, ScreenLayout &L);
int screen_run(const ScreenRun &r, const ScreenLayout &L, char *ws, cudaStream_t s);

// ---- pieces (screen_prep.cu, screen_gemm.cu, rerank.cu) -------------------

// Per-row statistics of the operand rounding, binary64.
struct RowStat {
    double unorm;   // ||u_i||
    double enorm;   // ||e_i|| (single) or ||lo_i|| (split)
    double rnorm;   // split: ||u_i - hi_i - lo_i||; single: 0
    double anorm;   // ||A row|| (tensor-core operand)
    double bnorm;   // ||B row||
    double sqnorm;  // ||u_i||^2
};
constexpr int ROWSTAT_FIELDS = 6;

struct ScreenPrepArgs {
    const float *x;
    const double *rnorm_ref;  // cosine: sqrt of the sequential sum of squares
    uint32_t n, d, metric;
    ScreenLayout L;
    char *ws;
};
int launch_screen_prep(const ScreenPrepArgs &a, cudaStream_t s);
int launch_screen_band(uint32_t n, uint32_t d, int metric, const ScreenLayout &L, char *ws,
                       uint32_t *band_max_bits, cudaStream_t s);

struct ScreenGemmArgs {
    uint32_t n, k, k_stages, col_tiles, parts, part_tiles, units, cap;
    float scale;              // 1 (cosine) or 2 (euclidean)
    const float *rowterm;     // euclidean ||u_i||^2 (binary32); null for cosine
    const float *colterm;     // per column additive term
    const float *band;        // per row keep band 2E_i
    unsigned long long *cand; // [slot*cap] = (c^ bits << 32) | j, slot = (row*parts + part)*2 + half
    uint32_t *cand_cnt;       // [slot]
    float *part_topk;         // [slot * k]: each list's k smallest c^, ascending
    uint32_t *error_code;
    unsigned long long *emitted;
    const unsigned long long *zero_rows;  // cosine: rows with ||x|| = 0
    uint32_t *rowthr;         // per row: smallest list threshold so far (order-preserving key)
    float *dump;
    uint32_t idesc;
};
int launch_screen_gemm(const ScreenGemmArgs &g, int kind, uint32_t kpl_regs,
                       const CUtensorMap &ta, const CUtensorMap &tb, cudaStream_t s);

struct RerankArgs {
    const float *x;
    const double *rnorm;
    uint32_t n, d, k, parts, cap;
    const unsigned long long *cand;
    const uint32_t *cand_cnt;
    const float *part_topk;
    const float *band;
    const uint8_t *force_exact;
    uint32_t *ovf_list;
    uint32_t *ovf_cnt;
    uint32_t *idx_out;
    float *dist_out;
    ScreenCounters *counters;
};
int launch_rerank(const RerankArgs &a, int metric, uint32_t kpl, cudaStream_t s);

}  // namespace hm
