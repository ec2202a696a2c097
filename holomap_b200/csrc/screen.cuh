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

#include "hm_internal.cuh"

namespace hm {

// Screen GEMM tile: 128 query rows (UMMA M) x 256 columns (UMMA N), 128-byte
// K slices (64 bf16 or 32 tf32 elements) per pipeline stage.
constexpr int SC_BM = 128;
constexpr int SC_BN = 256;
constexpr int SC_SLICE_BYTES = 128;
constexpr int SC_STAGES = 4;
// K slices of the A block kept resident in shared memory for a whole unit
// (96 KB: 6 slices of 128 B x 128 rows); deeper operands stream A with B
constexpr uint32_t SC_ARES_STAGES = 6;
// Epilogue warps per CTA: warp 0 issues the TMA loads, warp 1 the MMAs, the
// rest read the accumulator, (warp & 3) naming their TMEM lane quadrant (32
// query rows) and (warp - 2) / 4 their segment of the tile's 256 columns.
// Both emission passes take 16 (four segments of 64 columns: twice the
// warps to hide the latency of the per-row tests; each warp writes its own
// list, so a row has four lists per column part); the threshold pass (its
// sorted arrays need the registers) takes 8 (two segments of 128 columns).
// A 16-warp threshold pass for k <= 32 (96 registers, some spilled, four
// k-arrays per part) measured slower.
__host__ __device__ constexpr int sc_epi_warps(int pass, int kp = 32) {
    return (pass >= 1 && kp > 0) ? 16 : 8;
}
__host__ __device__ constexpr int sc_threads(int pass, int kp = 32) { return 64 + 32 * sc_epi_warps(pass, kp); }
constexpr int SC_FULL_LISTS = 4;  // candidate lists per row and column part of the emission passes
// column-side candidate stages per CTA of the symmetric emission pass (one
// per epilogue warp)
constexpr int SC_STAGE_SLOTS = 16;

enum ScreenKind { SCREEN_KIND_BF16 = 0, SCREEN_KIND_TF32 = 1 };

// Per-row statistics of the operand rounding, binary64.
struct RowStat {
    double unorm;   // ||u_i||
    double enorm;   // ||e_i|| (single) or ||lo_i|| (split)
    double rnorm;   // split: ||u_i - hi_i - lo_i||; single: 0
    double anorm;   // ||A row|| (tensor-core operand)
    double bnorm;   // ||B row||
    double sqnorm;  // ||u_i||^2
};

// One screen group: the screened jobs that share an operand format.  Their
// rows are concatenated into the group's row space (job g owns rows
// [row_starts[g], row_starts[g+1])), one operand matrix of rows x kpmax
// elements serves all of them through one TMA map, and the persistent
// screen kernel drains the group's (job, row block, column part) units.
struct GroupDev {
    uint32_t rows, njobs, units;
    uint32_t kind, split, elem_bytes, kslice, kpmax;
    const uint32_t *job_ids;      // [njobs] index of each group job in the job table
    const uint32_t *row_starts;   // [njobs + 1]
    const uint32_t *unit_starts;  // [njobs + 1]
    void *opa, *opb;              // rows x kpmax operands (opb == opa unless split)
    RowStat *rowstat;
    float *rowterm, *colterm, *band;  // colterm padded by SC_BN zeros
    uint8_t *force;               // rows the screen cannot bound (cosine zero vectors)
    uint32_t *rowthr;             // per row, ordered key: pass 0 the smallest list k-th so
                                  // far; pass 1 tau1, the k-th smallest mini-chunk minimum
    unsigned long long *cand;     // candidate lists, (c^ bits << 32) | job-local column
    uint32_t *cand_cnt;
    float *topk;                  // each list's k smallest mini-chunk minima, ascending
    uint32_t *row_cnt;            // rerank: survivors per group row (0: none or exact fallback)
    // emission pass: its work units (x = group job slot | sym << 31, y = row
    // block, z = first column tile, w = end column tile | column part << 24),
    // largest first
    const uint4 *eunits;
    uint32_t neunits;
    // emission pass in the 2-SM form (a cluster of two CTAs per unit, one
    // MMA of 256 rows; eunits' y is then a block of 256 rows)
    uint32_t pair;
    // the group has jobs whose padded row length K1 is at most / above the
    // packed operand kernel's limit (which operand kernels run)
    uint32_t any_short_rows, any_long_rows;
    // symmetric emission: per group row (padded like colterm) the emission
    // limit tau1 + 2 band and its cosine raw-product form; the column-side
    // candidates each CTA staged (group row of the column, raw product bits
    // << 32 | job-local row) and their counts
    float *ethr, *evstar;
    uint32_t *stage_row, *stage_cnt;
    unsigned long long *stage_key;
    uint32_t stage_cap;
};

// binary32 <-> unsigned key with the same order (for atomicMin)
__device__ __forceinline__ uint32_t ord32(float f) {
    const uint32_t b = __float_as_uint(f);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float unord32(uint32_t o) {
    return __uint_as_float((o & 0x80000000u) ? (o & 0x7fffffffu) : ~o);
}

// Row i's threshold-pass list s (s < tlists * parts) of job J (its k-array).
__device__ __forceinline__ size_t list_index(const JobDev &J, uint32_t i, uint32_t s) {
    return (size_t)J.slot0 + (size_t)i * J.tlists * J.parts + s;
}

// Row i's candidate list s (s < elists) of job J: its count is
// G.cand_cnt[cand_list(J, i, s)], its slots follow cand_slots.
__device__ __forceinline__ size_t cand_list(const JobDev &J, uint32_t i, uint32_t s) {
    return (size_t)J.eslot0 + (size_t)i * J.elists + s;
}
__device__ __forceinline__ unsigned long long *cand_slots(const JobDev &J, const GroupDev &G, size_t list) {
    return G.cand + J.cand0 + (list - J.eslot0) * J.cap;
}

int launch_screen_prep(const JobDev *jobs, const GroupDev &G, const GroupDev *Gd, cudaStream_t s);
int launch_screen_band(const JobDev *jobs, const GroupDev &G, const GroupDev *Gd, cudaStream_t s);
int launch_screen_gemm(const JobDev *jobs, const GroupDev &G, const GroupDev *Gd, uint32_t kp,
                       const CUtensorMap &ta, const CUtensorMap &tb, float *dump, int pass,
                       cudaStream_t s);
int launch_screen_threshold(const JobDev *jobs, const GroupDev &G, const GroupDev *Gd, uint32_t kpl,
                            cudaStream_t s);
int launch_rerank(const JobDev *jobs, const GroupDev &G, const GroupDev *Gd, uint32_t kpl,
                  uint32_t dmax, int metric_mask, cudaStream_t s);
// symmetric emission: the per-row limits before the emission pass, and the
// column-side candidates moved from the CTAs' staging into the rows' column
// lists after it (grid: the emission pass's CTAs)
int launch_emit_limits(const JobDev *jobs, const GroupDev &G, const GroupDev *Gd, cudaStream_t s);
// After the threshold pass of a group holding jobs with an escalation copy:
// sets each such job's escalate flag (JobCounters::escalate).
int launch_escalation(const JobDev *jobs, const GroupDev &G, const GroupDev *Gd, cudaStream_t s);
int launch_column_scatter(const JobDev *jobs, const GroupDev &G, const GroupDev *Gd, uint32_t ctas,
                          cudaStream_t s);
// the emission pass's grid (one CTA per SM, at most one per unit)
uint32_t emission_grid(const GroupDev &G);

}  // namespace hm
