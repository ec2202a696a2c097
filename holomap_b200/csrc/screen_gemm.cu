// screen_gemm.cu -- the tensor-core screen: U U^T on tcgen05 with TMEM
// accumulators, fused with the per-row thresholds and the candidate emission,
// so the N x N similarity matrix never leaves the SM.
//
// One CTA per SM (persistent), 10 warps (18 in the emission passes):
//   warp 0     TMA producer: the unit's 128-row A block stays resident in
//              shared memory when its K slices fit 96 KB (else it streams
//              with B), 256-row B slices per stage (128-byte K slices, 128B
//              swizzle, 4-stage mbarrier ring; every CTA loads its own tiles),
//   warp 1     allocates 512 TMEM columns (two 128 x 256 fp32 accumulators)
//              and issues tcgen05.mma (one thread) + tcgen05.commit,
//   warps 2-   epilogue: each thread owns one query row (its TMEM lane) and
//              one segment of every tile's 256 columns (half, read 32 columns
//              at a time, in the threshold pass; a quarter, read 16 columns
//              at a time, in the emission passes).
// The emission passes can also run in the 2-SM form: a cluster of two
// CTAs shares each 256 x 256 tile (one tcgen05.mma.cta_group::2 of M = 256
// issued by the leader CTA), each CTA holding its own 128 rows of A and
// loading half of the column tile into an 8-stage ring.
// Two launches per group (template PASS):
//   0  threshold pass over a sample of each part's columns: per list, the k
//      smallest minima of column chunks, sorted in registers and shared
//      between the row's lists (atomicMin); threshold_kernel then takes the
//      k-th of the union, tau1, an upper bound of the row's k-th screened value;
//   1  emission pass over all columns with the fixed limit tau1 + band: 8-column
//      group minima gate the per-column test, which writes every column within
//      the limit into the row's list;
//   2  the emission pass of a group whose whole datasets take the symmetric
//      form: a row block walks only the tiles from its diagonal on, with the
//      limit tau1 + 2 band, and each value above the diagonal is also tested
//      for its column's row (one ballot per column; staged per epilogue
//      warp, moved to that row's column list by column_scatter_kernel).
// Work units are (row block of 128, column part); the columns of a unit are
// walked in 256-wide tiles with the two accumulators double buffered, so the
// epilogue of one tile overlaps the MMAs of the next.
//
// Every wait on an mbarrier is bounded (wall clock via %globaltimer and an
// iteration cap): on expiry the CTA records an error code, stops issuing,
// waits (bounded) for its own copies and MMAs, frees TMEM and returns.
#include <mutex>
#include <vector>

#include <cuda.h>
#include <cuda_runtime.h>

#include "hm_internal.cuh"
#include "mbarrier.cuh"
#include "screen.cuh"

namespace hm {

constexpr uint32_t SC_A_BYTES = SC_BM * SC_SLICE_BYTES;  // 16 KB
constexpr uint32_t SC_B_BYTES = SC_BN * SC_SLICE_BYTES;  // 32 KB
constexpr uint32_t SC_OPND_BYTES = SC_ARES_STAGES * SC_A_BYTES + SC_STAGES * SC_B_BYTES;  // 224 KB
constexpr uint32_t SC_SMEM_BYTES = 1024 + SC_OPND_BYTES + 256;
constexpr uint32_t SC_TMEM_COLS = 512;
// 2-SM form: each CTA holds half of the 256-row B tile, 16 KB per K slice,
// in 8 stages (the same 128 KB as 4 stages of whole tiles)
constexpr uint32_t SC_B2_BYTES = (SC_BN / 2) * SC_SLICE_BYTES;
constexpr uint32_t SC_STAGES2 = 8;
constexpr uint32_t SC_MAXST = SC_STAGES2;
enum : uint32_t {
    SC_ERR_PRODUCER = 1,
    SC_ERR_MMA_FULL = 2,
    SC_ERR_MMA_ACC = 3,
    SC_ERR_EPILOGUE = 4,
    SC_ERR_DRAIN = 5,
};

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap *map, uint32_t bar,
                                            int32_t x, int32_t y) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3}], [%4];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
        : "memory");
}

// The 2-SM form (a cluster of two CTAs sharing each MMA): both CTAs' loads
// complete on the leader's (rank 0's) barrier, whose cluster address is the
// local one with the rank bit (bit 24) cleared.
// 2-SM copy: the bytes land in this CTA's shared memory and complete on the
// barrier at `leader_bar` (a shared::cluster address in the pair's leader)
__device__ __forceinline__ void tma_load_2d_pair(uint32_t dst, const CUtensorMap *map, uint32_t leader_bar,
                                                 int32_t x, int32_t y) {
    asm volatile(
        "cp.async.bulk.tensor.2d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3}], [%4];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(leader_bar)
        : "memory");
}

// arrive on a barrier given by its shared::cluster address
__device__ __forceinline__ void mbar_arrive_cluster(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cluster.b64 _, [%0];" ::"r"(bar) : "memory");
}

// the shared::cluster address of a shared-memory word of this CTA in CTA `rank`
__device__ __forceinline__ uint32_t cluster_addr(uint32_t local, uint32_t rank) {
    uint32_t r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(local), "r"(rank));
    return r;
}

__device__ __forceinline__ void cluster_sync() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}

__device__ __forceinline__ uint32_t cluster_rank() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}


__device__ __forceinline__ void fence_before_sync() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_after_sync() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// Shared-memory matrix descriptor: K-major operand, 128-byte swizzle, rows
// of 128 bytes stored back to back (8-row groups 1024 bytes apart).
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr) {
    return (uint64_t)((addr >> 4) & 0x3fffu)  // start address
           | ((uint64_t)1 << 16)              // leading byte offset (unused for SW128 K-major)
           | ((uint64_t)(1024 >> 4) << 32)    // stride byte offset: 8 rows x 128 B
           | ((uint64_t)1 << 46)              // descriptor version (sm_100)
           | ((uint64_t)2 << 61);             // swizzle mode: 128B
}

template <int KIND, bool PAIR = false>
__device__ __forceinline__ void mma_issue(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc,
                                          uint32_t idesc, uint32_t accum) {
    if (PAIR) {
        if (KIND == SCREEN_KIND_BF16)
            asm volatile(
                "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                "tcgen05.mma.cta_group::2.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
                "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accum)
                : "memory");
        else
            asm volatile(
                "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                "tcgen05.mma.cta_group::2.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
                "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accum)
                : "memory");
        return;
    }
    if (KIND == SCREEN_KIND_BF16) {
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
            "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accum)
            : "memory");
    } else {
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
            "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accum)
            : "memory");
    }
}

template <bool PAIR = false>
__device__ __forceinline__ void mma_commit(uint32_t bar) {
    if (PAIR)  // the barrier at this offset in both CTAs of the pair
        asm volatile(
            "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64 [%0], %1;" ::
                "r"(bar), "h"((uint16_t)3)
            : "memory");
    else
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                     : "memory");
}

// tcgen05.ld of 32 consecutive accumulator columns of this warp's 32 lanes;
// the registers are valid only after tmem_ld_wait on the same array (the
// wait names them as in/out operands so no use can be scheduled before it).
__device__ __forceinline__ void tmem_ld32_issue(uint32_t taddr, uint32_t (&v)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32"
        " {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15,"
        " %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31},"
        " [%32];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
          "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]),
          "=r"(v[14]), "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]),
          "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]), "=r"(v[25]),
          "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
        : "r"(taddr));
}

__device__ __forceinline__ void tmem_ld16_issue(uint32_t taddr, uint32_t (&v)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32"
        " {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
          "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]),
          "=r"(v[14]), "=r"(v[15])
        : "r"(taddr));
}
__device__ __forceinline__ void tmem_ld_wait16(uint32_t (&v)[16]) {
    asm volatile("tcgen05.wait::ld.sync.aligned;"
                 : "+r"(v[0]), "+r"(v[1]), "+r"(v[2]), "+r"(v[3]), "+r"(v[4]), "+r"(v[5]),
                   "+r"(v[6]), "+r"(v[7]), "+r"(v[8]), "+r"(v[9]), "+r"(v[10]), "+r"(v[11]),
                   "+r"(v[12]), "+r"(v[13]), "+r"(v[14]), "+r"(v[15])
                 :
                 : "memory");
}
__device__ __forceinline__ void tmem_ld_wait(uint32_t (&v)[32]) {
    asm volatile("tcgen05.wait::ld.sync.aligned;"
                 : "+r"(v[0]), "+r"(v[1]), "+r"(v[2]), "+r"(v[3]), "+r"(v[4]), "+r"(v[5]),
                   "+r"(v[6]), "+r"(v[7]), "+r"(v[8]), "+r"(v[9]), "+r"(v[10]), "+r"(v[11]),
                   "+r"(v[12]), "+r"(v[13]), "+r"(v[14]), "+r"(v[15]), "+r"(v[16]), "+r"(v[17]),
                   "+r"(v[18]), "+r"(v[19]), "+r"(v[20]), "+r"(v[21]), "+r"(v[22]), "+r"(v[23]),
                   "+r"(v[24]), "+r"(v[25]), "+r"(v[26]), "+r"(v[27]), "+r"(v[28]), "+r"(v[29]),
                   "+r"(v[30]), "+r"(v[31])
                 :
                 : "memory");
}


__device__ __forceinline__ void raise_error(volatile uint32_t *abort_flag, uint32_t *error_code,
                                            uint32_t code, uint32_t peer_abort = 0) {
    *abort_flag = 1;
    if (peer_abort)  // the other CTA of a pair stops waiting too
        asm volatile("st.shared::cluster.u32 [%0], %1;" ::"r"(peer_abort), "r"(1u) : "memory");
    atomicCAS(error_code, 0u, code);
}

struct UnitTiles {
    uint32_t job, rb, part, ct_begin, ct_end, sym;
};

// Pass 0 (the threshold pass) walks only the first seed_tiles tiles of each
// part: a sample of the row's columns whose k-th smallest screened value
// already bounds the row's k-th from above.  Pass 1 (the emission pass) takes
// its units from the group's table.
__device__ __forceinline__ UnitTiles unit_tiles(const JobDev *jobs, const GroupDev &G, uint32_t u, int pass) {
    UnitTiles t;
    if (pass >= 1) {
        const uint4 e = G.eunits[u];
        t.job = G.job_ids[e.x & 0x7fffffffu];
        t.sym = e.x >> 31;
        t.rb = e.y;
        t.ct_begin = e.z;
        t.ct_end = e.w & 0xffffffu;
        t.part = e.w >> 24;
        return t;
    }
    const uint32_t g = find_job(G.unit_starts, G.njobs, u);
    t.sym = 0;
    t.job = G.job_ids[g];
    const JobDev &J = jobs[t.job];
    const uint32_t lu = u - G.unit_starts[g];
    t.rb = J.rb0 + lu / J.parts;
    t.part = lu % J.parts;
    t.ct_begin = t.part * J.part_tiles;
    t.ct_end = min(J.col_tiles, t.ct_begin + (pass == 0 ? J.seed_tiles : J.part_tiles));
    return t;
}

template <int KIND, int KP, int PASS, bool PAIR>
__global__ void __launch_bounds__(sc_threads(PASS, KP), 1)
    screen_gemm_kernel(const __grid_constant__ CUtensorMap tma, const __grid_constant__ CUtensorMap tmb,
                       const JobDev *__restrict__ jobs, const GroupDev G, float *dump, uint32_t idesc,
                       uint32_t a_res) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t *smem = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) &
                                                ~(uintptr_t)1023);
    // streaming: stage s holds A at sA + s * 16 KB and B at sB + s * 32 KB;
    // resident A: the unit's A slices at smem + ks * 16 KB, B stages after them
    // 2-SM form (a_res always): the A block resident, B half-tile stages
    uint8_t *sA = smem;
    uint8_t *sB = (PAIR || a_res) ? smem + SC_ARES_STAGES * SC_A_BYTES : smem + SC_STAGES * SC_A_BYTES;
    constexpr uint32_t NST = PAIR ? SC_STAGES2 : SC_STAGES;  // B stages
    constexpr uint32_t BST = PAIR ? SC_B2_BYTES : SC_B_BYTES;  // bytes of one B stage
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem + SC_OPND_BYTES);
    uint64_t *full = bars;                  // [NST]
    uint64_t *empty = bars + SC_MAXST;      // [NST]
    uint64_t *accf = bars + 2 * SC_MAXST;   // [2]
    uint64_t *acce = accf + 2;              // [2]
    uint64_t *afull = acce + 2;             // resident A loaded
    uint64_t *aempty = afull + 1;           // resident A consumed by the unit's MMAs
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(aempty + 1);
    volatile uint32_t *abort_flag = tmem_slot + 1;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t nunits = PASS >= 1 ? G.neunits : G.units;
    // 2-SM form: a cluster of two CTAs works on a unit of 256 rows (rank r
    // owns the 128-row block 2 rb + r); rank 0 (the leader) issues the MMAs
    const uint32_t rank = PAIR ? cluster_rank() : 0u;
    const bool leader = rank == 0;
    const uint32_t wid = PAIR ? blockIdx.x >> 1 : blockIdx.x;
    const uint32_t nworkers = PAIR ? gridDim.x >> 1 : gridDim.x;
    // PASS 2 is the emission pass of a group with symmetric units (the
    // column-side tests exist only in that instantiation)
    constexpr bool SYMK = PASS == 2;
    constexpr uint32_t EW = sc_epi_warps(PASS, KP);  // epilogue warps
    static_assert(!SYMK || EW == SC_STAGE_SLOTS, "one column-side stage per epilogue warp");
    constexpr uint32_t NSEG = EW / 4;             // column segments per tile (= lists per part)
    constexpr uint32_t SEGW = SC_BN / NSEG;       // columns per segment

    if (threadIdx.x == 0) {
        for (uint32_t s = 0; s < NST; ++s) {
            mbar_init(smem_u32(&full[s]), 1);
            mbar_init(smem_u32(&empty[s]), 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(smem_u32(&accf[b]), 1);
            // the leader's accumulator is released by both CTAs' epilogues
            mbar_init(smem_u32(&acce[b]), PAIR ? 2 * EW : EW);
        }
        mbar_init(smem_u32(afull), 1);
        mbar_init(smem_u32(aempty), 1);
        *abort_flag = 0;
        mbar_init_fence();
    }
    if (warp == 1) {
        if (PAIR) {
            asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                             smem_u32(tmem_slot)),
                         "r"(SC_TMEM_COLS));
            asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;");
        } else {
            asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                             smem_u32(tmem_slot)),
                         "r"(SC_TMEM_COLS));
            asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
        }
    }
    fence_before_sync();
    __syncthreads();
    if (PAIR) cluster_sync();  // both CTAs' barriers exist before either signals the other's
    fence_after_sync();
    const uint32_t tmem_base = *tmem_slot;
    const uint32_t peer_abort = PAIR ? cluster_addr(smem_u32((const void *)abort_flag), rank ^ 1u) : 0u;

    if (warp == 0) {
        // ------------------------------------------------------ TMA producer
        if (lane == 0) {
            uint32_t it = 0, un = 0;
            bool ok = true;
            constexpr uint32_t kelems = SC_SLICE_BYTES / (KIND == SCREEN_KIND_BF16 ? 2 : 4);
            for (uint32_t u = wid; ok && u < nunits; u += nworkers) {
                const UnitTiles ut = unit_tiles(jobs, G, u, PASS);
                const JobDev &J = jobs[ut.job];
                if (!job_active(J)) continue;  // every role skips the same units
                const uint32_t myrb = PAIR ? 2 * ut.rb + rank : ut.rb;  // this CTA's 128-row block
                if (PAIR || a_res) {
                    // the previous unit's MMAs must be done with the A block
                    if (un > 0 && !mbar_wait(smem_u32(aempty), (un - 1) & 1, abort_flag)) {
                        raise_error(abort_flag, &J.out->error_code, SC_ERR_PRODUCER, peer_abort);
                        ok = false;
                        break;
                    }
                    const uint32_t fb = smem_u32(afull);
                    if (!PAIR || leader) mbar_arrive_expect_tx(fb, (PAIR ? 2u : 1u) * J.k_stages * SC_A_BYTES);
                    for (uint32_t ks = 0; ks < J.k_stages; ++ks) {
                        if (PAIR)
                            tma_load_2d_pair(smem_u32(sA + ks * SC_A_BYTES), &tma, cluster_addr(fb, 0), (int32_t)(ks * kelems),
                                             (int32_t)(J.row0 + myrb * SC_BM));
                        else
                            tma_load_2d(smem_u32(sA + ks * SC_A_BYTES), &tma, fb, (int32_t)(ks * kelems),
                                        (int32_t)(J.row0 + myrb * SC_BM));
                    }
                    ++un;
                }
                for (uint32_t ct = ut.ct_begin; ok && ct < ut.ct_end; ++ct) {
                    for (uint32_t ks = 0; ks < J.k_stages; ++ks, ++it) {
                        const uint32_t s = it % NST, r = it / NST;
                        if (!mbar_wait(smem_u32(&empty[s]), (r & 1) ^ 1, abort_flag)) {
                            raise_error(abort_flag, &J.out->error_code, SC_ERR_PRODUCER, peer_abort);
                            ok = false;
                            break;
                        }
                        const uint32_t fb = smem_u32(&full[s]);
                        const int32_t kx = (int32_t)(ks * kelems);
                        if (PAIR) {
                            // both halves of the B tile complete on the leader's barrier
                            if (leader) mbar_arrive_expect_tx(fb, 2 * SC_B2_BYTES);
                            tma_load_2d_pair(smem_u32(sB + s * BST), &tmb, cluster_addr(fb, 0), kx,
                                             (int32_t)(J.row0 + ct * SC_BN + rank * (SC_BN / 2)));
                        } else {
                            if (a_res) {
                                mbar_arrive_expect_tx(fb, SC_B_BYTES);
                            } else {
                                mbar_arrive_expect_tx(fb, SC_A_BYTES + SC_B_BYTES);
                                tma_load_2d(smem_u32(sA + s * SC_A_BYTES), &tma, fb, kx, (int32_t)(J.row0 + myrb * SC_BM));
                            }
                            tma_load_2d(smem_u32(sB + s * SC_B_BYTES), &tmb, fb, kx, (int32_t)(J.row0 + ct * SC_BN));
                        }
                    }
                }
            }
            if (PAIR) {
                // drain: the leader's MMAs have consumed (so both CTAs' copies
                // have landed in) every issued stage and A block
                const uint32_t issued = it;
                for (uint32_t t = issued > NST ? issued - NST : 0; t < issued; ++t) {
                    const uint32_t s = t % NST, r = t / NST;
                    if (!mbar_wait(smem_u32(&empty[s]), r & 1, abort_flag, true)) {
                        raise_error(abort_flag, &jobs[G.job_ids[0]].out->error_code, SC_ERR_DRAIN, peer_abort);
                        break;
                    }
                }
                if (un > 0 && !mbar_wait(smem_u32(aempty), (un - 1) & 1, abort_flag, true))
                    raise_error(abort_flag, &jobs[G.job_ids[0]].out->error_code, SC_ERR_DRAIN, peer_abort);
            } else {
                // drain: the last A block must have landed before the CTA exits
                if (a_res && un > 0 && !mbar_wait(smem_u32(afull), (un - 1) & 1, abort_flag, true))
                    raise_error(abort_flag, &jobs[G.job_ids[0]].out->error_code, SC_ERR_DRAIN, peer_abort);
                // drain: every issued stage must have landed before the CTA exits
                const uint32_t issued = it;
                for (uint32_t t = issued > NST ? issued - NST : 0; t < issued; ++t) {
                    const uint32_t s = t % NST, r = t / NST;
                    if (!mbar_wait(smem_u32(&full[s]), r & 1, abort_flag, true)) {
                        raise_error(abort_flag, &jobs[G.job_ids[0]].out->error_code, SC_ERR_DRAIN, peer_abort);
                        break;
                    }
                }
            }
        }
        __syncwarp();
    } else if (warp == 1) {
        // ------------------------------------------------------- MMA issuer
        // (2-SM form: the leader's alone, for both CTAs)
        if (lane == 0 && (!PAIR || leader)) {
            uint32_t it = 0, tile = 0, un = 0;
            bool ok = true;
            for (uint32_t u = wid; ok && u < nunits; u += nworkers) {
                const UnitTiles ut = unit_tiles(jobs, G, u, PASS);
                const JobDev &J = jobs[ut.job];
                if (!job_active(J)) continue;
                if (PAIR || a_res) {
                    if (!mbar_wait(smem_u32(afull), un & 1, abort_flag)) {
                        raise_error(abort_flag, &J.out->error_code, SC_ERR_MMA_FULL, peer_abort);
                        ok = false;
                        break;
                    }
                    fence_after_sync();
                }
                for (uint32_t ct = ut.ct_begin; ok && ct < ut.ct_end; ++ct, ++tile) {
                    const uint32_t buf = tile & 1, use = tile >> 1;
                    if (!mbar_wait(smem_u32(&acce[buf]), (use & 1) ^ 1, abort_flag)) {
                        raise_error(abort_flag, &J.out->error_code, SC_ERR_MMA_ACC, peer_abort);
                        ok = false;
                        break;
                    }
                    fence_after_sync();
                    const uint32_t d_tmem = tmem_base + buf * SC_BN;
                    for (uint32_t ks = 0; ks < J.k_stages; ++ks, ++it) {
                        const uint32_t s = it % NST, r = it / NST;
                        if (!mbar_wait(smem_u32(&full[s]), r & 1, abort_flag)) {
                            raise_error(abort_flag, &J.out->error_code, SC_ERR_MMA_FULL, peer_abort);
                            ok = false;
                            break;
                        }
                        fence_after_sync();
                        const uint32_t a0 = smem_u32(sA + ((PAIR || a_res) ? ks : s) * SC_A_BYTES);
                        const uint32_t b0 = smem_u32(sB + s * BST);
#pragma unroll
                        for (uint32_t kk = 0; kk < SC_SLICE_BYTES / 32; ++kk)
                            mma_issue<KIND, PAIR>(d_tmem, smem_desc(a0 + kk * 32), smem_desc(b0 + kk * 32),
                                                  idesc, (ks | kk) != 0);
                        mma_commit<PAIR>(smem_u32(&empty[s]));
                    }
                    if (!ok) break;
                    mma_commit<PAIR>(smem_u32(&accf[buf]));
                }
                if (ok && (PAIR || a_res)) {
                    mma_commit<PAIR>(smem_u32(aempty));  // the A block is free once these MMAs finish
                    ++un;
                }
            }
            // drain: the last commits must have landed before TMEM is freed
            if (it > 0) {
                const uint32_t s = (it - 1) % NST, r = (it - 1) / NST;
                if (!mbar_wait(smem_u32(&empty[s]), r & 1, abort_flag, true))
                    raise_error(abort_flag, &jobs[G.job_ids[0]].out->error_code, SC_ERR_DRAIN, peer_abort);
            }
            if ((PAIR || a_res) && un > 0 && !mbar_wait(smem_u32(aempty), (un - 1) & 1, abort_flag, true))
                raise_error(abort_flag, &jobs[G.job_ids[0]].out->error_code, SC_ERR_DRAIN, peer_abort);
        }
        __syncwarp();
    } else {
        // --------------------------------------------------------- epilogue
        // warps 2..EW+1: quadrant (warp & 3) of the TMEM lanes = 32 query
        // rows, segment (warp - 2) / 4 of the tile's 256 columns
        const uint32_t quad = (uint32_t)(warp & 3);
        const uint32_t seg = (uint32_t)(warp - 2) >> 2;
        const uint32_t row_in_tile = quad * 32 + lane;
        const float INF = __int_as_float(0x7f800000);
        // symmetric pass: this warp's stage of column-side candidates
        const uint32_t stage_slot = blockIdx.x * EW + (uint32_t)(warp - 2);
        const size_t stage0 = (size_t)stage_slot * G.stage_cap;
        uint32_t staged = 0;
        uint32_t tile = 0;
        bool ok = true;
        for (uint32_t u = wid; ok && u < nunits; u += nworkers) {
            const UnitTiles ut = unit_tiles(jobs, G, u, PASS);
            const JobDev &J = jobs[ut.job];
            if (!job_active(J)) continue;
            const uint32_t n = J.n;
            const uint32_t myrb = PAIR ? 2 * ut.rb + rank : ut.rb;  // this CTA's 128-row block
            const uint32_t row = myrb * SC_BM + row_in_tile;  // job-local
            const bool valid = row >= J.q0 && row < J.q1;
            const size_t gr = (size_t)J.row0 + row;              // group row
            // cosine rows compare 1 - v directly (every column term is 1 when
            // the job has no zero vectors)
            const bool fast_cos = J.metric == HM_METRIC_COSINE && J.cnt->maxb[7] == 0;
            const float band = valid ? G.band[gr] : 0.0f;
            const float rowterm = valid ? G.rowterm[gr] : 0.0f;
            const float scale = J.scale;
            // pass 0: the row's threshold-pass list (its k-array); pass 1: its
            // candidate list for this column part and segment
            const size_t list = PASS == 0 ? list_index(J, valid ? row : 0, ut.part * NSEG + seg)
                                          : cand_list(J, valid ? row : 0, ut.part * NSEG + seg);
            const float *colterm = G.colterm + J.row0;
            // pass 0: the k smallest mini-chunk minima seen (ascending;
            // arr[KP-1] is the list's k-th) and the row's shared k-th
            float arr[PASS == 0 ? KP : 1];
#pragma unroll
            for (int q = 0; q < (PASS == 0 ? KP : 1); ++q) arr[q] = (q < KP - (int)J.k) ? -INF : INF;
            float tglob = INF, published = INF;
            uint32_t tnext = 0xff800000u;  // ordered key of +inf
            const bool chunk_min = J.seed_tiles < J.part_tiles;
            // pass 1: the row's fixed limit, tau1 + band (symmetric: tau1 +
            // 2 band, precomputed; a pair's value may come from the tile of the
            // other orientation, within 2E of the threshold pass's value)
            float thr = -INF;
            if (PASS >= 1 && valid) thr = (SYMK && ut.sym) ? G.ethr[gr] : __fadd_ru(unord32(G.rowthr[gr]), band);
            // cosine fast path of pass 1: every v with fl(1 - v) <= thr has
            // v >= 1 - thr - ulp(thr)/2 >= vstar (2^-20 relative margin)
            const float vstar = !(thr < INF) ? -INF
                                             : __fsub_rd(__fsub_rd(1.0f, thr), fmaxf(fabsf(thr), 1.0f) * 0x1p-20f);
            uint32_t cnt = 0;
            unsigned long long *cand = PASS >= 1 ? cand_slots(J, G, list) : nullptr;
            // symmetric: this row's own term in its pairs' column-side values
            // (c^_ji = rowterm_j + colterm_i - scale v) and the column-side
            // candidates this thread staged in the unit
            const float own_ct = (SYMK && ut.sym && valid) ? G.colterm[gr] : 0.0f;
            uint32_t colsum = 0;

            for (uint32_t ct = ut.ct_begin; ct < ut.ct_end; ++ct, ++tile) {
                const uint32_t buf = tile & 1, use = tile >> 1;
                // symmetric emission: this warp's 64 columns lie in 128-column
                // block jb of the job; below the row block's diagonal its pairs
                // belong to another unit's column side, above it they also
                // serve the columns' rows
                const uint32_t c_base = ct * SC_BN + seg * SEGW;
                const uint32_t jb = c_base / SC_BM;
                const bool skip = SYMK && ut.sym && jb < myrb;
                const bool colside = SYMK && ut.sym && jb > myrb && c_base < n;
                // the columns' limits (lane t holds column c_base + 32 q + t),
                // loaded while the accumulator is still being filled
                constexpr int CQ = SEGW / 32;
                float cthr[CQ], cvs[CQ], cterm[CQ];
#pragma unroll
                for (int q = 0; q < CQ; ++q) {
                    cthr[q] = -INF;
                    cvs[q] = INF;
                    cterm[q] = 0.0f;
                }
                // and each 8-column group's smallest v* (lane t: its group's)
                float cgmin[CQ];
#pragma unroll
                for (int q = 0; q < CQ; ++q) cgmin[q] = INF;
                if (SYMK && colside) {
#pragma unroll
                    for (int q = 0; q < CQ; ++q) {
                        const size_t gc = (size_t)J.row0 + c_base + 32 * q + lane;
                        cthr[q] = G.ethr[gc];
                        cvs[q] = G.evstar[gc];
                        cterm[q] = G.colterm[gc];
                        float m = cvs[q];
                        m = fminf(m, __shfl_xor_sync(0xffffffffu, m, 1));
                        m = fminf(m, __shfl_xor_sync(0xffffffffu, m, 2));
                        cgmin[q] = fminf(m, __shfl_xor_sync(0xffffffffu, m, 4));
                    }
                }
                const bool got = mbar_wait(smem_u32(&accf[buf]), use & 1, abort_flag);
                if (!__all_sync(0xffffffffu, got)) {
                    raise_error(abort_flag, &J.out->error_code, SC_ERR_EPILOGUE, peer_abort);
                    ok = false;
                    break;
                }
                fence_after_sync();
                if (skip) {
                    __syncwarp();
                    if (lane == 0) {
                        if (PAIR)
                            mbar_arrive_cluster(cluster_addr(smem_u32(&acce[buf]), 0));
                        else
                            mbar_arrive(smem_u32(&acce[buf]));
                    }
                    continue;
                }
                if (PASS == 0 && valid) {
                    // the row's other lists may have tightened its k-th: use the
                    // value loaded during the previous tile, load the next one
                    tglob = fminf(tglob, unord32(tnext));
                    tnext = *(volatile const uint32_t *)(G.rowthr + gr);
                }
                const bool diag = (ct * SC_BN < myrb * SC_BM + SC_BM) && (myrb * SC_BM < ct * SC_BN + SC_BN);
                const uint32_t t_base = tmem_base + ((quad * 32) << 16) + buf * SC_BN + seg * SEGW;
                // the threshold pass's chunk = 32 columns; the accumulator
                // registers are overwritten in place by the screened values
                auto process = [&](uint32_t (&v)[32], uint32_t ch) {
                    float (&c)[32] = reinterpret_cast<float (&)[32]>(v);
                    const uint32_t j0 = c_base + ch * 32;  // job-local column
                    const bool full = j0 + 32 <= n;
                    const bool self_here = diag && (row - j0 < 32u);
                    // exact screened values of every column of the chunk
                    // (columns past n: +inf; the row itself: 0)
                    auto values = [&]() {
                        if (fast_cos) {
#pragma unroll
                            for (int t = 0; t < 32; ++t) c[t] = __fsub_rn(1.0f, c[t]);
                        } else {
                            const float4 *ctp = reinterpret_cast<const float4 *>(colterm + j0);
#pragma unroll
                            for (int q = 0; q < 8; ++q) {
                                const float4 cq = __ldg(ctp + q);
                                const float cs[4] = {cq.x, cq.y, cq.z, cq.w};
#pragma unroll
                                for (int e = 0; e < 4; ++e)
                                    c[4 * q + e] =
                                        __fsub_rn(__fadd_rn(rowterm, cs[e]), __fmul_rn(scale, c[4 * q + e]));
                            }
                        }
                        if (!full) {
#pragma unroll
                            for (int t = 0; t < 32; ++t)
                                if (j0 + t >= n) c[t] = INF;
                        }
                        if (self_here) {
#pragma unroll
                            for (int t = 0; t < 32; ++t)
                                if (j0 + t == row) c[t] = 0.0f;
                        }
                    };
                    // cosine fast path: c = 1 - v is monotone in v, so a
                    // minimum of c is 1 - (the maximum of v), bit for bit
                    const bool quick = fast_cos && full && !self_here && !dump;
                    if (PASS == 0) {
                        // mini-chunk minima: columns {t, t+8, t+16, t+24}
                        float m[8];
                        if (quick) {
#pragma unroll
                            for (int t = 0; t < 8; ++t)
                                m[t] = __fsub_rn(1.0f, fmaxf(fmaxf(c[t], c[t + 8]), fmaxf(c[t + 16], c[t + 24])));
                        } else {
                            values();
                            if (dump && valid) {
                                for (int t = 0; t < 32; ++t)
                                    if (j0 + t < n) dump[(size_t)row * n + j0 + t] = c[t];
                            }
#pragma unroll
                            for (int t = 0; t < 8; ++t)
                                m[t] = fminf(fminf(c[t], c[t + 8]), fminf(c[t + 16], c[t + 24]));
                        }
                        // a sampled threshold pass keeps one minimum per 32-column
                        // chunk (an eighth of the insertions; the sample's k smallest
                        // rarely share a chunk), a full one the eight mini-chunk minima
                        if (chunk_min) {
#pragma unroll
                            for (int t = 1; t < 8; ++t) m[0] = fminf(m[0], m[t]);
                        }
                        // minima that can be among the row's k smallest
                        uint32_t pm = 0;
#pragma unroll
                        for (int t = 0; t < 8; ++t)
                            pm |= (m[t] < arr[KP - 1] && !(m[t] > tglob) && (t == 0 || !chunk_min)) ? (1u << t) : 0u;
                        if (!valid) pm = 0;
                        if (pm) {
                            while (pm) {
                                const int t = __ffs(pm) - 1;
                                pm &= pm - 1;
                                float x = m[0];
#pragma unroll
                                for (int q = 1; q < 8; ++q) x = (t == q) ? m[q] : x;
                                if (x < arr[KP - 1]) {
#pragma unroll
                                    for (int q = KP - 1; q > 0; --q) arr[q] = fminf(arr[q], fmaxf(arr[q - 1], x));
                                    arr[0] = fminf(arr[0], x);
                                }
                            }
                            const float tl = arr[KP - 1];
                            if (tl < published) {
                                // share with the row's other lists: a reduction
                                // whose result is not waited for (the other
                                // lists' values arrive through tnext, loaded a
                                // tile ahead)
                                atomicMin(G.rowthr + gr, ord32(tl));
                                tglob = fminf(tglob, tl);
                                published = tl;
                            }
                        }
                    }
                };
                if constexpr (EW >= 16) {
                    // the full emission pass (96 registers a thread): 16-column
                    // loads, the next in flight while this one is tested
                    const uint32_t cap = J.cap;
                    // symmetric emission, column side, on the raw products:
                    // column j of the chunk takes this row as a candidate when
                    // c^_ji <= its limit (cosine without zero rows: the raw
                    // product against the column's v* form, a superset); one
                    // ballot per column names the warp's rows that it takes,
                    // staged for column_scatter_kernel
                    static_assert(!SYMK || CQ == 2, "two 32-column register slices per 64-column segment");
                    auto colside16 = [&](const float (&c)[16], uint32_t j0) {
                        const uint32_t cc = (j0 - c_base) >> 4;  // chunk of the segment
                        const bool hi = (cc >> 1) != 0;
                        const float thr_q = hi ? cthr[CQ - 1] : cthr[0];
                        const float vs_q = hi ? cvs[CQ - 1] : cvs[0];
                        const float term_q = hi ? cterm[CQ - 1] : cterm[0];
                        const float gmin_q = hi ? cgmin[CQ - 1] : cgmin[0];
                        const uint32_t lb = 16u * (cc & 1u);  // the chunk's first column's lane
                        const bool euc = J.metric == HM_METRIC_EUCLIDEAN;
                        // the warp's own stage (no atomics): its count is
                        // uniform over the warp
                        auto stage = [&](uint32_t m, int t) {
                            const uint32_t base = staged;
                            staged += (uint32_t)__popc(m);
                            if (lane == 0) colsum += (uint32_t)__popc(m);
                            if (m & (1u << lane)) {
                                const uint32_t pos = base + (uint32_t)__popc(m & ((1u << lane) - 1u));
                                if (pos < G.stage_cap) {
                                    const size_t at = stage0 + pos;
                                    G.stage_row[at] = J.row0 + j0 + t;
                                    G.stage_key[at] = ((unsigned long long)__float_as_uint(c[t]) << 32) | row;
                                } else {
                                    // a full stage: the column's row goes to the exact path
                                    atomicMax(&G.cand_cnt[cand_list(J, j0 + t, J.elists - 2)], 2 * J.cap + 1);
                                }
                            }
                        };
                        if (fast_cos) {
#pragma unroll
                            for (int g = 0; g < 2; ++g) {
                                float x = c[8 * g];
#pragma unroll
                                for (int e = 1; e < 8; ++e) x = fmaxf(x, c[8 * g + e]);
                                const float cm = __shfl_sync(0xffffffffu, gmin_q, (int)lb + 8 * g);
                                if (!__any_sync(0xffffffffu, valid && x >= cm)) continue;
#pragma unroll
                                for (int e = 0; e < 8; ++e) {
                                    const int t = 8 * g + e;
                                    const float vs = __shfl_sync(0xffffffffu, vs_q, (int)lb + t);
                                    const uint32_t m = __ballot_sync(0xffffffffu, valid && c[t] >= vs && j0 + t < n);
                                    if (m) stage(m, t);
                                }
                            }
                        } else {
#pragma unroll
                            for (int t = 0; t < 16; ++t) {
                                const float lim = __shfl_sync(0xffffffffu, thr_q, (int)lb + t);
                                const float rt = __shfl_sync(0xffffffffu, term_q, (int)lb + t);
                                const float c2 = __fsub_rn(__fadd_rn(euc ? rt : 0.0f, own_ct), __fmul_rn(scale, c[t]));
                                const uint32_t m = __ballot_sync(0xffffffffu, valid && j0 + t < n && !(c2 > lim));
                                if (m) stage(m, t);
                            }
                        }
                    };
                    auto emit16 = [&](uint32_t (&v)[16], uint32_t j0) {
                        float (&c)[16] = reinterpret_cast<float (&)[16]>(v);
                        if constexpr (SYMK) {
                            if (colside) colside16(c, j0);
                        }
                        const bool full = j0 + 16 <= n;
                        const bool self_here = diag && (row - j0 < 16u);
                        auto put = [&](uint32_t pm, int g, bool raw) {
                            while (pm) {
                                const int e = __ffs(pm) - 1;
                                pm &= pm - 1;
                                const float a0 = (e & 1) ? c[8 * g + 1] : c[8 * g];
                                const float a1 = (e & 1) ? c[8 * g + 3] : c[8 * g + 2];
                                const float a2 = (e & 1) ? c[8 * g + 5] : c[8 * g + 4];
                                const float a3 = (e & 1) ? c[8 * g + 7] : c[8 * g + 6];
                                const float b0 = (e & 2) ? a1 : a0, b1 = (e & 2) ? a3 : a2;
                                float x = (e & 4) ? b1 : b0;
                                if (raw) x = __fsub_rn(1.0f, x);
                                if (cnt < cap)
                                    cand[cnt] = ((unsigned long long)__float_as_uint(x) << 32) | (j0 + 8 * g + e);
                                ++cnt;
                            }
                        };
                        if (fast_cos && full && !self_here) {
                            // c = 1 - v <= thr  <=>  v >= vstar (a superset)
                            float gm[2];
#pragma unroll
                            for (int g = 0; g < 2; ++g) {
                                float x = c[8 * g];
#pragma unroll
                                for (int e = 1; e < 8; ++e) x = fmaxf(x, c[8 * g + e]);
                                gm[g] = x;
                            }
                            if (valid && fmaxf(gm[0], gm[1]) >= vstar) {
#pragma unroll
                                for (int g = 0; g < 2; ++g) {
                                    if (gm[g] >= vstar) {
                                        uint32_t pm = 0;
#pragma unroll
                                        for (int e = 0; e < 8; ++e) pm |= (c[8 * g + e] >= vstar) ? (1u << e) : 0u;
                                        put(pm, g, true);
                                    }
                                }
                            }
                            return;
                        }
                        // exact screened values (columns past n: +inf; the row itself: 0)
                        if (fast_cos) {
#pragma unroll
                            for (int t = 0; t < 16; ++t) c[t] = __fsub_rn(1.0f, c[t]);
                        } else {
                            const float4 *ctp = reinterpret_cast<const float4 *>(colterm + j0);
#pragma unroll
                            for (int q = 0; q < 4; ++q) {
                                const float4 cq = __ldg(ctp + q);
                                const float cs[4] = {cq.x, cq.y, cq.z, cq.w};
#pragma unroll
                                for (int e = 0; e < 4; ++e)
                                    c[4 * q + e] = __fsub_rn(__fadd_rn(rowterm, cs[e]), __fmul_rn(scale, c[4 * q + e]));
                            }
                        }
                        if (!full) {
#pragma unroll
                            for (int t = 0; t < 16; ++t)
                                if (j0 + t >= n) c[t] = INF;
                        }
                        if (self_here) {
#pragma unroll
                            for (int t = 0; t < 16; ++t)
                                if (j0 + t == row) c[t] = 0.0f;
                        }
                        float gm[2];
#pragma unroll
                        for (int g = 0; g < 2; ++g) {
                            float x = c[8 * g];
#pragma unroll
                            for (int e = 1; e < 8; ++e) x = fminf(x, c[8 * g + e]);
                            gm[g] = x;
                        }
                        if (valid && !(fminf(gm[0], gm[1]) > thr)) {
#pragma unroll
                            for (int g = 0; g < 2; ++g) {
                                if (!(gm[g] > thr)) {
                                    uint32_t pm = 0;
#pragma unroll
                                    for (int e = 0; e < 8; ++e)
                                        pm |= (!(c[8 * g + e] > thr) && j0 + 8 * g + e < n) ? (1u << e) : 0u;
                                    put(pm, g, false);
                                }
                            }
                        }
                    };
                    uint32_t va[16], vb[16];
                    tmem_ld16_issue(t_base, va);
                    tmem_ld_wait16(va);
#pragma unroll 1
                    for (uint32_t ch = 0; ch < SEGW / 16; ch += 2) {
                        tmem_ld16_issue(t_base + (ch + 1) * 16, vb);
                        emit16(va, c_base + ch * 16);
                        tmem_ld_wait16(vb);
                        if (ch + 2 < SEGW / 16) tmem_ld16_issue(t_base + (ch + 2) * 16, va);
                        emit16(vb, c_base + (ch + 1) * 16);
                        if (ch + 2 < SEGW / 16) tmem_ld_wait16(va);
                    }
                } else {
                    // two warps per scheduler: the next chunk loads while
                    // this one is processed
                    uint32_t va[32], vb[32];
                    tmem_ld32_issue(t_base, va);
                    tmem_ld_wait(va);
#pragma unroll 1
                    for (uint32_t ch = 0; ch < SEGW / 32; ch += 2) {
                        tmem_ld32_issue(t_base + (ch + 1) * 32, vb);
                        process(va, ch);
                        tmem_ld_wait(vb);
                        if (ch + 2 < SEGW / 32) tmem_ld32_issue(t_base + (ch + 2) * 32, va);
                        process(vb, ch + 1);
                        if (ch + 2 < SEGW / 32) tmem_ld_wait(va);
                    }
                }
                fence_before_sync();
                __syncwarp();
                if (lane == 0) {
                    if (PAIR)
                        mbar_arrive_cluster(cluster_addr(smem_u32(&acce[buf]), 0));
                    else
                        mbar_arrive(smem_u32(&acce[buf]));
                }
            }
            if (!ok) break;
            if (PASS == 0) {
                if (valid) {
                    // the list's k smallest mini-chunk minima (ascending)
                    float *kk = G.topk + J.topk0 + (list - J.slot0) * J.k;
#pragma unroll
                    for (int q = 0; q < KP; ++q)
                        if (q >= KP - (int)J.k) kk[q - (KP - (int)J.k)] = arr[q];
                }
            } else {
                if (valid) G.cand_cnt[list] = cnt;
                const uint32_t e = __reduce_add_sync(0xffffffffu, (valid ? cnt : 0u) + colsum);
                if (lane == 0 && e) atomicAdd(&J.out->emitted, (unsigned long long)e);
            }
        }
        if (SYMK && lane == 0 && G.stage_cnt) G.stage_cnt[stage_slot] = staged;
    }

    fence_before_sync();
    __syncthreads();
    if (PAIR) cluster_sync();  // neither CTA leaves while the other may still signal it
    if (warp == 1) {
        fence_after_sync();
        if (PAIR)
            asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem_base),
                         "r"(SC_TMEM_COLS));
        else
            asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_base),
                         "r"(SC_TMEM_COLS));
    }

}

// clusters of two CTAs of `func` (a screen kernel launched with `threads`
// threads) the device can hold at once; computed on first use per kernel and
// device, 0 when none fits
static uint32_t pair_slots(const void *func, uint32_t threads) {
    struct Entry {
        const void *func;
        int dev;
        uint32_t clusters;
    };
    static std::mutex mu;
    static std::vector<Entry> cache;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        (void)cudaGetLastError();
        return 0;
    }
    {
        std::lock_guard<std::mutex> lk(mu);
        for (const Entry &e : cache)
            if (e.func == func && e.dev == dev) return e.clusters;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(2 * (uint32_t)device_sm_count(), 1, 1);
    cfg.blockDim = dim3(threads, 1, 1);
    cfg.dynamicSmemBytes = SC_SMEM_BYTES;
    cudaLaunchAttribute attr;
    attr.id = cudaLaunchAttributeClusterDimension;
    attr.val.clusterDim.x = 2;
    attr.val.clusterDim.y = 1;
    attr.val.clusterDim.z = 1;
    cfg.attrs = &attr;
    cfg.numAttrs = 1;
    int clusters = 0;
    if (cudaOccupancyMaxActiveClusters(&clusters, func, &cfg) != cudaSuccess || clusters < 1) {
        (void)cudaGetLastError();
        return 0;
    }
    std::lock_guard<std::mutex> lk(mu);
    cache.push_back({func, dev, (uint32_t)clusters});
    return (uint32_t)clusters;
}

// an emission pass in the 2-SM form: clusters of two, the A block resident
// in each CTA, one MMA of M = 256 per K step
template <int KIND, int PASS>
static int launch_pair(const JobDev *jobs, const GroupDev &G, const CUtensorMap &ta, const CUtensorMap &tb,
                       uint32_t idesc, cudaStream_t s) {
    const void *func = (const void *)screen_gemm_kernel<KIND, 32, PASS, true>;
    HM_TRY(ensure_dynamic_smem(func, (int)SC_SMEM_BYTES));
    const uint32_t slots = pair_slots(func, (uint32_t)sc_threads(PASS));
    if (slots == 0) return set_error(HM_ERR_CUDA, "no room for a cluster of two screen CTAs");
    const uint32_t clusters = G.neunits < slots ? G.neunits : slots;
    if (clusters == 0) return HM_OK;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(2 * clusters, 1, 1);
    cfg.blockDim = dim3(sc_threads(PASS), 1, 1);
    cfg.dynamicSmemBytes = SC_SMEM_BYTES;
    cfg.stream = s;
    cudaLaunchAttribute attr;
    attr.id = cudaLaunchAttributeClusterDimension;
    attr.val.clusterDim.x = 2;
    attr.val.clusterDim.y = 1;
    attr.val.clusterDim.z = 1;
    cfg.attrs = &attr;
    cfg.numAttrs = 1;
    const uint32_t pidesc = (idesc & ~(0x1fu << 24)) | (((uint32_t)(2 * SC_BM) >> 4) << 24);  // M = 256
    HM_CUDA_TRY(cudaLaunchKernelEx(&cfg, screen_gemm_kernel<KIND, 32, PASS, true>, ta, tb, jobs, G,
                                   (float *)nullptr, pidesc, 1u));
    count_launch();
    return HM_OK;
}

template <int KIND, int KP, int PASS>
static int launch_kind(const JobDev *jobs, const GroupDev &G, const CUtensorMap &ta,
                       const CUtensorMap &tb, float *dump, uint32_t idesc, cudaStream_t s) {
    if constexpr (PASS >= 1 && KP == 32) {
        if (G.pair) return launch_pair<KIND, PASS>(jobs, G, ta, tb, idesc, s);
    }
    HM_TRY(ensure_dynamic_smem((const void *)screen_gemm_kernel<KIND, KP, PASS, false>, (int)SC_SMEM_BYTES));
    const uint32_t sms = (uint32_t)device_sm_count();
    const uint32_t grid = PASS >= 1 ? emission_grid(G) : (G.units < sms ? G.units : sms);
    if (grid == 0) return HM_OK;
    // every job's K slices fit the resident A block
    const uint32_t a_res = (G.kpmax / G.kslice) <= SC_ARES_STAGES ? 1u : 0u;
    screen_gemm_kernel<KIND, KP, PASS, false><<<grid, sc_threads(PASS, KP), SC_SMEM_BYTES, s>>>(ta, tb, jobs, G, dump,
                                                                                      idesc, a_res);
    HM_CUDA_TRY(cudaGetLastError());
    count_launch();
    return HM_OK;
}

uint32_t emission_grid(const GroupDev &G) {
    const uint32_t sms = (uint32_t)device_sm_count();
    return G.neunits < sms ? G.neunits : sms;
}

static uint32_t make_idesc(int kind) {
    const uint32_t fmt = kind == SCREEN_KIND_BF16 ? 1u : 2u;  // BF16 / TF32 operands
    return (1u << 4)                    // accumulator: F32
           | (fmt << 7) | (fmt << 10)   // A, B formats
           | (0u << 15) | (0u << 16)    // A, B K-major
           | ((uint32_t)(SC_BN >> 3) << 17) | ((uint32_t)(SC_BM >> 4) << 24);
}

template <int KIND>
static int launch_pass(const JobDev *jobs, const GroupDev &G, uint32_t kp, const CUtensorMap &ta,
                       const CUtensorMap &tb, float *dump, uint32_t idesc, int pass, cudaStream_t s) {
    if (pass == 1) return launch_kind<KIND, 32, 1>(jobs, G, ta, tb, nullptr, idesc, s);
    if (pass == 2) return launch_kind<KIND, 32, 2>(jobs, G, ta, tb, nullptr, idesc, s);
    if (kp == 32) return launch_kind<KIND, 32, 0>(jobs, G, ta, tb, dump, idesc, s);
    if (kp == 64) return launch_kind<KIND, 64, 0>(jobs, G, ta, tb, dump, idesc, s);
    return set_error(HM_ERR_UNSUPPORTED, "screen top-k width %u", kp);
}

// pass 0: each list's k smallest chunk minima over the column sample (-> tau1);
// pass 1: emission of every column within tau1 + band; pass 2: the same for a
// group with symmetric units (tiles on and above the diagonal, column side too)
int launch_screen_gemm(const JobDev *jobs, const GroupDev &G, const GroupDev *, uint32_t kp,
                       const CUtensorMap &ta, const CUtensorMap &tb, float *dump, int pass,
                       cudaStream_t s) {
    if (G.units == 0) return HM_OK;
    ScopedKernelTimer timer(HM_KCLASS_BULK, s);
    const uint32_t idesc = make_idesc((int)G.kind);
    if (G.kind == SCREEN_KIND_BF16)
        return launch_pass<SCREEN_KIND_BF16>(jobs, G, kp, ta, tb, dump, idesc, pass, s);
    return launch_pass<SCREEN_KIND_TF32>(jobs, G, kp, ta, tb, dump, idesc, pass, s);
}

}  // namespace hm
