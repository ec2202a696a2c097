// api.cu -- the extern "C" entry points of libholomap_cuda.so and the batch
// planner / executor behind them.
//
// Host side of the drop-in for src/api.rs:147-148 (exact_knn + smooth_knn).
// Every call is a batch of jobs (a single call is a batch of one).  The plan
// resolves each job's path (exact plain path, or a tensor-core screen whose
// operand format groups the jobs), lays out every buffer in one workspace
// and writes the job tables; the run enqueues, on one stream:
//   init counters + input check + cosine norms        (all jobs)
//   binary64 copies + exact plain kernel              (exact-path jobs)
//   screen prep -> band -> screen -> rerank           (per screen group)
//   binary64 copies + plain kernel on fallback rows   (screened jobs)
//   split merge                                       (exact jobs with splits)
//   smooth-kNN + global-mean floors                   (all jobs with outputs)
// Validation mirrors src/api.rs:114-145 on exact_knn's own domain.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "hm_internal.cuh"
#include "screen.cuh"

namespace hm {

static thread_local std::string g_last_error;

int set_error(int code, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}

void clear_error() { g_last_error.clear(); }

// tensor maps and the test hook live in screen.cu
int make_operand_map(CUtensorMap *m, void *base, uint64_t rows, uint32_t kpmax, uint32_t elem_bytes,
                     uint32_t kslice, uint32_t box_rows);
float *debug_dump_pointer();

static size_t align256(size_t x) { return round_up(x, 256); }

static uint32_t pow2ceil(uint32_t v) {
    uint32_t p = 1;
    while (p < v) p <<= 1;
    return p;
}

static int sm_count() { return device_sm_count(); }

// ------------------------------------------------------------ validation
static int validate_shape(uint64_t n, uint32_t d, uint32_t k, int metric) {
    if (d == 0 || n == 0)
        return set_error(HM_ERR_INVALID, "bad shape: n=%llu rows of n_features=%u",
                         (unsigned long long)n, d);
    // exact_knn's own domain is 1 <= k <= n (src/knn.rs:22-55 takes the first
    // k of n sorted entries); fit_transform narrows it to k >= 2 and n > k
    // (src/api.rs:123-141) before calling it.
    if (k < 1) return set_error(HM_ERR_INVALID, "n_neighbors must be >= 1");
    if (n < k)
        return set_error(HM_ERR_INVALID, "need at least n_neighbors=%u points, got %llu", k,
                         (unsigned long long)n);
    if (metric < HM_METRIC_EUCLIDEAN || metric > HM_METRIC_MANHATTAN)
        return set_error(HM_ERR_INVALID, "unknown metric %d", metric);
    if (n > 0x7fffffffull)
        return set_error(HM_ERR_UNSUPPORTED, "n=%llu exceeds the supported index range",
                         (unsigned long long)n);
    if (kpl_for_k(k) == 0)
        return set_error(HM_ERR_UNSUPPORTED, "k=%u exceeds the largest supported k (256)", k);
    return HM_OK;
}

static bool screen_capable(uint32_t d, uint32_t k, int metric) {
    return metric != HM_METRIC_MANHATTAN && k <= 64 && d <= 2048;
}

// ------------------------------------------------------------------ plan
struct JobPlan {
    hm_job spec{};
    int path = HM_PATH_PLAIN;
    uint32_t ldd = 0, n_pad = 0, splits = 1, split_cols = 0, arow0 = 0;
    uint32_t q0 = 0, q1 = 0, rb0 = 0;  // query rows [q0, q1) (a row shard)
    size_t off_x64 = 0, off_rnorm = 0, off_partial = 0, off_zero_rows = 0, off_ovf = 0;
    size_t off_mu = 0, off_csum = 0;
    int group = -1;
    uint32_t row0 = 0, unit0 = 0, kp1 = 0, k_stages = 0, row_blocks = 0, col_tiles = 0;
    uint32_t parts = 1, part_tiles = 0, cap = 0, seed_tiles = 0, tlists = 2;
    uint64_t slot0 = 0, cand0 = 0, topk0 = 0;
    // emission pass: symmetric (tiles on and above the diagonal), its column
    // parts per row block of ept tiles, candidate lists per row
    bool sym = false;
    uint32_t ept = 0, elists = 0;
    uint64_t eslot0 = 0;
    // escalation: the job's split-BF16 copy (clone), or the job a copy is of
    int clone = -1, clone_of = -1;
};

struct GroupPlan {
    int kind = SCREEN_KIND_BF16;
    bool split = false;
    uint32_t elem_bytes = 2, kslice = 64, kpmax = 0, rows = 0, units = 0;
    uint32_t kp = 32, kpl = 1, dmax = 0;
    int metric_mask = 0;
    std::vector<uint32_t> jobs;
    uint64_t lists = 0, cand = 0, topk = 0, elists = 0;
    std::vector<uint4> eunits;  // emission units, largest first
    bool any_sym = false;
    bool pair = false;  // emission pass in the 2-SM form (units of 256 rows)
    bool pair_vetoed = false;  // the autotuner table prefers one CTA per row block for a job
    bool any_escalation = false;  // a job of the group has a split-BF16 escalation copy
    uint32_t egrid = 0, stage_cap = 0;
    size_t off_opa = 0, off_opb = 0, off_rowstat = 0, off_rowterm = 0, off_colterm = 0;
    size_t off_band = 0, off_force = 0, off_rowthr = 0, off_cand = 0, off_cnt = 0, off_topk = 0;
    size_t off_ethr = 0, off_evstar = 0, off_stage_row = 0, off_stage_key = 0, off_stage_cnt = 0;
    size_t off_rowcnt = 0;
    // tables
    size_t off_gdev = 0, off_job_ids = 0, off_row_starts = 0, off_unit_starts = 0, off_eunits = 0;
    GroupDev host{};
    CUtensorMap ta{}, tb{};
    CUtensorMap tb_half{};  // 2-SM form: B in boxes of 128 rows (half a column tile)
};

}  // namespace hm

struct hm_batch {
    std::vector<hm::JobPlan> jobs;  // the caller's jobs, then their escalation copies
    uint32_t user_jobs = 0;
    hm::GroupPlan groups[3];  // bf16, tf32, split bf16
    uint32_t all_rows = 0, kmax = 0, kpl_all = 1, kpl_plain[3] = {1, 1, 1}, kpl_fb[3] = {1, 1, 1};
    std::vector<uint2> items[3];       // exact-path work per metric
    std::vector<uint32_t> fb_jobs[3];  // screened jobs per metric (fallback rows)
    uint32_t fb_per_job[3] = {1, 1, 1};
    std::vector<uint32_t> job_blocks;  // prep block offsets
    bool any_plain = false, any_screen = false, any_smooth = false, any_split = false;
    size_t off_tables = 0, off_jobs = 0, off_counters = 0, off_row_starts = 0, off_job_blocks = 0;
    size_t off_items[3] = {}, off_fb[3] = {};
    size_t tables_bytes = 0, tables_used = 0, total = 0;
    // bound state
    char *ws = nullptr;
    std::vector<char> table;           // host image of the tables
    cudaGraphExec_t graph = nullptr;
    cudaStream_t capture = nullptr;    // private stream the graph is captured on
    ~hm_batch() {
        if (graph) cudaGraphExecDestroy(graph);
        if (capture) cudaStreamDestroy(capture);
    }
};

namespace hm {

static int group_of_path(int path) {
    switch (path) {
    case HM_PATH_SCREEN_BF16: return 0;
    case HM_PATH_SCREEN_TF32: return 1;
    case HM_PATH_SCREEN_BF16X3: return 2;
    default: return -1;
    }
}

// `ranges` (optional): 2 per job, the job's query rows [begin, end); every
// point stays a column.  NULL: all rows.
static int plan_batch(const hm_job *user_specs, uint32_t user_jobs, hm_batch &B,
                      const uint64_t *user_ranges = nullptr) {
    if (user_jobs == 0) return set_error(HM_ERR_INVALID, "empty batch");
    if (user_jobs > (1u << 16)) return set_error(HM_ERR_UNSUPPORTED, "more than 65536 jobs");
    const uint32_t G = (uint32_t)sm_count();
    const bool batched = user_jobs > 1;
    // Escalation copies: a job left to the autotuner whose choice is the BF16
    // or TF32 screen also gets a split-BF16 copy on the same points and
    // outputs (no smooth-kNN of its own), appended after the caller's jobs;
    // on the device one of the two finishes the job.
    std::vector<hm_job> ext(user_specs, user_specs + user_jobs);
    std::vector<uint64_t> ext_ranges;
    if (user_ranges) ext_ranges.assign(user_ranges, user_ranges + 2 * (size_t)user_jobs);
    std::vector<uint32_t> clone_src;
    if (tuning_escalation()) {
        for (uint32_t j = 0; j < user_jobs; ++j) {
            const hm_job &s = user_specs[j];
            if (s.path != HM_PATH_AUTO || validate_shape(s.n, s.d, s.k, s.metric) != HM_OK) continue;
            const int p = autotune_choice(s.n, s.d, s.k, s.metric, nullptr, nullptr, nullptr, batched);
            if (p != HM_PATH_SCREEN_BF16 && p != HM_PATH_SCREEN_TF32) continue;
            hm_job c = s;
            c.path = HM_PATH_SCREEN_BF16X3;
            c.sigma_out = nullptr;
            c.rho_out = nullptr;
            ext.push_back(c);
            if (user_ranges) {
                ext_ranges.push_back(user_ranges[2 * j]);
                ext_ranges.push_back(user_ranges[2 * j + 1]);
            }
            clone_src.push_back(j);
        }
        clear_error();
    }
    const hm_job *specs = ext.data();
    const uint64_t *ranges = user_ranges ? ext_ranges.data() : nullptr;
    const uint32_t njobs = (uint32_t)ext.size();
    B.user_jobs = user_jobs;
    B.jobs.assign(njobs, JobPlan{});
    for (uint32_t c = 0; c < (uint32_t)clone_src.size(); ++c) {
        B.jobs[clone_src[c]].clone = (int)(user_jobs + c);
        B.jobs[user_jobs + c].clone_of = (int)clone_src[c];
    }
    for (int g = 0; g < 3; ++g) B.groups[g] = GroupPlan{};
    B.groups[0].kind = SCREEN_KIND_BF16;
    B.groups[1].kind = SCREEN_KIND_TF32;
    B.groups[1].elem_bytes = 4;
    B.groups[2].split = true;
    for (int g = 0; g < 3; ++g) B.groups[g].kslice = SC_SLICE_BYTES / B.groups[g].elem_bytes;

    // paths and exact-path geometry
    uint64_t plain_groups = 0;
    for (uint32_t j = 0; j < njobs; ++j) {
        JobPlan &P = B.jobs[j];
        P.spec = specs[j];
        const hm_job &s = P.spec;
        HM_TRY(validate_shape(s.n, s.d, s.k, s.metric));
        int path = s.path;
        if (path == HM_PATH_AUTO)
            path = autotune_choice(s.n, s.d, s.k, s.metric, nullptr, nullptr, nullptr, batched);
        if (path < HM_PATH_PLAIN || path > HM_PATH_SCREEN_BF16X3)
            return set_error(HM_ERR_INVALID, "unknown path %d", s.path);
        if (path != HM_PATH_PLAIN && !screen_capable(s.d, s.k, s.metric))
            return set_error(HM_ERR_UNSUPPORTED,
                             "the screened paths need euclidean or cosine, k <= 64 and d <= 2048");
        P.path = path;
        const uint64_t q0 = ranges ? ranges[2 * j] : 0, q1 = ranges ? ranges[2 * j + 1] : s.n;
        if (q0 >= q1 || q1 > s.n)
            return set_error(HM_ERR_INVALID, "query rows [%llu, %llu) outside [0, %llu)",
                             (unsigned long long)q0, (unsigned long long)q1, (unsigned long long)s.n);
        if (ranges && (s.sigma_out || s.rho_out))
            return set_error(HM_ERR_INVALID, "a row shard has no smooth-kNN outputs");
        P.q0 = (uint32_t)q0;
        P.q1 = (uint32_t)q1;
        P.ldd = (uint32_t)round_up(s.d, PL_BK);
        P.n_pad = (uint32_t)(round_up(s.n, PL_ROW_PAD) + PL_ROW_PAD);
        P.arow0 = B.all_rows;
        B.all_rows += (uint32_t)s.n;
        B.kpl_all = std::max<uint32_t>(B.kpl_all, (uint32_t)kpl_for_k(s.k));
        B.kmax = std::max<uint32_t>(B.kmax, s.k);
        if (s.sigma_out && s.rho_out) B.any_smooth = true;
        if (path == HM_PATH_PLAIN) plain_groups += (P.q1 + PL_BM - 1) / PL_BM - P.q0 / PL_BM;
    }
    // column splits of the exact path: about 8 CTAs per SM over the batch, down
    // to one 128-column tile per split (C1, 1,000 points: 0.147 -> 0.128 ms
    // against splits of at least two tiles)
    uint32_t S = plain_groups ? (uint32_t)((1184 + plain_groups - 1) / plain_groups) : 1;
    S = std::min<uint32_t>(std::max<uint32_t>(S, 1), 32);
    for (uint32_t j = 0; j < njobs; ++j) {
        JobPlan &P = B.jobs[j];
        const uint64_t n = P.spec.n;
        const uint32_t col_tiles = (uint32_t)((n + PL_BN - 1) / PL_BN);
        uint32_t splits = 1;
        if (P.path == HM_PATH_PLAIN) {
            splits = std::min<uint32_t>(S, std::max<uint32_t>(1, col_tiles));
            B.any_plain = true;
        }
        P.split_cols = (uint32_t)round_up((n + splits - 1) / splits, PL_BN);
        P.splits = (uint32_t)((n + P.split_cols - 1) / P.split_cols);
        if (P.splits > 1) B.any_split = true;
    }

    // screen groups
    for (uint32_t j = 0; j < njobs; ++j) {
        JobPlan &P = B.jobs[j];
        const int g = group_of_path(P.path);
        if (g < 0) continue;
        GroupPlan &Gp = B.groups[g];
        P.group = g;
        Gp.jobs.push_back(j);
        B.any_screen = true;
        P.kp1 = (uint32_t)round_up(P.spec.d, Gp.kslice);
        const uint32_t kp = Gp.split ? 3 * P.kp1 : P.kp1;
        P.k_stages = kp / Gp.kslice;
        Gp.kpmax = std::max(Gp.kpmax, kp);
        Gp.dmax = std::max(Gp.dmax, P.spec.d);
        if (P.spec.k > 32) {
            Gp.kp = 64;
            Gp.kpl = 2;
        }
        Gp.metric_mask |= 1 << P.spec.metric;
        P.rb0 = P.q0 / SC_BM;
        P.row_blocks = (P.q1 + SC_BM - 1) / SC_BM - P.rb0;
        P.col_tiles = (uint32_t)((P.spec.n + SC_BN - 1) / SC_BN);
    }
    for (int g = 0; g < 3; ++g) {
        GroupPlan &Gp = B.groups[g];
        if (Gp.jobs.empty()) continue;
        uint64_t units1 = 0;
        for (uint32_t j : Gp.jobs) units1 += B.jobs[j].row_blocks;
        for (uint32_t j : Gp.jobs) {
            JobPlan &P = B.jobs[j];
            if (Gp.jobs.size() == 1) {
                // one job: balance the persistent grid (makespan in tiles)
                // against the extra lists each column part costs
                double best = 1e300;
                for (uint32_t sp = 1; sp <= 8 && sp <= P.col_tiles; ++sp) {
                    const uint32_t pt = (P.col_tiles + sp - 1) / sp;
                    const uint32_t parts = (P.col_tiles + pt - 1) / pt;
                    const uint64_t units = (uint64_t)P.row_blocks * parts;
                    const double cost = (double)((units + G - 1) / G) * pt * (1.0 + 0.03 * parts);
                    if (cost < best - 1e-9) {
                        best = cost;
                        P.part_tiles = pt;
                        P.parts = parts;
                    }
                }
            } else {
                uint32_t parts = units1 >= G ? 1u : (uint32_t)((G + units1 - 1) / units1);
                parts = std::min<uint32_t>(std::min<uint32_t>(parts, 8), P.col_tiles);
                P.part_tiles = (P.col_tiles + parts - 1) / parts;
                P.parts = (P.col_tiles + P.part_tiles - 1) / P.part_tiles;
            }
            // threshold-pass sample: 1/seed_div of the columns (the autotuner
            // table's choice for the shape), at least 2048 (all of them for
            // small jobs), spread over the parts
            uint32_t seed_div = 8;
            bool sym_ok = true, pair_ok = true;
            autotune_choice(P.spec.n, P.spec.d, P.spec.k, P.spec.metric, &seed_div, &sym_ok, &pair_ok,
                            batched);
            if (P.clone >= 0 || P.clone_of >= 0) sym_ok = false;  // an escalation pair runs the full pass
            if (P.clone >= 0) Gp.any_escalation = true;
            if (!pair_ok) Gp.pair_vetoed = true;
            const uint64_t seed_cols = std::max<uint64_t>(P.spec.n / std::max<uint32_t>(seed_div, 1), 2048);
            P.seed_tiles = std::min<uint32_t>(
                P.part_tiles, (uint32_t)((seed_cols + (uint64_t)SC_BN * P.parts - 1) / ((uint64_t)SC_BN * P.parts)));
            P.seed_tiles = std::max<uint32_t>(P.seed_tiles, 1);
            P.row0 = Gp.rows;
            Gp.rows += (uint32_t)round_up(P.spec.n, 32);  // rows of each job start 32-aligned
            P.unit0 = Gp.units;
            Gp.units += P.row_blocks * P.parts;
            P.slot0 = Gp.lists;
            // threshold-pass lists: one per epilogue segment and column part
            P.tlists = (uint32_t)sc_epi_warps(0, (int)Gp.kp) / 4;
            const uint64_t lists = P.spec.n * (uint64_t)P.tlists * P.parts;
            Gp.lists += lists;
            P.topk0 = Gp.topk;
            Gp.topk += lists * P.spec.k;
            // Emission pass.  A whole dataset (not a row shard) with at least
            // two column tiles takes the symmetric form: row block rb walks
            // the column tiles from the one holding its own diagonal block
            // (rb / 2) to the end, in parts of ept tiles; the rows of the
            // blocks above the diagonal get their candidates as columns.
            P.sym = sym_ok && P.q0 == 0 && P.q1 == P.spec.n && P.col_tiles >= 2;
            if (P.sym) {
                uint64_t tiles = 0;
                for (uint32_t rb = 0; rb < P.row_blocks; ++rb) tiles += P.col_tiles - rb / 2;
                P.ept = (uint32_t)std::max<uint64_t>(4, (tiles + 4ull * G - 1) / (4ull * G));
                P.ept = std::max<uint32_t>(P.ept, (P.col_tiles + 6) / 7);  // at most 7 parts: 30 lists
                Gp.any_sym = true;
            } else {
                P.ept = P.part_tiles;
            }
        }
        // Candidate lists per row: SC_FULL_LISTS per column part (one per
        // epilogue segment of the emission pass), and for a symmetric job the
        // column list, which takes two lists' room.  The cap of a list grows
        // with the columns it covers.
        for (uint32_t j : Gp.jobs) {
            JobPlan &P = B.jobs[j];
            const uint32_t eparts = (P.col_tiles + P.ept - 1) / P.ept;
            const uint32_t per_part = (uint32_t)SC_FULL_LISTS;
            P.elists = per_part * eparts + (P.sym ? 2u : 0u);
            const double per_list = (double)P.spec.n / ((double)per_part * eparts);
            const double expect = 1.5 * P.spec.k * (2.0 + std::log(std::fmax(1.0, per_list / P.spec.k)));
            P.cap = std::min<uint32_t>(std::max<uint32_t>(pow2ceil((uint32_t)expect), 128), 4096);
            // an escalation copy runs only where the coarse screen kept most of
            // the dataset, and its band is about 2^-16 of the norms: the
            // smallest lists suffice (an overflowing row takes the exact path)
            if (P.clone_of >= 0) P.cap = 128;
            P.eslot0 = Gp.elists;
            Gp.elists += P.spec.n * (uint64_t)P.elists;
            P.cand0 = Gp.cand;
            Gp.cand += P.spec.n * (uint64_t)P.elists * P.cap;
        }
        // The emission pass takes the 2-SM form (a cluster of two CTAs per
        // block of 256 rows, each loading half of every column tile) when
        // every job's K slices fit the resident A block and the autotuner
        // table prefers it for every job.
        Gp.pair = !Gp.pair_vetoed && Gp.kpmax / Gp.kslice <= SC_ARES_STAGES;
        // emission units of the group: (job slot | sym, row block (2-SM form:
        // block of 256 rows), first tile, end tile | part); a symmetric unit
        // starts at the tile holding its diagonal block
        const uint32_t ubm = Gp.pair ? 2 * SC_BM : SC_BM;
        for (uint32_t gj = 0; gj < Gp.jobs.size(); ++gj) {
            const JobPlan &P = B.jobs[Gp.jobs[gj]];
            const uint32_t ub0 = P.q0 / ubm, ub1 = (P.q1 + ubm - 1) / ubm;
            for (uint32_t rb = ub0; rb < ub1; ++rb) {
                const uint32_t first = P.sym ? rb * ubm / SC_BN : 0u;
                for (uint32_t part = 0, t0 = first; t0 < P.col_tiles; ++part, t0 += P.ept) {
                    const uint32_t t1 = std::min<uint32_t>(P.col_tiles, t0 + P.ept);
                    Gp.eunits.push_back(make_uint4(gj | (P.sym ? 0x80000000u : 0u), rb, t0, t1 | (part << 24)));
                }
            }
        }
        // symmetric units differ in size: the largest first, so the
        // persistent CTAs' static round-robin finishes together
        if (Gp.any_sym)
            std::stable_sort(Gp.eunits.begin(), Gp.eunits.end(), [](const uint4 &a, const uint4 &b) {
                return (a.w & 0xffffffu) - a.z > (b.w & 0xffffffu) - b.z;
            });
        // CTAs of the emission pass (the 2-SM form runs two per unit, at most
        // one per SM): the column-side stages are per CTA
        const uint64_t eunits_n = Gp.eunits.size();
        Gp.egrid = (uint32_t)std::min<uint64_t>(Gp.pair ? 2 * eunits_n : eunits_n, G);
        if (Gp.any_sym) {
            // column-side candidates staged per epilogue warp of every CTA
            // (SC_STAGE_SLOTS stages per CTA): room for half of every sym
            // row's expected list share (a full stage sends the affected
            // rows to the exact path, it never loses a candidate silently)
            uint64_t want = 0;
            for (uint32_t j : Gp.jobs)
                if (B.jobs[j].sym) want += B.jobs[j].spec.n * (uint64_t)B.jobs[j].cap / 2;
            const uint64_t slots = (uint64_t)Gp.egrid * SC_STAGE_SLOTS;
            Gp.stage_cap = (uint32_t)std::min<uint64_t>(0x7fffffffull, (want + slots - 1) / slots + 512);
        }
    }

    // work tables of the exact path and of the screened fallback
    for (uint32_t j = 0; j < njobs; ++j) {
        const JobPlan &P = B.jobs[j];
        const int m = P.spec.metric;
        if (P.path == HM_PATH_PLAIN) {
            const uint32_t g_end = (P.q1 + PL_BM - 1) / PL_BM;
            for (uint32_t gi = P.q0 / PL_BM; gi < g_end; ++gi)
                for (uint32_t sp = 0; sp < P.splits; ++sp) B.items[m].push_back(make_uint2(j, gi << 6 | sp));
            B.kpl_plain[m] = std::max<uint32_t>(B.kpl_plain[m], (uint32_t)kpl_for_k(P.spec.k));
        } else if (P.clone_of < 0) {
            // (an escalation copy's fallback rows are the original's: same
            // points, outputs and row list)
            B.fb_jobs[m].push_back(j);
            B.kpl_fb[m] = std::max<uint32_t>(B.kpl_fb[m], (uint32_t)kpl_for_k(P.spec.k));
        }
    }
    for (int m = 0; m < 3; ++m)
        if (!B.fb_jobs[m].empty())
            B.fb_per_job[m] = std::max<uint32_t>(
                1, std::min<uint32_t>(64, (uint32_t)((2 * G + B.fb_jobs[m].size() - 1) / B.fb_jobs[m].size())));
    // prep blocks: about one block per 2048 elements of a job, at most 2048
    B.job_blocks.assign(njobs + 1, 0);
    for (uint32_t j = 0; j < njobs; ++j) {
        const JobPlan &P = B.jobs[j];
        const uint64_t work = std::max<uint64_t>(P.spec.n * P.spec.d, (uint64_t)P.n_pad * P.ldd);
        const uint32_t b = (uint32_t)std::min<uint64_t>(2048, std::max<uint64_t>(1, (work + 2047) / 2048));
        B.job_blocks[j + 1] = B.job_blocks[j] + b;
    }

    // ---------------------------------------------------------- layout
    size_t off = 0;
    auto take = [&](size_t bytes) {
        const size_t where = off;
        off = align256(off + std::max<size_t>(bytes, 1));
        return where;
    };
    // tables (written by bind as one blob; packed at 16-byte alignment so a
    // single job's tables fit in one kernel's parameters)
    B.off_tables = off;
    auto pack = [&](size_t bytes) {
        const size_t where = off;
        off = round_up(off + bytes, 16);
        return where;
    };
    B.off_jobs = pack(sizeof(JobDev) * njobs);
    B.off_row_starts = pack(sizeof(uint32_t) * (njobs + 1));
    B.off_job_blocks = pack(sizeof(uint32_t) * (njobs + 1));
    for (int m = 0; m < 3; ++m) {
        B.off_items[m] = pack(sizeof(uint2) * B.items[m].size());
        B.off_fb[m] = pack(sizeof(uint32_t) * B.fb_jobs[m].size());
    }
    for (int g = 0; g < 3; ++g) {
        GroupPlan &Gp = B.groups[g];
        if (Gp.jobs.empty()) continue;
        Gp.off_gdev = pack(sizeof(GroupDev));
        Gp.off_job_ids = pack(sizeof(uint32_t) * Gp.jobs.size());
        Gp.off_row_starts = pack(sizeof(uint32_t) * (Gp.jobs.size() + 1));
        Gp.off_unit_starts = pack(sizeof(uint32_t) * (Gp.jobs.size() + 1));
        Gp.off_eunits = pack(sizeof(uint4) * Gp.eunits.size());
    }
    B.tables_used = off - B.off_tables;
    off = align256(off);
    B.tables_bytes = off - B.off_tables;
    // device-written
    B.off_counters = take(sizeof(JobCounters) * njobs);
    for (uint32_t j = 0; j < njobs; ++j) {
        JobPlan &P = B.jobs[j];
        const uint64_t n = P.spec.n;
        if (P.clone_of >= 0) {
            // an escalation copy shares its original's norms, binary64 rows
            // and overflow list (only one of the two reaches them)
            const JobPlan &O = B.jobs[P.clone_of];
            P.off_x64 = O.off_x64;
            P.off_rnorm = O.off_rnorm;
            P.off_zero_rows = O.off_zero_rows;
            P.off_ovf = O.off_ovf;
            P.off_mu = take((size_t)P.spec.d * sizeof(double));
            P.off_csum = take((size_t)64 * P.spec.d * sizeof(double));
            continue;
        }
        P.off_x64 = take((size_t)P.n_pad * P.ldd * sizeof(double));  // exact path or fallback rows
        P.off_rnorm = take((size_t)P.n_pad * sizeof(double));
        P.off_zero_rows = take(n * sizeof(uint32_t));
        if (P.splits > 1) P.off_partial = take((size_t)P.splits * n * P.spec.k * sizeof(uint64_t));
        if (P.group >= 0) {
            P.off_ovf = take(n * sizeof(uint32_t));
            P.off_mu = take((size_t)P.spec.d * sizeof(double));
            P.off_csum = take((size_t)64 * P.spec.d * sizeof(double));
        }
    }
    for (int g = 0; g < 3; ++g) {
        GroupPlan &Gp = B.groups[g];
        if (Gp.jobs.empty()) continue;
        const size_t rows = Gp.rows;
        Gp.off_opa = take(rows * Gp.kpmax * Gp.elem_bytes);
        Gp.off_opb = Gp.split ? take(rows * Gp.kpmax * Gp.elem_bytes) : Gp.off_opa;
        Gp.off_rowstat = take(rows * sizeof(RowStat));
        Gp.off_rowterm = take(rows * sizeof(float));
        Gp.off_colterm = take((round_up(rows, SC_BN) + SC_BN) * sizeof(float));
        Gp.off_band = take(rows * sizeof(float));
        Gp.off_force = take(rows);
        Gp.off_rowthr = take(rows * sizeof(uint32_t));
        Gp.off_cand = take(Gp.cand * sizeof(unsigned long long));
        Gp.off_cnt = take(Gp.elists * sizeof(uint32_t));
        Gp.off_topk = take(Gp.topk * sizeof(float));
        Gp.off_rowcnt = take(rows * sizeof(uint32_t));
        if (Gp.any_sym) {
            const size_t padded = round_up(rows, SC_BN) + SC_BN;
            Gp.off_ethr = take(padded * sizeof(float));
            Gp.off_evstar = take(padded * sizeof(float));
            const size_t slots = (size_t)Gp.egrid * SC_STAGE_SLOTS;
            Gp.off_stage_row = take(slots * Gp.stage_cap * sizeof(uint32_t));
            Gp.off_stage_key = take(slots * Gp.stage_cap * sizeof(unsigned long long));
            Gp.off_stage_cnt = take(slots * sizeof(uint32_t));
        }
    }
    B.total = off;
    return HM_OK;
}

// --------------------------------------------------------------- binding
// Tables are written by kernels from their parameters (no host memory stays
// referenced).
constexpr uint32_t kParamTable = 3968;  // + the destination pointer: within 4 KB
struct ParamTable {
    uint32_t bytes;
    unsigned char data[kParamTable];
};

__global__ void write_table_kernel(char *dst, const ParamTable t) {
    for (uint32_t i = threadIdx.x; i < t.bytes; i += blockDim.x) dst[i] = (char)t.data[i];
}

template <typename T>
static T *at(char *base, size_t off) {
    return reinterpret_cast<T *>(base + off);
}

static int bind_batch(hm_batch &B, void *d_ws, size_t bytes, cudaStream_t s) {
    if (!d_ws) return set_error(HM_ERR_INVALID, "workspace is NULL");
    if (bytes < B.total)
        return set_error(HM_ERR_INVALID, "workspace of %zu bytes is below the %zu needed", bytes, B.total);
    if (reinterpret_cast<uintptr_t>(d_ws) % 256)
        return set_error(HM_ERR_INVALID, "workspace must be 256-byte aligned");
    char *ws = static_cast<char *>(d_ws);
    B.ws = ws;
    if (B.graph) {
        cudaGraphExecDestroy(B.graph);
        B.graph = nullptr;
    }
    const uint32_t njobs = (uint32_t)B.jobs.size();
    B.table.assign(B.tables_bytes, 0);
    char *host = B.table.data() - B.off_tables;  // host image addressed like the workspace

    std::vector<uint32_t> row_starts(njobs + 1, 0);
    for (uint32_t j = 0; j < njobs; ++j) {
        const JobPlan &P = B.jobs[j];
        const hm_job &s = P.spec;
        JobDev J{};
        J.n = (uint32_t)s.n;
        J.d = s.d;
        J.k = s.k;
        J.metric = (uint32_t)s.metric;
        J.path = (uint32_t)P.path;
        J.arow0 = P.arow0;
        J.q0 = P.q0;
        J.q1 = P.q1;
        J.rb0 = P.rb0;
        J.x = s.data;
        // outputs hold rows [q0, q1): kernels address them as row * k
        J.idx = reinterpret_cast<uint32_t *>(reinterpret_cast<uintptr_t>(s.idx_out) -
                                             (uintptr_t)P.q0 * s.k * sizeof(uint32_t));
        J.dist = reinterpret_cast<float *>(reinterpret_cast<uintptr_t>(s.dist_out) -
                                           (uintptr_t)P.q0 * s.k * sizeof(float));
        J.sigma = (s.sigma_out && s.rho_out) ? s.sigma_out : nullptr;
        J.rho = (s.sigma_out && s.rho_out) ? s.rho_out : nullptr;
        J.x64 = at<double>(ws, P.off_x64);
        J.rnorm = at<double>(ws, P.off_rnorm);
        J.ldd = P.ldd;
        J.n_pad = P.n_pad;
        J.splits = P.splits;
        J.split_cols = P.split_cols;
        J.partial = P.splits > 1 ? at<uint64_t>(ws, P.off_partial) : nullptr;
        J.target = std::log2((double)s.k);  // src/smooth_knn.rs:25 (platform log2)
        J.zero_rows = at<uint32_t>(ws, P.off_zero_rows);
        J.group = P.group < 0 ? 0u : (uint32_t)P.group;
        J.row0 = P.row0;
        J.unit0 = P.unit0;
        J.kp1 = P.kp1;
        J.k_stages = P.k_stages;
        J.row_blocks = P.row_blocks;
        J.col_tiles = P.col_tiles;
        J.parts = P.parts;
        J.part_tiles = P.part_tiles;
        J.seed_tiles = P.seed_tiles;
        J.cap = P.cap;
        J.slot0 = P.slot0;
        J.tlists = P.tlists;
        J.cand0 = P.cand0;
        J.topk0 = P.topk0;
        J.elists = P.elists;
        J.sym = P.sym ? 1u : 0u;
        J.eslot0 = P.eslot0;
        J.scale = s.metric == HM_METRIC_EUCLIDEAN ? 2.0f : 1.0f;
        J.mu = P.group >= 0 ? at<double>(ws, P.off_mu) : nullptr;
        J.csum = P.group >= 0 ? at<double>(ws, P.off_csum) : nullptr;
        J.ovf_list = P.group >= 0 ? at<uint32_t>(ws, P.off_ovf) : nullptr;
        J.cnt = at<JobCounters>(ws, B.off_counters) + j;
        J.out = J.cnt;
        if (P.clone >= 0) {
            J.gate = &J.cnt->escalate;
            J.gate_on = 0;
            J.escalation = 1;
        } else if (P.clone_of >= 0) {
            J.out = at<JobCounters>(ws, B.off_counters) + P.clone_of;
            J.gate = &J.out->escalate;
            J.gate_on = 1;
        }
        at<JobDev>(host, B.off_jobs)[j] = J;
        row_starts[j + 1] = row_starts[j] + J.n;
    }
    memcpy(host + B.off_row_starts, row_starts.data(), sizeof(uint32_t) * (njobs + 1));
    memcpy(host + B.off_job_blocks, B.job_blocks.data(), sizeof(uint32_t) * (njobs + 1));
    for (int m = 0; m < 3; ++m) {
        if (!B.items[m].empty())
            memcpy(host + B.off_items[m], B.items[m].data(), sizeof(uint2) * B.items[m].size());
        if (!B.fb_jobs[m].empty())
            memcpy(host + B.off_fb[m], B.fb_jobs[m].data(), sizeof(uint32_t) * B.fb_jobs[m].size());
    }
    for (int g = 0; g < 3; ++g) {
        GroupPlan &Gp = B.groups[g];
        if (Gp.jobs.empty()) continue;
        const uint32_t gj = (uint32_t)Gp.jobs.size();
        std::vector<uint32_t> rs(gj + 1), us(gj + 1);
        for (uint32_t i = 0; i < gj; ++i) {
            const JobPlan &P = B.jobs[Gp.jobs[i]];
            rs[i] = P.row0;
            us[i] = P.unit0;
        }
        rs[gj] = Gp.rows;
        us[gj] = Gp.units;
        memcpy(host + Gp.off_job_ids, Gp.jobs.data(), sizeof(uint32_t) * gj);
        memcpy(host + Gp.off_row_starts, rs.data(), sizeof(uint32_t) * (gj + 1));
        memcpy(host + Gp.off_unit_starts, us.data(), sizeof(uint32_t) * (gj + 1));
        if (!Gp.eunits.empty())
            memcpy(host + Gp.off_eunits, Gp.eunits.data(), sizeof(uint4) * Gp.eunits.size());
        GroupDev D{};
        D.rows = Gp.rows;
        D.njobs = gj;
        D.units = Gp.units;
        D.kind = (uint32_t)Gp.kind;
        D.split = Gp.split ? 1u : 0u;
        D.elem_bytes = Gp.elem_bytes;
        D.kslice = Gp.kslice;
        D.kpmax = Gp.kpmax;
        D.job_ids = at<uint32_t>(ws, Gp.off_job_ids);
        D.row_starts = at<uint32_t>(ws, Gp.off_row_starts);
        D.unit_starts = at<uint32_t>(ws, Gp.off_unit_starts);
        D.opa = ws + Gp.off_opa;
        D.opb = ws + Gp.off_opb;
        D.rowstat = at<RowStat>(ws, Gp.off_rowstat);
        D.rowterm = at<float>(ws, Gp.off_rowterm);
        D.colterm = at<float>(ws, Gp.off_colterm);
        D.band = at<float>(ws, Gp.off_band);
        D.force = at<uint8_t>(ws, Gp.off_force);
        D.rowthr = at<uint32_t>(ws, Gp.off_rowthr);
        D.cand = at<unsigned long long>(ws, Gp.off_cand);
        D.cand_cnt = at<uint32_t>(ws, Gp.off_cnt);
        D.topk = at<float>(ws, Gp.off_topk);
        D.row_cnt = at<uint32_t>(ws, Gp.off_rowcnt);
        D.eunits = at<uint4>(ws, Gp.off_eunits);
        D.neunits = (uint32_t)Gp.eunits.size();
        D.pair = Gp.pair ? 1u : 0u;
        for (uint32_t j : Gp.jobs) {
            const bool short_rows = B.jobs[j].kp1 <= operand_short_k1();
            D.any_short_rows |= short_rows ? 1u : 0u;
            D.any_long_rows |= short_rows ? 0u : 1u;
        }
        if (Gp.any_sym) {
            D.ethr = at<float>(ws, Gp.off_ethr);
            D.evstar = at<float>(ws, Gp.off_evstar);
            D.stage_row = at<uint32_t>(ws, Gp.off_stage_row);
            D.stage_key = at<unsigned long long>(ws, Gp.off_stage_key);
            D.stage_cnt = at<uint32_t>(ws, Gp.off_stage_cnt);
            D.stage_cap = Gp.stage_cap;
        }
        Gp.host = D;
        memcpy(host + Gp.off_gdev, &D, sizeof D);
        HM_TRY(make_operand_map(&Gp.ta, D.opa, Gp.rows, Gp.kpmax, Gp.elem_bytes, Gp.kslice, SC_BM));
        HM_TRY(make_operand_map(&Gp.tb, D.opb, Gp.rows, Gp.kpmax, Gp.elem_bytes, Gp.kslice, SC_BN));
        if (Gp.pair)
            HM_TRY(make_operand_map(&Gp.tb_half, D.opb, Gp.rows, Gp.kpmax, Gp.elem_bytes, Gp.kslice, SC_BM));
    }

    // written by kernels from their parameters, 3968 bytes per launch: no
    // host memory stays referenced by the stream or by a captured graph
    char *dst = ws + B.off_tables;
    const size_t used = B.tables_used;  // tables_bytes adds the 256-byte padding
    for (size_t o = 0; o < used; o += kParamTable) {
        ParamTable t;
        t.bytes = (uint32_t)std::min<size_t>(kParamTable, used - o);
        memcpy(t.data, B.table.data() + o, t.bytes);
        write_table_kernel<<<1, 256, 0, s>>>(dst + o, t);
        HM_CUDA_TRY(cudaGetLastError());
        count_launch();
    }
    return HM_OK;
}

// ------------------------------------------------------------------- run
static int run_batch(hm_batch &B, cudaStream_t s) {
    if (!B.ws) return set_error(HM_ERR_INVALID, "batch has no workspace bound");
    char *ws = B.ws;
    const uint32_t njobs = (uint32_t)B.jobs.size();
    const JobDev *jobs = at<JobDev>(ws, B.off_jobs);
    const uint32_t *row_starts = at<uint32_t>(ws, B.off_row_starts);
    const uint32_t *job_blocks = at<uint32_t>(ws, B.off_job_blocks);
    const uint32_t blocks = B.job_blocks.back();

    HM_TRY(launch_prep_jobs(jobs, njobs, job_blocks, blocks, PREP_CHECK_AND_NORMS, s, row_starts, B.all_rows));
    if (B.any_plain) HM_TRY(launch_prep_jobs(jobs, njobs, job_blocks, blocks, PREP_X64_EXACT, s));
    for (int m = 0; m < 3; ++m) {
        if (B.items[m].empty()) continue;
        PlainWork w{};
        w.jobs = jobs;
        w.njobs = njobs;
        w.items = at<uint2>(ws, B.off_items[m]);
        w.nitems = (uint32_t)B.items[m].size();
        w.kpl = B.kpl_plain[m];
        HM_TRY(launch_plain(w, m, s));
    }
    for (int g = 0; g < 3; ++g) {
        GroupPlan &Gp = B.groups[g];
        if (Gp.jobs.empty()) continue;
        const GroupDev *Gd = at<GroupDev>(ws, Gp.off_gdev);
        HM_TRY(launch_screen_prep(jobs, Gp.host, Gd, s));
        HM_TRY(launch_screen_band(jobs, Gp.host, Gd, s));
        HM_TRY(launch_screen_gemm(jobs, Gp.host, Gd, Gp.kp, Gp.ta, Gp.tb, debug_dump_pointer(), 0, s));
        HM_TRY(launch_screen_threshold(jobs, Gp.host, Gd, Gp.kpl, s));
        if (Gp.any_escalation) HM_TRY(launch_escalation(jobs, Gp.host, Gd, s));
        // lists no unit writes (parts a row block does not have) and the
        // column lists the scatter fills start empty
        HM_CUDA_TRY(cudaMemsetAsync(Gp.host.cand_cnt, 0, Gp.elists * sizeof(uint32_t), s));
        // (stages of CTAs the emission pass does not launch stay empty)
        if (Gp.any_sym)
            HM_CUDA_TRY(cudaMemsetAsync(Gp.host.stage_cnt, 0, (size_t)Gp.egrid * SC_STAGE_SLOTS * sizeof(uint32_t), s));
        if (Gp.any_sym) HM_TRY(launch_emit_limits(jobs, Gp.host, Gd, s));
        HM_TRY(launch_screen_gemm(jobs, Gp.host, Gd, Gp.kp, Gp.ta, Gp.pair ? Gp.tb_half : Gp.tb, nullptr,
                                  Gp.any_sym ? 2 : 1, s));
        if (Gp.any_sym) HM_TRY(launch_column_scatter(jobs, Gp.host, Gd, Gp.egrid * SC_STAGE_SLOTS, s));
        HM_TRY(launch_rerank(jobs, Gp.host, Gd, Gp.kpl, Gp.dmax, Gp.metric_mask, s));
    }
    if (B.any_screen) {
        // exact plain path for the rows the screen could not settle (binary64
        // copies are built only for jobs that have such rows)
        HM_TRY(launch_prep_jobs(jobs, njobs, job_blocks, blocks, PREP_X64_FALLBACK, s));
        for (int m = 0; m < 3; ++m) {
            if (B.fb_jobs[m].empty()) continue;
            PlainWork w{};
            w.jobs = jobs;
            w.njobs = njobs;
            w.kpl = B.kpl_fb[m];
            w.fallback = 1;
            w.per_job = B.fb_per_job[m];
            w.fb_jobs = at<uint32_t>(ws, B.off_fb[m]);
            w.fb_njobs = (uint32_t)B.fb_jobs[m].size();
            HM_TRY(launch_plain(w, m, s));
        }
    }
    if (B.any_split)
        HM_TRY(launch_merge(jobs, njobs, njobs > 1 ? row_starts : nullptr, B.all_rows, B.kpl_all, s));
    if (B.any_smooth) {
        HM_TRY(launch_smooth(jobs, njobs, njobs > 1 ? row_starts : nullptr, B.all_rows, B.kmax, s));
        HM_TRY(launch_mean_all_floor(jobs, njobs, s));
    }
    return HM_OK;
}

static void stats_from_counters(const hm_batch &B, uint32_t j, const JobCounters &c, hm_stats *st) {
    memset(st, 0, sizeof *st);
    // an escalated job reports its split-BF16 copy's path (the copy's counts
    // went to the job's own counters)
    const JobPlan &P = (c.escalate && B.jobs[j].clone >= 0) ? B.jobs[B.jobs[j].clone] : B.jobs[j];
    st->path_used = P.path;
    st->col_splits = P.splits;
    st->zero_rho_rows = c.zero_count;
    if (P.path != HM_PATH_PLAIN) {
        st->candidate_cap = P.cap;
        st->candidates_total = c.candidates;
        st->candidates_max_row = c.max_row;
        st->overflow_rows = c.ovf_count;
        st->candidates_emitted = c.emitted;
        float band;
        memcpy(&band, &c.band_max_bits, sizeof band);
        st->screen_band = band;
    }
}

static int check_counters(const JobCounters &c) {
    if (c.nonfinite_min != 0xffffffffu)
        return set_error(HM_ERR_INVALID, "data contains a non-finite value at index %u", c.nonfinite_min);
    if (c.error_code)
        return set_error(HM_ERR_TIMEOUT, "screen kernel gave up waiting (code %u)", c.error_code);
    return HM_OK;
}

// Counters of a finished single-job call whose workspace is `ws`, read after
// the work queued on `s` (no allocation: the copy lands in a host struct).
int single_job_stats(const void *ws, uint64_t n, uint32_t d, uint32_t k, int metric, int path,
                     cudaStream_t s, hm_stats *stats) {
    hm_batch B;
    hm_job spec{};
    spec.n = n;
    spec.d = d;
    spec.k = k;
    spec.metric = metric;
    spec.path = path;
    HM_TRY(plan_batch(&spec, 1, B));
    JobCounters c{};
    HM_CUDA_TRY(cudaMemcpyAsync(&c, static_cast<const char *>(ws) + B.off_counters, sizeof c,
                                cudaMemcpyDeviceToHost, s));
    HM_CUDA_TRY(cudaStreamSynchronize(s));
    hm_stats local;
    stats_from_counters(B, 0, c, stats ? stats : &local);
    return check_counters(c);
}

// batch internals for the request loop (serve.cu)
size_t batch_counters_offset(const hm_batch *B) { return B->off_counters; }

int batch_job_result(const hm_batch *B, uint32_t job, const JobCounters &c, hm_stats *st) {
    stats_from_counters(*B, job, c, st);
    return check_counters(c);
}

// ---------------------------------------------- per-thread device context
struct ThreadCtx {
    int device = -1;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
};
static thread_local ThreadCtx g_ctx;

static int thread_ctx(ThreadCtx *&out) {
    int dev = 0;
    HM_CUDA_TRY(cudaGetDevice(&dev));
    if (g_ctx.device != dev || !g_ctx.stream) {
        HM_CUDA_TRY(cudaStreamCreateWithFlags(&g_ctx.stream, cudaStreamNonBlocking));
        HM_CUDA_TRY(cudaEventCreate(&g_ctx.ev0));
        HM_CUDA_TRY(cudaEventCreate(&g_ctx.ev1));
        // keep freed stream-ordered allocations cached in the device pool
        cudaMemPool_t pool;
        if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
            uint64_t threshold = ~0ull;
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &threshold);
        }
        g_ctx.device = dev;
    }
    out = &g_ctx;
    return HM_OK;
}

// RAII list of stream-ordered allocations, freed on every exit path.
struct Allocs {
    cudaStream_t s;
    void *p[8] = {};
    int count = 0;
    explicit Allocs(cudaStream_t st) : s(st) {}
    int get(void **out, size_t bytes) {
        cudaError_t e = cudaMallocAsync(out, bytes ? bytes : 256, s);
        if (e != cudaSuccess)
            return set_error(e == cudaErrorMemoryAllocation ? HM_ERR_OOM : HM_ERR_CUDA,
                             "cudaMallocAsync(%zu): %s", bytes, cudaGetErrorString(e));
        p[count++] = *out;
        return HM_OK;
    }
    ~Allocs() {
        for (int i = 0; i < count; ++i) cudaFreeAsync(p[i], s);
        cudaStreamSynchronize(s);
    }
};

static hm_job one_job(const float *data, uint64_t n, uint32_t d, uint32_t k, int metric, int path,
                      uint32_t *idx, float *dist, float *sigma, float *rho) {
    hm_job j{};
    j.data = data;
    j.n = n;
    j.d = d;
    j.k = k;
    j.metric = metric;
    j.path = path;
    j.idx_out = idx;
    j.dist_out = dist;
    j.sigma_out = sigma;
    j.rho_out = rho;
    return j;
}

// Replaces a planned job's buffers (the plan only depended on which were
// present) and those of its escalation copy, which shares the points and the
// kNN outputs but never the smooth-kNN ones.
static void set_job_buffers(hm_batch &B, uint32_t j, const hm_job &spec) {
    B.jobs[j].spec = spec;
    const int c = B.jobs[j].clone;
    if (c < 0) return;
    hm_job &cs = B.jobs[c].spec;
    cs.data = spec.data;
    cs.idx_out = spec.idx_out;
    cs.dist_out = spec.dist_out;
}

static int host_pipeline(const float *data, uint64_t n, uint32_t d, uint32_t k, int metric,
                         int path, uint32_t *idx_out, float *dist_out, float *sigma_out,
                         float *rho_out, hm_stats *stats) {
    if (!data) return set_error(HM_ERR_INVALID, "data is NULL");
    hm_batch B;
    // planned with the host outputs standing in for the device buffers (only
    // their presence matters to the plan)
    hm_job spec = one_job(data, n, d, k, metric, path, idx_out, dist_out, sigma_out, rho_out);
    HM_TRY(plan_batch(&spec, 1, B));
    if (!idx_out || !dist_out) return set_error(HM_ERR_INVALID, "output pointer is NULL");
    ThreadCtx *ctx;
    HM_TRY(thread_ctx(ctx));
    cudaStream_t s = ctx->stream;
    const bool smooth = sigma_out && rho_out;
    JobCounters cnt{};
    {
        Allocs A(s);
        void *d_data, *d_idx, *d_dist, *d_sigma = nullptr, *d_rho = nullptr, *ws;
        HM_TRY(A.get(&d_data, n * d * sizeof(float)));
        HM_TRY(A.get(&d_idx, n * k * sizeof(uint32_t)));
        HM_TRY(A.get(&d_dist, n * k * sizeof(float)));
        if (smooth) {
            HM_TRY(A.get(&d_sigma, n * sizeof(float)));
            HM_TRY(A.get(&d_rho, n * sizeof(float)));
        }
        HM_TRY(A.get(&ws, B.total));
        set_job_buffers(B, 0, one_job(static_cast<float *>(d_data), n, d, k, metric, path,
                                      static_cast<uint32_t *>(d_idx), static_cast<float *>(d_dist),
                                      static_cast<float *>(d_sigma), static_cast<float *>(d_rho)));
        HM_CUDA_TRY(cudaMemcpyAsync(d_data, data, n * d * sizeof(float), cudaMemcpyHostToDevice, s));
        HM_CUDA_TRY(cudaEventRecord(ctx->ev0, s));
        HM_TRY(bind_batch(B, ws, B.total, s));
        HM_TRY(run_batch(B, s));
        HM_CUDA_TRY(cudaEventRecord(ctx->ev1, s));
        HM_CUDA_TRY(cudaMemcpyAsync(idx_out, d_idx, n * k * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
        HM_CUDA_TRY(cudaMemcpyAsync(dist_out, d_dist, n * k * sizeof(float), cudaMemcpyDeviceToHost, s));
        if (smooth) {
            HM_CUDA_TRY(cudaMemcpyAsync(sigma_out, d_sigma, n * sizeof(float), cudaMemcpyDeviceToHost, s));
            HM_CUDA_TRY(cudaMemcpyAsync(rho_out, d_rho, n * sizeof(float), cudaMemcpyDeviceToHost, s));
        }
        HM_CUDA_TRY(cudaMemcpyAsync(&cnt, static_cast<char *>(ws) + B.off_counters, sizeof cnt,
                                    cudaMemcpyDeviceToHost, s));
        HM_CUDA_TRY(cudaStreamSynchronize(s));
        if (stats) {
            float ms = 0.f;
            cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
            stats_from_counters(B, 0, cnt, stats);
            stats->device_ms = ms;
        }
    }
    return check_counters(cnt);
}

}  // namespace hm

using namespace hm;

extern "C" {

int hm_abi_version(void) { return HM_ABI_VERSION; }

const char *hm_last_error(void) { return g_last_error.c_str(); }

int hm_knn(const float *data, uint64_t n, uint32_t d, uint32_t k, int metric, int path,
           uint32_t *idx_out, float *dist_out, hm_stats *stats) {
    clear_error();
    return host_pipeline(data, n, d, k, metric, path, idx_out, dist_out, nullptr, nullptr, stats);
}

int hm_knn_smooth(const float *data, uint64_t n, uint32_t d, uint32_t k, int metric, int path,
                  uint32_t *idx_out, float *dist_out, float *sigma_out, float *rho_out,
                  hm_stats *stats) {
    clear_error();
    if (!sigma_out || !rho_out) return set_error(HM_ERR_INVALID, "sigma/rho output is NULL");
    return host_pipeline(data, n, d, k, metric, path, idx_out, dist_out, sigma_out, rho_out, stats);
}

size_t hm_workspace_bytes(uint64_t n, uint32_t d, uint32_t k, int metric, int path) {
    clear_error();
    hm_batch B;
    hm_job spec = one_job(nullptr, n, d, k, metric, path, nullptr, nullptr, nullptr, nullptr);
    if (plan_batch(&spec, 1, B) != HM_OK) return 0;
    return B.total;
}

int hm_knn_smooth_device(const float *d_data, uint64_t n, uint32_t d, uint32_t k, int metric,
                         int path, uint32_t *d_idx, float *d_dist, float *d_sigma, float *d_rho,
                         void *d_workspace, size_t workspace_bytes, void *stream,
                         hm_stats *stats) {
    clear_error();
    if (!d_data) return set_error(HM_ERR_INVALID, "data is NULL");
    hm_batch B;
    hm_job spec = one_job(d_data, n, d, k, metric, path, d_idx, d_dist, d_sigma, d_rho);
    HM_TRY(plan_batch(&spec, 1, B));
    if (!d_idx || !d_dist || !d_workspace) return set_error(HM_ERR_INVALID, "NULL pointer argument");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    HM_TRY(bind_batch(B, d_workspace, workspace_bytes, s));
    HM_TRY(run_batch(B, s));
    if (stats) {
        memset(stats, 0, sizeof *stats);
        stats->path_used = B.jobs[0].path;
        stats->col_splits = B.jobs[0].splits;
        stats->candidate_cap = B.jobs[0].path == HM_PATH_PLAIN ? 0 : B.jobs[0].cap;
    }
    return HM_OK;
}

int hm_stats_from_workspace(const void *d_workspace, uint64_t n, uint32_t d, uint32_t k,
                            int metric, int path, hm_stats *stats) {
    clear_error();
    if (!d_workspace || !stats) return set_error(HM_ERR_INVALID, "NULL pointer argument");
    hm_batch B;
    hm_job spec = one_job(nullptr, n, d, k, metric, path, nullptr, nullptr, nullptr, nullptr);
    HM_TRY(plan_batch(&spec, 1, B));
    JobCounters c{};
    HM_CUDA_TRY(cudaMemcpy(&c, static_cast<const char *>(d_workspace) + B.off_counters, sizeof c,
                           cudaMemcpyDeviceToHost));
    stats_from_counters(B, 0, c, stats);
    return check_counters(c);
}

// A row shard: query rows [row_begin, row_end) against all n points.
size_t hm_knn_rows_workspace_bytes(uint64_t n, uint32_t d, uint32_t k, int metric, int path,
                                   uint64_t row_begin, uint64_t row_end) {
    clear_error();
    hm_batch B;
    hm_job spec = one_job(nullptr, n, d, k, metric, path, nullptr, nullptr, nullptr, nullptr);
    const uint64_t r[2] = {row_begin, row_end};
    if (plan_batch(&spec, 1, B, r) != HM_OK) return 0;
    return B.total;
}

int hm_knn_rows_device(const float *d_data, uint64_t n, uint32_t d, uint32_t k, int metric, int path,
                       uint64_t row_begin, uint64_t row_end, uint32_t *d_idx, float *d_dist,
                       void *d_workspace, size_t workspace_bytes, void *stream, hm_stats *stats) {
    clear_error();
    if (!d_data) return set_error(HM_ERR_INVALID, "data is NULL");
    hm_batch B;
    hm_job spec = one_job(d_data, n, d, k, metric, path, d_idx, d_dist, nullptr, nullptr);
    const uint64_t r[2] = {row_begin, row_end};
    HM_TRY(plan_batch(&spec, 1, B, r));
    if (!d_idx || !d_dist || !d_workspace) return set_error(HM_ERR_INVALID, "NULL pointer argument");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    HM_TRY(bind_batch(B, d_workspace, workspace_bytes, s));
    HM_TRY(run_batch(B, s));
    if (stats) {
        memset(stats, 0, sizeof *stats);
        stats->path_used = B.jobs[0].path;
        stats->col_splits = B.jobs[0].splits;
        stats->candidate_cap = B.jobs[0].path == HM_PATH_PLAIN ? 0 : B.jobs[0].cap;
    }
    return HM_OK;
}

int hm_knn_rows_stats(const void *d_workspace, uint64_t n, uint32_t d, uint32_t k, int metric, int path,
                      uint64_t row_begin, uint64_t row_end, hm_stats *stats) {
    clear_error();
    if (!d_workspace || !stats) return set_error(HM_ERR_INVALID, "NULL pointer argument");
    hm_batch B;
    hm_job spec = one_job(nullptr, n, d, k, metric, path, nullptr, nullptr, nullptr, nullptr);
    const uint64_t r[2] = {row_begin, row_end};
    HM_TRY(plan_batch(&spec, 1, B, r));
    JobCounters c{};
    HM_CUDA_TRY(cudaMemcpy(&c, static_cast<const char *>(d_workspace) + B.off_counters, sizeof c,
                           cudaMemcpyDeviceToHost));
    stats_from_counters(B, 0, c, stats);
    return check_counters(c);
}

// smooth-kNN alone: a job whose distances are given (no kNN stage)
size_t hm_smooth_workspace_bytes(uint64_t n) {
    return align256(sizeof(JobDev)) + align256(sizeof(JobCounters)) + align256(n * sizeof(uint32_t));
}

__global__ void write_smooth_job_kernel(JobDev *dst, const JobDev j) {
    if (threadIdx.x == 0) {
        *dst = j;
        JobCounters c{};
        c.nonfinite_min = 0xffffffffu;
        *j.cnt = c;
    }
}

int hm_smooth_knn_device(const float *d_dists, uint64_t n, uint32_t k, float *d_sigma,
                         float *d_rho, void *d_workspace, void *stream) {
    clear_error();
    if (!d_dists || !d_sigma || !d_rho || !d_workspace)
        return set_error(HM_ERR_INVALID, "NULL pointer argument");
    if (n == 0 || k == 0) return set_error(HM_ERR_INVALID, "empty distance matrix");
    if (n > 0x7fffffffull) return set_error(HM_ERR_UNSUPPORTED, "n exceeds the supported range");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    char *w = static_cast<char *>(d_workspace);
    JobDev J{};
    J.n = (uint32_t)n;
    J.k = k;
    J.dist = const_cast<float *>(d_dists);
    J.sigma = d_sigma;
    J.rho = d_rho;
    J.target = std::log2((double)k);  // src/smooth_knn.rs:25 (platform log2)
    J.cnt = reinterpret_cast<JobCounters *>(w + align256(sizeof(JobDev)));
    J.out = J.cnt;
    J.zero_rows = reinterpret_cast<uint32_t *>(w + align256(sizeof(JobDev)) + align256(sizeof(JobCounters)));
    JobDev *jd = reinterpret_cast<JobDev *>(w);
    write_smooth_job_kernel<<<1, 32, 0, s>>>(jd, J);
    HM_CUDA_TRY(cudaGetLastError());
    count_launch();
    HM_TRY(launch_smooth(jd, 1, nullptr, (uint32_t)n, k, s));
    HM_TRY(launch_mean_all_floor(jd, 1, s));
    return HM_OK;
}

// smooth-kNN of rows [row_begin, row_end) of an n x k distance matrix: the
// job's rows are addressed from row_begin (arow0 = -row_begin in the kernels'
// unsigned arithmetic) and its outputs through pointers shifted by the same
// amount, while the global-mean floor still averages all n * k distances.
int hm_smooth_knn_rows_device(const float *d_dists, uint64_t n, uint32_t k, uint64_t row_begin,
                              uint64_t row_end, float *d_sigma, float *d_rho, void *d_workspace,
                              void *stream) {
    clear_error();
    if (!d_dists || !d_sigma || !d_rho || !d_workspace)
        return set_error(HM_ERR_INVALID, "NULL pointer argument");
    if (n == 0 || k == 0) return set_error(HM_ERR_INVALID, "empty distance matrix");
    if (n > 0x7fffffffull) return set_error(HM_ERR_UNSUPPORTED, "n exceeds the supported range");
    if (row_begin >= row_end || row_end > n)
        return set_error(HM_ERR_INVALID, "rows [%llu, %llu) outside [0, %llu)", (unsigned long long)row_begin,
                         (unsigned long long)row_end, (unsigned long long)n);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    char *w = static_cast<char *>(d_workspace);
    JobDev J{};
    J.n = (uint32_t)n;
    J.k = k;
    J.arow0 = (uint32_t)(0u - (uint32_t)row_begin);
    J.dist = const_cast<float *>(d_dists);
    J.sigma = d_sigma - row_begin;
    J.rho = d_rho - row_begin;
    J.target = std::log2((double)k);  // src/smooth_knn.rs:25 (platform log2)
    J.cnt = reinterpret_cast<JobCounters *>(w + align256(sizeof(JobDev)));
    J.out = J.cnt;
    J.zero_rows = reinterpret_cast<uint32_t *>(w + align256(sizeof(JobDev)) + align256(sizeof(JobCounters)));
    JobDev *jd = reinterpret_cast<JobDev *>(w);
    write_smooth_job_kernel<<<1, 32, 0, s>>>(jd, J);
    HM_CUDA_TRY(cudaGetLastError());
    count_launch();
    HM_TRY(launch_smooth(jd, 1, nullptr, (uint32_t)(row_end - row_begin), k, s));
    HM_TRY(launch_mean_all_floor(jd, 1, s));
    return HM_OK;
}

int hm_smooth_knn(const float *dists, uint64_t n, uint32_t k, float *sigma_out, float *rho_out) {
    clear_error();
    if (!dists || !sigma_out || !rho_out) return set_error(HM_ERR_INVALID, "NULL pointer argument");
    if (n == 0 || k == 0) return set_error(HM_ERR_INVALID, "empty distance matrix");
    ThreadCtx *ctx;
    HM_TRY(thread_ctx(ctx));
    cudaStream_t s = ctx->stream;
    Allocs A(s);
    void *d_dists, *d_sigma, *d_rho, *ws;
    HM_TRY(A.get(&d_dists, n * k * sizeof(float)));
    HM_TRY(A.get(&d_sigma, n * sizeof(float)));
    HM_TRY(A.get(&d_rho, n * sizeof(float)));
    HM_TRY(A.get(&ws, hm_smooth_workspace_bytes(n)));
    HM_CUDA_TRY(cudaMemcpyAsync(d_dists, dists, n * k * sizeof(float), cudaMemcpyHostToDevice, s));
    HM_TRY(hm_smooth_knn_device(static_cast<float *>(d_dists), n, k, static_cast<float *>(d_sigma),
                                static_cast<float *>(d_rho), ws, s));
    HM_CUDA_TRY(cudaMemcpyAsync(sigma_out, d_sigma, n * sizeof(float), cudaMemcpyDeviceToHost, s));
    HM_CUDA_TRY(cudaMemcpyAsync(rho_out, d_rho, n * sizeof(float), cudaMemcpyDeviceToHost, s));
    HM_CUDA_TRY(cudaStreamSynchronize(s));
    return HM_OK;
}

// ----------------------------------------------------------------- batches
int hm_batch_create(const hm_job *jobs, uint32_t njobs, hm_batch **out) {
    clear_error();
    if (!jobs || !out) return set_error(HM_ERR_INVALID, "NULL pointer argument");
    *out = nullptr;
    for (uint32_t j = 0; j < njobs; ++j) {
        if (!jobs[j].data || !jobs[j].idx_out || !jobs[j].dist_out)
            return set_error(HM_ERR_INVALID, "job %u has a NULL data/output pointer", j);
    }
    hm_batch *B = new (std::nothrow) hm_batch();
    if (!B) return set_error(HM_ERR_OOM, "host allocation failed");
    const int rc = plan_batch(jobs, njobs, *B);
    if (rc != HM_OK) {
        delete B;
        return rc;
    }
    *out = B;
    return HM_OK;
}

void hm_batch_destroy(hm_batch *batch) { delete batch; }

size_t hm_batch_workspace_bytes(const hm_batch *batch) { return batch ? batch->total : 0; }

int hm_batch_bind(hm_batch *batch, void *d_workspace, size_t workspace_bytes, void *stream) {
    clear_error();
    if (!batch) return set_error(HM_ERR_INVALID, "batch is NULL");
    return bind_batch(*batch, d_workspace, workspace_bytes, static_cast<cudaStream_t>(stream));
}

int hm_batch_run(hm_batch *batch, void *stream) {
    clear_error();
    if (!batch) return set_error(HM_ERR_INVALID, "batch is NULL");
    return run_batch(*batch, static_cast<cudaStream_t>(stream));
}

int hm_batch_graph_launch(hm_batch *batch, void *stream) {
    clear_error();
    if (!batch) return set_error(HM_ERR_INVALID, "batch is NULL");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (!batch->graph) {
        // captured on a private stream (the caller's may be the legacy
        // default stream, which cannot be captured); launched on the caller's
        if (!batch->capture) HM_CUDA_TRY(cudaStreamCreateWithFlags(&batch->capture, cudaStreamNonBlocking));
        const bool timing = timing_enabled();
        hm_timing_enable(0);  // no event records inside the graph
        cudaGraph_t g = nullptr;
        HM_CUDA_TRY(cudaStreamBeginCapture(batch->capture, cudaStreamCaptureModeThreadLocal));
        const int rc = run_batch(*batch, batch->capture);
        const cudaError_t e = cudaStreamEndCapture(batch->capture, &g);
        hm_timing_enable(timing ? 1 : 0);
        if (rc != HM_OK) {
            if (g) cudaGraphDestroy(g);
            return rc;
        }
        HM_CUDA_TRY(e);
        const cudaError_t ei = cudaGraphInstantiate(&batch->graph, g, 0);
        cudaGraphDestroy(g);
        HM_CUDA_TRY(ei);
    }
    HM_CUDA_TRY(cudaGraphLaunch(batch->graph, s));
    return HM_OK;
}

int hm_batch_job_stats(const hm_batch *batch, uint32_t job, hm_stats *stats) {
    clear_error();
    if (!batch || !stats || !batch->ws) return set_error(HM_ERR_INVALID, "unbound batch or NULL stats");
    if (job >= batch->user_jobs) return set_error(HM_ERR_INVALID, "job %u out of range", job);
    JobCounters c{};
    HM_CUDA_TRY(cudaMemcpy(&c, batch->ws + batch->off_counters + job * sizeof(JobCounters), sizeof c,
                           cudaMemcpyDeviceToHost));
    stats_from_counters(*batch, job, c, stats);
    return check_counters(c);
}

int hm_batch_job_path(const hm_batch *batch, uint32_t job) {
    if (!batch || job >= batch->user_jobs) return set_error(HM_ERR_INVALID, "job out of range");
    return batch->jobs[job].path;
}

}  // extern "C"
