// autotune.cu -- the autotuner table: which path HM_PATH_AUTO takes and how
// large a column sample the screen's threshold pass uses, per (n, d, k,
// metric).
//
// The table (autotune_table.inc) is generated by holomap_b200/autotune.py from
// measurements on the GPU: at every grid point it holds the fastest of the
// plain path and the three screens (each with 1/4, 1/8 or 1/16 of the columns
// sampled), all of which return the same bytes.  A problem takes the choice of
// the nearest grid point (n by ratio, d by ratio, k by the nearer of the
// measured k), including whether the emission pass takes the symmetric or
// the 2-SM form.  Where no screen applies (manhattan, k > 64, d > 2048) the
// path is plain.  A job planned in a batch of several takes the batch table:
// the same grid measured as batches of jobs of that shape, where the
// screens' fixed costs are shared and small jobs favour them.
#include <cuda_runtime.h>

#include <cmath>

#include "hm_internal.cuh"
#include "autotune_table.inc"

namespace hm {

static thread_local uint32_t g_seed_override = 0;
// emission forms: -1 the table's choice, 0 never, 1 wherever a job can take it
static thread_local int g_symmetric = -1;
static thread_local int g_pair = -1;
static thread_local bool g_escalation = true;

template <size_t N>
static size_t nearest_ratio(const uint32_t (&grid)[N], double v) {
    size_t best = 0;
    double bd = 1e300;
    for (size_t i = 0; i < N; ++i) {
        const double dist = std::fabs(std::log(v / (double)grid[i]));
        if (dist < bd) {
            bd = dist;
            best = i;
        }
    }
    return best;
}

static uint16_t table_entry(uint64_t n, uint32_t d, uint32_t k, int metric, bool batched) {
    const size_t in = nearest_ratio(kTuneN, (double)(n ? n : 1));
    const size_t id = nearest_ratio(kTuneD, (double)(d ? d : 1));
    const size_t ik = nearest_ratio(kTuneK, (double)(k ? k : 1));
    const int m = metric == HM_METRIC_COSINE ? 1 : 0;
    return batched ? kTuneBatch[m][ik][id][in] : kTune[m][ik][id][in];
}

int autotune_choice(uint64_t n, uint32_t d, uint32_t k, int metric, uint32_t *seed_div, bool *symmetric,
                    bool *pair, bool batched) {
    if (metric == HM_METRIC_MANHATTAN || k > 64 || d > 2048) {
        if (seed_div) *seed_div = 8;
        if (symmetric) *symmetric = true;
        if (pair) *pair = true;
        return HM_PATH_PLAIN;
    }
    const uint16_t e = table_entry(n, d, k, metric, batched);
    if (seed_div) *seed_div = g_seed_override ? g_seed_override : (uint32_t)((e >> 8) & 0x7f);
    if (symmetric) *symmetric = g_symmetric < 0 ? (e >> 15) != 0 : g_symmetric != 0;
    if (pair) *pair = g_pair < 0 ? ((e >> 4) & 1) != 0 : g_pair != 0;
    return (int)(e & 0xf);
}

bool tuning_escalation() { return g_escalation; }

}  // namespace hm

using namespace hm;

extern "C" {

int hm_autotune_path(uint64_t n, uint32_t d, uint32_t k, int metric) {
    return autotune_choice(n, d, k, metric, nullptr, nullptr, nullptr, false);
}

int hm_autotune_path_batched(uint64_t n, uint32_t d, uint32_t k, int metric) {
    return autotune_choice(n, d, k, metric, nullptr, nullptr, nullptr, true);
}

int hm_tuning_override(int seed_div) {
    if (seed_div < 0 || seed_div > 64) return set_error(HM_ERR_INVALID, "seed_div %d outside [0, 64]", seed_div);
    g_seed_override = (uint32_t)seed_div;
    return HM_OK;
}

int hm_tuning_symmetric(int mode) {
    if (mode < -1 || mode > 1) return set_error(HM_ERR_INVALID, "symmetric mode %d outside [-1, 1]", mode);
    g_symmetric = mode;
    return HM_OK;
}

int hm_tuning_pair(int mode) {
    if (mode < -1 || mode > 1) return set_error(HM_ERR_INVALID, "pair mode %d outside [-1, 1]", mode);
    g_pair = mode;
    return HM_OK;
}

int hm_tuning_escalation(int on) {
    g_escalation = on != 0;
    return HM_OK;
}

}  // extern "C"
