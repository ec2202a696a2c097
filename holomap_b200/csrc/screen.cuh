// screen.cuh -- the screened distance bulk: a tensor-core similarity screen
// with a proven error band, followed by an exact rerank of the survivors.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

namespace hm {

// Counters the screened path leaves in the workspace (device-written).
struct ScreenCounters {
    unsigned long long candidates;  // candidates reranked exactly, all rows
    uint32_t max_row;               // most candidates kept by one row
    uint32_t overflow_rows;         // rows whose candidates exceeded the cap
    float band_max;                 // widest keep band used (distance units)
    uint32_t error_code;            // nonzero if a bounded wait gave up
};

struct ScreenLayout {
    uint32_t cap = 0;  // candidates kept per row
    size_t total = 0;  // workspace bytes
    size_t off[8] = {};
};

struct ScreenRun {
    const float *data;
    const double *x64;
    const double *rnorm;
    uint32_t n, d, ldd, k;
    int metric, path;
    uint32_t *idx_out;
    float *dist_out;
    ScreenCounters *counters;
};

int screen_plan(uint64_t n, uint32_t d, uint32_t k, int metric, int path, ScreenLayout &L);
int screen_run(const ScreenRun &r, const ScreenLayout &L, char *ws, cudaStream_t s);

}  // namespace hm
