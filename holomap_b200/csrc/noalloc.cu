// noalloc.cu -- kNN + smooth-kNN for callers that cannot allocate device
// memory.
//
// Some callers cannot call cudaMalloc: a plugin running inside a host engine
// that has already reserved the whole card for its own allocator (a raw
// cudaMalloc would fail or fragment that pool), and latency-bound request
// loops that must not call the allocator at all because cudaMalloc/cudaFree
// can block and implicitly synchronise the device.  They still own their
// inputs and outputs; what they cannot provide is the scratch the plain path
// needs (the binary64 copy of the points, per-split partial top-k lists and
// the smooth-kNN bookkeeping).
//
// hm_knn_smooth_noalloc serves them from a fixed scratch array that is part of
// the library image: a file-scope __device__ array of HM_NOALLOC_SCRATCH_BYTES.
// Every GPU that loads this library holds that array until the process exits.
// In host code the array's name is only a host-side stand-in, so its device
// address is looked up once per device with cudaGetSymbolAddress (with that
// device current) on the first call on the device, and then passed to the
// kernels; the first call on a device should therefore come before any
// stream capture.  All calls share the one array and it keeps the last call's
// contents: the pipeline clears what must start at zero itself, and calls that
// overlap on the GPU (different streams, or host threads racing) race on it.
#include <cuda_runtime.h>

#include <mutex>

#include "hm_internal.cuh"

namespace hm {

static __device__ __align__(256) unsigned char g_noalloc_scratch[HM_NOALLOC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
static void *g_scratch_addr[kMaxDevices] = {};
static std::mutex g_scratch_mu;

// Device address of g_noalloc_scratch on the current device (set-up on the
// first call per device).
static int scratch_address(void **out) {
    int dev = 0;
    HM_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices)
        return set_error(HM_ERR_UNSUPPORTED, "device ordinal %d above %d", dev, kMaxDevices - 1);
    std::lock_guard<std::mutex> lk(g_scratch_mu);
    if (!g_scratch_addr[dev]) {
        void *p = nullptr;
        HM_CUDA_TRY(cudaGetSymbolAddress(&p, g_noalloc_scratch));
        g_scratch_addr[dev] = p;
    }
    *out = g_scratch_addr[dev];
    return HM_OK;
}

}  // namespace hm

using namespace hm;

extern "C" {

size_t hm_noalloc_scratch_bytes(void) { return HM_NOALLOC_SCRATCH_BYTES; }

int hm_knn_smooth_noalloc(const float *d_data, uint64_t n, uint32_t d, uint32_t k, int metric,
                          uint32_t *d_idx, float *d_dist, float *d_sigma, float *d_rho,
                          void *stream) {
    const size_t need = hm_workspace_bytes(n, d, k, metric, HM_PATH_PLAIN);
    if (need == 0) return HM_ERR_INVALID;  // message set by hm_workspace_bytes
    if (need > HM_NOALLOC_SCRATCH_BYTES)
        return set_error(HM_ERR_UNSUPPORTED,
                         "n=%llu d=%u k=%u needs %zu bytes of scratch; the static scratch of "
                         "hm_knn_smooth_noalloc holds %zu (use hm_knn_smooth_device with a "
                         "caller-provided workspace)",
                         (unsigned long long)n, d, k, need, (size_t)HM_NOALLOC_SCRATCH_BYTES);
    void *scratch = nullptr;
    HM_TRY(scratch_address(&scratch));
    return hm_knn_smooth_device(d_data, n, d, k, metric, HM_PATH_PLAIN, d_idx, d_dist, d_sigma,
                                d_rho, scratch, HM_NOALLOC_SCRATCH_BYTES, stream, nullptr);
}

}  // extern "C"
