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
// address is looked up with cudaGetSymbolAddress (with the device current) on
// the first call in each CUDA context of a device, and then passed to the
// kernels; the first call on a device should therefore come before any stream
// capture.  The lookup is keyed on the device and its current context, so a
// context that was destroyed and recreated (cudaDeviceReset) gets the array's
// new address.  All calls share the one array and it keeps the last call's
// contents: the pipeline clears what must start at zero itself, and calls that
// overlap on the GPU (different streams, or host threads racing) race on it.
//
// The counters of the last call (the non-finite-input flag among them) also
// stay in that array; hm_noalloc_stats reads them back without allocating.
#include <cuda.h>
#include <cuda_runtime.h>

#include <mutex>

#include "hm_internal.cuh"

namespace hm {

static __device__ __align__(256) unsigned char g_noalloc_scratch[HM_NOALLOC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;

struct ScratchSlot {
    CUcontext ctx = nullptr;  // context the address was looked up in
    void *addr = nullptr;
    // the last call's problem, so its counters can be found in the scratch
    bool called = false;
    uint64_t n = 0;
    uint32_t d = 0, k = 0;
    int metric = 0;
};
static ScratchSlot g_slots[kMaxDevices];
static std::mutex g_scratch_mu;

typedef CUresult (*CtxGetCurrentFn)(CUcontext *);

// The calling thread's current driver context, or NULL when the thread has
// none bound yet.
static int current_context(CUcontext *out) {
    static std::once_flag once;
    static CtxGetCurrentFn fn = nullptr;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<CtxGetCurrentFn>(p);
    });
    if (!fn) return set_error(HM_ERR_CUDA, "cuCtxGetCurrent unavailable");
    CUcontext c = nullptr;
    if (fn(&c) != CUDA_SUCCESS) return set_error(HM_ERR_CUDA, "cuCtxGetCurrent failed");
    *out = c;
    return HM_OK;
}

// Slot of the current device with the device address of g_noalloc_scratch
// in the current context (set-up on the first call per device and context).
static int scratch_slot(ScratchSlot **out) {
    int dev = 0;
    HM_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices)
        return set_error(HM_ERR_UNSUPPORTED, "device ordinal %d above %d", dev, kMaxDevices - 1);
    CUcontext ctx = nullptr;
    HM_TRY(current_context(&ctx));
    ScratchSlot &S = g_slots[dev];
    if (!S.addr || !ctx || S.ctx != ctx) {
        // the lookup binds the runtime's context of the device to the thread
        void *p = nullptr;
        HM_CUDA_TRY(cudaGetSymbolAddress(&p, g_noalloc_scratch));
        HM_TRY(current_context(&ctx));
        if (S.ctx != ctx) S.called = false;  // a new context: no counters of it yet
        S.addr = p;
        S.ctx = ctx;
    }
    *out = &S;
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
    {
        std::lock_guard<std::mutex> lk(g_scratch_mu);
        ScratchSlot *S = nullptr;
        HM_TRY(scratch_slot(&S));
        scratch = S->addr;
        S->called = true;
        S->n = n;
        S->d = d;
        S->k = k;
        S->metric = metric;
    }
    return hm_knn_smooth_device(d_data, n, d, k, metric, HM_PATH_PLAIN, d_idx, d_dist, d_sigma,
                                d_rho, scratch, HM_NOALLOC_SCRATCH_BYTES, stream, nullptr);
}

int hm_noalloc_stats(void *stream, hm_stats *stats) {
    clear_error();
    uint64_t n;
    uint32_t d, k;
    int metric;
    void *scratch;
    {
        std::lock_guard<std::mutex> lk(g_scratch_mu);
        ScratchSlot *S = nullptr;
        HM_TRY(scratch_slot(&S));
        if (!S->called)
            return set_error(HM_ERR_INVALID, "no hm_knn_smooth_noalloc call on this device yet");
        n = S->n;
        d = S->d;
        k = S->k;
        metric = S->metric;
        scratch = S->addr;
    }
    return single_job_stats(scratch, n, d, k, metric, HM_PATH_PLAIN, static_cast<cudaStream_t>(stream),
                            stats);
}

}  // extern "C"
