// timing.cu -- launch counting and optional CUDA-event timing per kernel class.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <mutex>
#include <vector>

#include "hm_internal.cuh"

namespace hm {

static std::atomic<uint64_t> g_launches{0};
static std::atomic<bool> g_timing{false};

struct Pending {
    cudaEvent_t start, stop;
};
struct ClassTimes {
    std::vector<Pending> pending;   // recorded, not yet read
    std::vector<cudaEvent_t> open;  // starts waiting for their stop
    double ms = 0.0;
    uint64_t launches = 0;
};
static std::mutex g_mu;
static ClassTimes g_classes[HM_KCLASS_COUNT];
static std::vector<cudaEvent_t> g_free;

void count_launch(uint64_t n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

namespace {
struct SmemSetting {
    const void *func;
    int device;
    int bytes;
};
std::mutex g_attr_mu;
std::vector<SmemSetting> g_attr;
int g_sms[64] = {};
}  // namespace

int ensure_dynamic_smem(const void *func, int bytes) {
    int dev = 0;
    HM_CUDA_TRY(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(g_attr_mu);
    for (const SmemSetting &a : g_attr)
        if (a.func == func && a.device == dev && a.bytes >= bytes) return HM_OK;
    HM_CUDA_TRY(cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    for (SmemSetting &a : g_attr)
        if (a.func == func && a.device == dev) {
            a.bytes = bytes;
            return HM_OK;
        }
    g_attr.push_back({func, dev, bytes});
    return HM_OK;
}

int device_sm_count() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
        cudaGetLastError();
        return 148;
    }
    if (!g_sms[dev]) {
        int sms = 0;
        if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0) {
            cudaGetLastError();
            return 148;
        }
        g_sms[dev] = sms;
    }
    return g_sms[dev];
}
bool timing_enabled() { return g_timing.load(std::memory_order_relaxed); }

static cudaEvent_t take_event() {
    if (!g_free.empty()) {
        cudaEvent_t e = g_free.back();
        g_free.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}

void timing_record(int kclass, cudaStream_t s, bool start) {
    if (kclass < 0 || kclass >= HM_KCLASS_COUNT) return;
    std::lock_guard<std::mutex> lk(g_mu);
    ClassTimes &c = g_classes[kclass];
    if (start) {
        cudaEvent_t e = take_event();
        if (e && cudaEventRecord(e, s) == cudaSuccess) c.open.push_back(e);
    } else if (!c.open.empty()) {
        cudaEvent_t st = c.open.back();
        c.open.pop_back();
        cudaEvent_t e = take_event();
        if (e && cudaEventRecord(e, s) == cudaSuccess) c.pending.push_back({st, e});
    }
}

// Binary64 throughput probe: every thread runs eight independent chains of
// a round-to-nearest multiply and add (the operations of the exact kernels),
// so the FP64 pipe, not latency, bounds it.  The sum lands in a device
// variable only under a condition the compiler cannot rule out.
static __device__ double g_fp64_sink;

__global__ void __launch_bounds__(256) fp64_rate_kernel(double seed, uint32_t iters) {
    double a[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) a[q] = seed + (double)(threadIdx.x * 8 + q) * 1e-6;
    const double m = 1.0000000001, c = 1e-12;
    for (uint32_t i = 0; i < iters; ++i) {
#pragma unroll
        for (int q = 0; q < 8; ++q) a[q] = __dadd_rn(__dmul_rn(a[q], m), c);
    }
    double t = 0.0;
#pragma unroll
    for (int q = 0; q < 8; ++q) t = __dadd_rn(t, a[q]);
    if (t == 12345.678) g_fp64_sink = t;
}

}  // namespace hm

using namespace hm;

extern "C" {

int hm_measure_fp64_rate(double *ops_per_s) {
    clear_error();
    if (!ops_per_s) return set_error(HM_ERR_INVALID, "NULL pointer argument");
    const int sms = device_sm_count();
    const uint32_t iters = 4096, threads = 256, blocks = (uint32_t)sms * 8;
    cudaStream_t s = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    HM_CUDA_TRY(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    int rc = HM_OK;
    double best = 0.0;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
        rc = set_error(HM_ERR_CUDA, "cudaEventCreate failed");
    } else {
        for (int rep = 0; rep < 4 && rc == HM_OK; ++rep) {  // the first run warms the clocks
            cudaEventRecord(e0, s);
            fp64_rate_kernel<<<blocks, threads, 0, s>>>(1.0 + rep, iters);
            count_launch();
            cudaEventRecord(e1, s);
            float ms = 0.f;
            const cudaError_t e = cudaEventSynchronize(e1);
            if (e != cudaSuccess || cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess || ms <= 0.f) {
                rc = set_error(HM_ERR_CUDA, "fp64 probe failed: %s", cudaGetErrorString(e));
                break;
            }
            const double ops = (double)blocks * threads * iters * 16.0;  // 8 chains x (mul + add)
            if (rep > 0) best = std::max(best, ops / (ms * 1e-3));
        }
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaStreamDestroy(s);
    if (rc == HM_OK) *ops_per_s = best;
    return rc;
}

int hm_timing_enable(int on) {
    g_timing.store(on != 0);
    return HM_OK;
}

int hm_timing_read(int kernel_class, double *total_ms, uint64_t *launches, int reset) {
    if (kernel_class < 0 || kernel_class >= HM_KCLASS_COUNT)
        return set_error(HM_ERR_INVALID, "unknown kernel class %d", kernel_class);
    std::lock_guard<std::mutex> lk(g_mu);
    ClassTimes &c = g_classes[kernel_class];
    for (const Pending &p : c.pending) {
        float ms = 0.f;
        if (cudaEventSynchronize(p.stop) == cudaSuccess &&
            cudaEventElapsedTime(&ms, p.start, p.stop) == cudaSuccess)
            c.ms += ms;
        c.launches += 1;
        g_free.push_back(p.start);
        g_free.push_back(p.stop);
    }
    c.pending.clear();
    if (total_ms) *total_ms = c.ms;
    if (launches) *launches = c.launches;
    if (reset) {
        c.ms = 0.0;
        c.launches = 0;
    }
    return HM_OK;
}

uint64_t hm_launch_count(void) { return g_launches.load(); }

}  // extern "C"
