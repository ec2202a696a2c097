// mbarrier.cuh -- shared-memory barriers (mbarrier) with bounded waits, as
// the tensor-core screen uses them.
//
// Every wait is bounded twice: by wall clock (%globaltimer) and by an
// iteration cap, so a copy or an arrival that never comes ends the wait with
// a status the caller turns into an error code instead of a hang.
#pragma once

#include <cstdint>

#include <cuda_runtime.h>

namespace hm {

constexpr uint64_t HM_WAIT_LIMIT_NS = 4000000000ull;  // 4 s
constexpr uint64_t HM_DRAIN_LIMIT_NS = 200000000ull;  // 0.2 s for copies already in flight
constexpr uint32_t HM_WAIT_SPIN_CAP = 1u << 30;

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ uint64_t globaltimer_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait for the phase of parity `parity` to complete.  Gives up when
// another role has raised the abort flag (unless draining) or after the
// time / iteration limits.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, volatile uint32_t *abort_flag,
                                          bool draining = false) {
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = globaltimer_ns();
    const uint64_t limit = draining ? HM_DRAIN_LIMIT_NS : HM_WAIT_LIMIT_NS;
    for (uint32_t spin = 1; spin < HM_WAIT_SPIN_CAP; ++spin) {
        if (mbar_try_wait(bar, parity)) return true;
        if ((spin & 31) == 0) {
            if (!draining && *abort_flag) return false;
            if (globaltimer_ns() - t0 > limit) return false;
        }
    }
    return false;
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
                 : "memory");
}

// Makes barrier initialisation visible to the asynchronous proxy (the copy
// engine completes transactions on the barriers).
__device__ __forceinline__ void mbar_init_fence() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

}  // namespace hm
