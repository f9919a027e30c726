// tma.cuh -- mbarrier helpers (bounded waits) for the tcgen05 kernels, sm_100a.
//
// Every wait is bounded in wall time; on expiry the caller's error word gets
// the given code (first writer wins) and the wait returns false, so a kernel
// never spins forever and the host can report IPFC_ERR_TIMEOUT.  No
// multicast form is used anywhere.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace ipfc {


__device__ __forceinline__ unsigned smem_u32(const void* p) {
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// Makes barrier initialisation visible to the async (TMA) proxy.
__device__ __forceinline__ void fence_barrier_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile(
        "{\n\t.reg .b64 st;\n\t"
        "mbarrier.arrive.shared::cta.b64 st, [%0];\n\t}" ::"r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, unsigned bytes) {
    asm volatile(
        "{\n\t.reg .b64 st;\n\t"
        "mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}" ::"r"(smem_u32(bar)),
        "r"(bytes)
        : "memory");
}

// try_wait with a suspend-time hint: the thread sleeps until the phase
// completes or about hint_ns nanoseconds pass, instead of spinning -- a
// waiting warp then takes no issue slots from the warps doing the work.
__device__ __forceinline__ bool mbar_try_wait_sleep(uint64_t* bar, unsigned parity, unsigned hint_ns) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity), "r"(hint_ns)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ unsigned long long globaltimer_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Default bound of a pipeline wait, and the bound of the final drain wait
// before tensor memory is freed (independent of the pipeline bound, so a
// shortened pipeline bound never frees memory under a running MMA).
constexpr unsigned long long kWaitNsDefault = 250ull * 1000 * 1000;
constexpr unsigned long long kDrainNs = 2000ull * 1000 * 1000;

// Bounded wait for the phase of the given parity to complete.  The bound is
// wall time on the global timer (try_wait may suspend the thread for a
// system-dependent time per poll, so a poll count bounds nothing).  On
// expiry the error word gets `code` (first writer wins) and it returns false.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity, unsigned* err, unsigned code,
                                          unsigned long long limit_ns = kWaitNsDefault) {
    if (mbar_try_wait(bar, parity)) return true;
    const unsigned long long t0 = globaltimer_ns();
    for (unsigned i = 1;; ++i) {
        if (mbar_try_wait(bar, parity)) return true;
        if ((i & 63u) == 0 && globaltimer_ns() - t0 > limit_ns) break;
    }
    if (err) atomicCAS(err, 0u, code);
    return false;
}

}  // namespace ipfc
