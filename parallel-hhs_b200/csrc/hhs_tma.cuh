// hhs_tma.cuh -- shared-memory transaction barriers and 1-D bulk copies (sm_90+ PTX,
// used here on sm_100a) for the kernels that stream contiguous data through shared
// memory: a single CTA issues cp.async.bulk global -> shared copies that complete on an
// mbarrier, and its threads wait on the barrier's phase parity. No cluster multicast is
// used anywhere: every copy lands in the issuing CTA's own shared memory and reads this
// GPU's own global memory.
//
// Every wait is bounded: after kMbarWaitLimit polls (each try_wait suspends for a
// hardware-chosen time, so the limit is well above a second) the wait records an error
// bit and returns false instead of hanging.
#pragma once
#include <cstdint>

#include "hhs_common.cuh"

constexpr unsigned kMbarWaitLimit = 1u << 24;

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

// One arrival expected per phase (the thread that posts the transaction count).
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned arrivals) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(arrivals)
                 : "memory");
}

// Makes barrier initialisation visible to the asynchronous (bulk-copy) proxy and to the
// other threads (which must still synchronise with the initialising thread).
__device__ __forceinline__ void fence_barrier_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Arrive and add `bytes` to the transaction count of the current phase.
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
                 "r"(bytes)
                 : "memory");
}

// Bulk copy of `bytes` (a multiple of 16; both addresses 16-byte aligned) from global to
// this CTA's shared memory, completing `bytes` transactions on `bar`.
__device__ __forceinline__ void bulk_load(void* dst, const void* src, unsigned bytes,
                                          uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
            "r"(smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0u;
}

// Waits for the phase with the given parity to complete. Returns false (and records
// HHS_ERRBIT_BARRIER_TIMEOUT in *err) if it did not within the poll limit.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity, unsigned* err) {
    for (unsigned i = 0; i < kMbarWaitLimit; i++) {
        if (mbar_try_wait(bar, parity)) return true;
    }
    if (err) atomicOr(err, HHS_ERRBIT_BARRIER_TIMEOUT);
    return false;
}
