// hhs_common.cuh -- device-side building blocks shared by the HOLD kernels.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

#include "hhs_internal.h"

// Error bits recorded in a device error word instead of trapping.
#define HHS_ERRBIT_LOOKBACK_TIMEOUT 1u
#define HHS_ERRBIT_BARRIER_TIMEOUT 2u
#define HHS_ERRBIT_DEPTH 4u
#define HHS_ERRBIT_BOUNDS 8u
#define HHS_ERRBIT_CAPACITY 16u

// Spin-wait limits: every wait on another CTA gives up after this many polls
// (with nanosleep back-off, well above a second), records an error bit and
// returns, so a broken invariant can never hang the device.
#define HHS_SPIN_LIMIT (1u << 22)

#define HHS_FULL_MASK 0xffffffffu

// SoA particle arrays as the kernels see them (by value).
struct SoA {
    double *x, *y, *z, *vx, *vy, *vz, *m, *ts;
    int32_t* id;
};

__device__ __forceinline__ int warp_incl_scan(int v, int lane) {
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int t = __shfl_up_sync(HHS_FULL_MASK, v, o);
        if (lane >= o) v += t;
    }
    return v;
}

__device__ __forceinline__ int warp_sum(int v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(HHS_FULL_MASK, v, o);
    return v;
}

__device__ __forceinline__ unsigned long long ld_relaxed_u64(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_relaxed_u64(unsigned long long* p, unsigned long long v) {
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_release_u32(unsigned* p, unsigned v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ unsigned atom_add_acq_rel_u32(unsigned* p, unsigned v) {
    unsigned old;
    asm volatile("atom.add.acq_rel.gpu.global.u32 %0, [%1], %2;"
                 : "=r"(old) : "l"(p), "r"(v) : "memory");
    return old;
}

__device__ __forceinline__ void red_add_release_u32(unsigned* p, unsigned v) {
    asm volatile("red.add.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Kernel launches issued by the library (hhs_kernel_launch_count).
void hhs_count_launch();

// Host-side launch check after every kernel launch: counts the launch and converts a
// pending launch error into a status.
#define HHS_LAUNCH_CHECK()                                        \
    do {                                                          \
        hhs_count_launch();                                       \
        cudaError_t e__ = cudaGetLastError();                     \
        if (e__ != cudaSuccess) return hhs_from_cuda(e__);        \
    } while (0)

#define HHS_CUDA_TRY(call)                                        \
    do {                                                          \
        cudaError_t e__ = (call);                                 \
        if (e__ != cudaSuccess) return hhs_from_cuda(e__);        \
    } while (0)

static inline hhs_status hhs_from_cuda(cudaError_t e) {
    if (e == cudaSuccess) return HHS_OK;
    if (e == cudaErrorMemoryAllocation) return HHS_ERR_OOM;
    return HHS_ERR_CUDA;
}
