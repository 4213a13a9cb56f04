// Device-side synchronisation and copy primitives of the persistent sweep kernels: shared-memory
// mbarriers, relaxed / acquire global accesses, cp.async stages, and a bounded mbarrier wait that
// reports through the device error word instead of spinning forever.
#pragma once

#include <cstdint>

#include <cuda_runtime.h>

#include "idc_internal.hpp"

namespace idc {

constexpr unsigned kFullMask = 0xffffffffu;

__device__ __forceinline__ uint32_t saddr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(saddr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
    asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}" ::"r"(saddr(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(saddr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ bool mbar_test(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(saddr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ int ld_relaxed(const int *p) {
    int v;
    asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ double ld_relaxed_f64(const double *p) {
    double v;
    asm volatile("ld.relaxed.gpu.global.f64 %0, [%1];" : "=d"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_relaxed_f64(double *p, double v) {
    asm volatile("st.relaxed.gpu.global.f64 [%0], %1;" ::"l"(p), "d"(v) : "memory");
}
__device__ __forceinline__ bool is_sentinel(double v) {
    return (unsigned long long)__double_as_longlong(v) == kTraceSentinel;
}
__device__ __forceinline__ double sentinel_value() { return __longlong_as_double((long long)kTraceSentinel); }

__device__ __forceinline__ void cp_async8(void *dst, const void *src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(saddr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int n>
__device__ __forceinline__ void cp_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(n) : "memory");
}

// Bounded, warp-uniform wait on an mbarrier phase.  Returns false if the wait gave up or another warp
// has recorded an error; in both cases the device error word is non-zero afterwards.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, int *error, long long limit) {
    if (mbar_test(bar, parity)) return true;   // a completed phase: the non-blocking test is cheaper
    for (long long n = 0;; ++n) {
        if (mbar_try(bar, parity)) return true;
        if ((n & 63) == 63 && ld_relaxed(error) != kDevOk) return false;
        if (n > limit) {
            atomicCAS(error, kDevOk, kDevTimeout);
            return false;
        }
    }
}

}  // namespace idc
