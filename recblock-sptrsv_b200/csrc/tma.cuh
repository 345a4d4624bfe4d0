// tma.cuh -- shared-memory, mbarrier and 1D bulk-copy (TMA) helpers.
#pragma once

#include "kernels.cuh"

namespace rbs {

__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long *bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(unsigned long long *bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long *bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, unsigned bytes, unsigned long long *bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

// Rounded 16-byte copy window of `count` elements of size `es` starting at
// `src`: returns bytes to copy, sets the aligned source and the element
// offset of src inside the window.
__device__ __forceinline__ unsigned bulk_window(const void *src, int count, int es, const void *&asrc, int &delta) {
    const unsigned long long a = (unsigned long long)src;
    const unsigned long long a0 = a & ~15ull;
    const unsigned long long a1 = (a + (unsigned long long)count * es + 15ull) & ~15ull;
    asrc = (const void *)a0;
    delta = (int)((a - a0) / es);
    return (unsigned)(a1 - a0);
}

}  // namespace rbs
