// mbar.cuh -- shared-memory mbarrier helpers for the TMA-staged kernels:
// initialisation, expected-transaction arrival and a bounded phase wait.
#pragma once
#include <cstdint>

namespace hc {

__device__ __forceinline__ unsigned smem_addr(const void *p)
{
    return (unsigned)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

// Bounded wait on an mbarrier phase; returns false if the limit ran out.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, unsigned parity)
{
    const unsigned a = smem_addr(bar);
    for (int it = 0; it < (1 << 22); it++) {
        unsigned ok;
        asm volatile("{\n\t.reg .pred p;\n\t"
                     "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                     "selp.u32 %0, 1, 0, p;\n\t}"
                     : "=r"(ok)
                     : "r"(a), "r"(parity)
                     : "memory");
        if (ok) return true;
        if (it > 64) __nanosleep(32);
    }
    return false;
}

}  // namespace hc
