// Shared-memory addresses, mbarriers and bulk (TMA engine) copies used by the kernels.
#pragma once
#include <cstdint>

namespace tdi {

// Bounded waits give up after this many SM cycles (about a second).
constexpr long long WAIT_CYCLES = 2000000000ll;

__device__ __forceinline__ uint32_t smem_addr(const void *p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(bar), "r"(count) : "memory");
}

// Waits for the completion of the phase with the given parity; false after ~1 s.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity)
{
    const long long t0 = clock64();
    for (;;) {
        uint32_t done;
        asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                     "selp.u32 %0, 1, 0, p;\n\t}"
                     : "=r"(done) : "r"(bar), "r"(parity) : "memory");
        if (done) return true;
        if (clock64() - t0 > WAIT_CYCLES) return false;
    }
}

// The mbarrier's current phase completes after one more arrival and `bytes` of
// asynchronous copies.
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" :: "r"(bar), "r"(bytes) : "memory");
}

// One arrival on the mbarrier's current phase.
__device__ __forceinline__ void mbar_arrive(uint32_t bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" :: "r"(bar) : "memory");
}

// Contiguous global -> shared copy by the TMA engine (no multicast); size and both addresses
// are multiples of 16 bytes. Completion is counted on the mbarrier.
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void *src, uint32_t bytes, uint32_t bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 :: "r"(dst), "l"(src), "r"(bytes), "r"(bar) : "memory");
}

}  // namespace tdi
