// One-dimensional bulk copies global -> shared memory (cp.async.bulk, sm_90+) completed through an
// mbarrier, for the ROI staging of the QI kernel. Single-CTA form only: the destination is this
// CTA's own shared memory and the source this GPU's own global memory.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace qtrk {

__device__ __forceinline__ uint32_t smem_addr(const void *p) { return static_cast<uint32_t>(__cvta_generic_to_shared(p)); }

// Initialise an mbarrier expecting one arrival per phase (one thread; a barrier must follow).
__device__ __forceinline__ void mbar_init(uint64_t *mbar)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(mbar)));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Start a copy of `bytes` (a multiple of 16; both addresses 16-byte aligned) from global `src`
// to shared `dst`, completing the current phase of `mbar` when all bytes have landed. One
// thread. Shared-memory reads and writes of the CTA's threads that precede this call (ordered
// by a barrier) are ordered before the copy's writes by the proxy fence.
__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes, uint64_t *mbar)
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(mbar)), "r"(bytes)
                 : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_addr(mbar))
                 : "memory");
}

__device__ __forceinline__ bool mbar_test(uint64_t *mbar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(smem_addr(mbar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Wait until the phase with the given parity of `mbar` has completed, polling at most `limit`
// times (each poll may suspend the thread for a hardware-defined interval). Returns false when
// the limit was reached.
__device__ __forceinline__ bool mbar_wait(uint64_t *mbar, uint32_t parity, uint32_t limit)
{
    for (uint32_t i = 0; i < limit; i++)
        if (mbar_test(mbar, parity)) return true;
    return false;
}

}  // namespace qtrk
