// async.cuh -- helpers of the kernels fed by asynchronous bulk copies (the staged pressure
// solve, the TMA-fed y-pad): shared-memory addresses, the global timer, and bounded
// mbarrier waits.  A wait gives up after kStageWaitNs so that a copy that never lands
// raises an error flag instead of hanging the GPU.
#pragma once
#include <cuda_runtime.h>

namespace obl {

constexpr unsigned long long kStageWaitNs = 1000000000ULL;

__device__ __forceinline__ unsigned smem_addr(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ bool mbar_try_wait(unsigned bar, unsigned parity)
{
    unsigned ok;
    asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(ok)
                 : "r"(bar), "r"(parity)
                 : "memory");
    return ok != 0;
}
// true once the phase of the given parity has completed; false after kStageWaitNs
__device__ __forceinline__ bool mbar_wait_bounded(unsigned bar, unsigned parity)
{
    if (mbar_try_wait(bar, parity)) return true;
    const unsigned long long t0 = global_ns();
    while (!mbar_try_wait(bar, parity))
        if (global_ns() - t0 > kStageWaitNs) return false;
    return true;
}

} // namespace obl
