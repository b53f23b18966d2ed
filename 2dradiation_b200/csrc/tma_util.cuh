// Shared-memory staging primitives of the precision-form kernels: mbarrier
// phases with bounded waits, and TMA tensor copies into shared memory.
// Every wait has a time limit (the global nanosecond timer), after which the
// caller reports a fault instead of spinning on.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

namespace grlbm
{
__device__ __forceinline__ unsigned smem_addr(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
// the issuing thread's arrival on the current phase, announcing `bytes` of copies
__device__ __forceinline__ void mbar_arrive_expect(unsigned bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_test(unsigned bar, unsigned parity)
{
    unsigned done;
    asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, "
                 "p;\n}\n"
                 : "=r"(done)
                 : "r"(bar), "r"(parity)
                 : "memory");
    return done != 0;
}
// The same, but the thread may sleep in the instruction until the phase
// completes or about `hint_ns` nanoseconds pass (no busy spinning).
__device__ __forceinline__ bool mbar_test_sleep(unsigned bar, unsigned parity, unsigned hint_ns)
{
    unsigned done;
    asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\tselp.u32 %0, "
                 "1, 0, p;\n}\n"
                 : "=r"(done)
                 : "r"(bar), "r"(parity), "r"(hint_ns)
                 : "memory");
    return done != 0;
}
__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
// Wait for the phase of the given parity to complete, for limit_ns at most;
// false at once when another block has already raised the fault word.  The
// thread sleeps in the wait instruction (up to 20 us at a time) instead of
// spinning.
__device__ __forceinline__ bool mbar_wait(unsigned bar, unsigned parity, unsigned long long limit_ns,
                                          const unsigned *fault)
{
    if (mbar_test(bar, parity))
        return true;
    if (fault && *reinterpret_cast<const volatile unsigned *>(fault))
        return false;
    const unsigned long long t0 = global_ns();
    do
    {
        if (mbar_test_sleep(bar, parity, 20000u))
            return true;
    } while (global_ns() - t0 < limit_ns);
    return false;
}

// One box of a 4D tensor at element coordinates (c0, c1, c2, c3) into shared
// memory, completing on the mbarrier.
__device__ __forceinline__ void tma_load_4d(unsigned dst, const CUtensorMap *map, int c0, int c1, int c2, int c3,
                                            unsigned bar)
{
    asm volatile("cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, "
                 "%3, %4, %5}], [%6];\n" ::"r"(dst),
                 "l"(reinterpret_cast<unsigned long long>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(bar)
                 : "memory");
}
// Orders this thread's earlier generic-proxy accesses of shared memory before
// later async-proxy (TMA) accesses of it: issued before a copy that
// overwrites a buffer the threads have been reading.
__device__ __forceinline__ void fence_proxy_async_smem()
{
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}
} // namespace grlbm
