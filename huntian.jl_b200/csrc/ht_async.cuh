// Asynchronous-copy helpers shared by the TMA pipelines (peak scan, pencil FFT passes):
// mbarrier set-up, bounded waits and 1-D bulk copies global -> shared.
//
// Every wait is bounded: a wait that has not completed after its limit of %globaltimer
// (kWaitNs unless the context sets another, ht_ctx_tune HT_TUNE_WAIT_NS) returns false,
// and the kernel records that in the context's status word, drains its own copies in
// flight (again with bounded waits) and returns, so that a stalled copy shows up as an
// error code on the host instead of a hung device.
#pragma once

#include <cuda_runtime.h>

namespace htasync {

constexpr long long kWaitNs = 2000000000LL;   // 2 s, the default limit

__device__ __forceinline__ unsigned smem_addr(const void* p) {
    return (unsigned)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ long long global_ns() {
    long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Initialise an mbarrier expecting `count` arrivals per phase (one thread), and make the
// initialisation visible to the async proxy.
__device__ __forceinline__ void bar_init(unsigned long long* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_addr(bar)), "r"(count));
}
__device__ __forceinline__ void bar_init_fence() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Order this thread's earlier shared-memory accesses before later async-proxy writes (a
// slot that was read is about to be refilled by a bulk copy).
__device__ __forceinline__ void fence_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Arrive on bar announcing `bytes` of transactions for the current phase.
__device__ __forceinline__ void bar_expect(unsigned long long* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;"
                 :: "r"(smem_addr(bar)), "r"(bytes) : "memory");
}

// 1-D bulk copy of `bytes` (multiple of 16; both addresses 16-byte aligned) from global to
// this CTA's shared memory, completing as transactions on bar.
__device__ __forceinline__ void bulk_load(void* dst, const void* src, unsigned bytes,
                                          unsigned long long* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
        :: "r"(smem_addr(dst)), "l"(src), "r"(bytes), "r"(smem_addr(bar)) : "memory");
}

// Wait for phase `parity` of the barrier, giving up after limit_ns.
__device__ __forceinline__ bool bar_wait(unsigned long long* bar, unsigned parity,
                                         long long limit_ns = kWaitNs) {
    const unsigned b = smem_addr(bar);
    long long t0 = 0;
    for (int it = 0;; ++it) {
        unsigned ok;
        asm volatile("{\n .reg .pred p;\n"
                     " mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
                     " selp.u32 %0, 1, 0, p;\n}"
                     : "=r"(ok) : "r"(b), "r"(parity) : "memory");
        if (ok) return true;
        if (it == 0) t0 = global_ns();
        else if ((it & 63) == 0 && global_ns() - t0 > limit_ns) return false;
    }
}

}  // namespace htasync
