// Staging into shared memory by TMA bulk copies: an mbarrier per buffer, completed by the copy's
// byte count (cp.async.bulk ... mbarrier::complete_tx::bytes), and waits on it bounded by the
// global timer so that a copy that never lands becomes an error the host reads, not a hang.
#pragma once

#include <cstdint>

namespace qm {

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
    unsigned a = (unsigned)__cvta_generic_to_shared(bar);
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(a), "r"(count));
}

__device__ __forceinline__ void bulk_load(void *dst, const void *src, unsigned bytes, uint64_t *bar) {
    unsigned d = (unsigned)__cvta_generic_to_shared(dst), b = (unsigned)__cvta_generic_to_shared(bar);
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(b), "r"(bytes) : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(d),
                 "l"(src), "r"(bytes), "r"(b)
                 : "memory");
}

__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

// Waits for the barrier's phase for at most `limit_ns` (about a second by default); false when it
// gave up.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, unsigned phase, uint64_t limit_ns = 1000000000ull) {
    unsigned b = (unsigned)__cvta_generic_to_shared(bar);
    const uint64_t start = global_ns();
    for (;;) {
        unsigned done;
        asm volatile(
            "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
            : "=r"(done)
            : "r"(b), "r"(phase)
            : "memory");
        if (done) return true;
        if (global_ns() - start > limit_ns) return false;
    }
}

// Orders this thread's earlier generic-proxy accesses of shared memory before later async-proxy
// (bulk copy) accesses: a buffer read by the threads is then safe to refill by a bulk copy.
__device__ __forceinline__ void fence_proxy_async_shared() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

}  // namespace qm
