// One-dimensional bulk copies (the TMA unit's cp.async.bulk) between this GPU's global memory and a
// CTA's shared memory, completing on a shared-memory mbarrier, for the BATCHED kernels (sm_100a).
// Every copy here is a plain CTA-local copy: no cluster multicast, and the global side is always
// this GPU's own tables.  Sources and destinations are 16-byte aligned, sizes multiples of 16.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace parw2v {

__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned) __cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// One arrival that also announces `bytes` of copies completing on the barrier in this phase.
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait for the phase with the given parity: false after max_polls unsuccessful polls (each
// poll may suspend the thread for a hardware-chosen time), so a copy that never completes ends in
// an error status instead of a hung kernel.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, unsigned parity, unsigned max_polls) {
    for (unsigned i = 0; i < max_polls; i++)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}
// global -> shared, completing `bytes` on bar
__device__ __forceinline__ void bulk_load(void *dst_smem, const void *src_gmem, unsigned bytes, uint64_t *bar) {
    asm volatile("cp.async.bulk.shared::cta.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst_smem)),
                 "l"(src_gmem), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}
// shared -> global, in the thread's current bulk async-group
__device__ __forceinline__ void bulk_store(void *dst_gmem, const void *src_smem, unsigned bytes) {
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst_gmem),
                 "r"(smem_u32(src_smem)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
// this thread's bulk stores have read their shared-memory sources (the staging may be reused)
__device__ __forceinline__ void bulk_wait_read_all() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
// this thread's bulk stores are complete in global memory
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

// Orders this thread's generic-proxy accesses before its later async-proxy (bulk copy) accesses,
// and the other way round: shared memory rewritten by the bulk unit after being read by ldmatrix,
// global rows written by plain stores and then read by bulk copies.
__device__ __forceinline__ void fence_proxy_async_shared() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async_global() { asm volatile("fence.proxy.async.global;" ::: "memory"); }

// Polls allowed per staging wait: far beyond any real copy latency (a poll suspends for up to
// about a microsecond), small enough that a lost completion ends the kernel in seconds.
constexpr unsigned kMaxBulkPolls = 1u << 22;

}  // namespace parw2v
