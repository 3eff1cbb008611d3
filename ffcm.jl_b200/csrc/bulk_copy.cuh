// Bulk asynchronous copies from global to shared memory (the TMA's untiled
// form, cp.async.bulk) with an mbarrier for completion, and the bulk-group
// bookkeeping of stores from shared to global memory. Each block fills only
// its own shared memory from this GPU's memory. Addresses and sizes must be
// multiples of 16 bytes.
#pragma once

#include "common.cuh"

namespace ffcm {

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
    // make the initialised barrier visible to the copy engine
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Arrive once and announce `bytes` of copies that will complete on `bar`.
__device__ __forceinline__ void mbar_arrive_expect(uint64_t* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Wait for phase `parity` of `bar` with an iteration limit; false if it gave up.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, unsigned parity, int max_iter) {
    for (int it = 0; it < max_iter; ++it)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

// Orders this thread's earlier shared-memory accesses, and those of other
// threads made visible to it by a barrier, before later bulk copies (the copy
// engine is another proxy): needed before a copy overwrites shared memory that
// threads have just read.
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// global -> shared, completing `bytes` of transactions on `bar`.
__device__ __forceinline__ void bulk_load(void* dst_smem, const void* src_global, unsigned bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_addr(dst_smem)),
        "l"(src_global), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

// Bulk stores (shared -> global, the async proxy reading this block's shared
// memory) are tracked as bulk groups of the issuing thread.
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }

// The issuing thread waits until its committed bulk stores have finished
// reading shared memory (the source may then be overwritten).
__device__ __forceinline__ void bulk_wait_read_all() {
    asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
}

// The issuing thread waits until its committed bulk stores are complete.
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

}  // namespace ffcm
