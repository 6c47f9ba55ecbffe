// Bulk copies global -> shared memory by the Tensor Memory Accelerator (cp.async.bulk, 1-D) with
// transaction-count mbarriers, for row passes that stream a contiguous block.
//
// A copy moves `bytes` (a multiple of 16) from a 16-byte-aligned global address to a 16-byte-
// aligned shared address and completes on an mbarrier whose phase expects that many bytes. Every
// wait is bounded: a wait that runs out returns false and the kernel reports it through an error
// flag instead of spinning on.
#pragma once

#include "device.cuh"

namespace fereg {

__device__ __forceinline__ u32 smem_addr(const void* p) { return static_cast<u32>(__cvta_generic_to_shared(p)); }

// Asynchronous 4- and 8-byte copies global -> shared memory (cp.async, no registers held while in
// flight), committed in groups: the issuing thread waits for its own groups (cp_async_wait_all, or
// cp_async_wait_prior for all but the latest), then a warp or CTA barrier before other threads
// read them.
__device__ __forceinline__ void cp_async8(void* dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_addr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async4(void* dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(smem_addr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }
// Waits until at most one of this thread's committed groups is still in flight.
__device__ __forceinline__ void cp_async_wait_prior() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }

__device__ __forceinline__ void mbar_init(u64* bar, u32 count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

// Makes the initialized barriers visible to the async proxy (before the CTA-wide sync).
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

// The calling thread's arrival, announcing `bytes` of transactions for the current phase.
__device__ __forceinline__ void mbar_expect_tx(u64* bar, u32 bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

// Global -> shared bulk copy completing on `bar` (the issuing CTA is its own cluster).
__device__ __forceinline__ void bulk_load(void* dst, const void* src, u32 bytes, u64* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}

__device__ __forceinline__ bool mbar_test(u64* bar, u32 parity) {
    u32 ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Waits for the phase of `bar` with parity `parity` to complete; false after `limit` attempts.
__device__ __forceinline__ bool mbar_wait(u64* bar, u32 parity, u32 limit) {
    for (u32 i = 0; i < limit; i++)
        if (mbar_test(bar, parity)) return true;
    return false;
}

constexpr u32 MBAR_WAIT_LIMIT = 1u << 22;  // attempts (each may suspend briefly): far beyond any copy

}  // namespace fereg
