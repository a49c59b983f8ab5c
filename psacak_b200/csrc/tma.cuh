// tma.cuh -- bulk global->shared copies through the TMA engine, completed
// on a shared-memory mbarrier (sm_90+ PTX; used here on sm_100a).
//
// One elected thread arms the barrier with the expected byte count and
// issues the copies; every thread then waits on the barrier's phase.  No
// cluster multicast is used: each CTA copies into its own shared memory.
// Waits are bounded; a wait that gives up reports DEVERR_TIMEOUT, and the
// CTA agrees on the outcome and waits once more (bounded) before it retires,
// so no copy is left writing into shared memory that has been released.
#pragma once

#include "common.cuh"

namespace psk {

constexpr uint32_t TMA_SPIN_LIMIT = 1u << 22;

__device__ __forceinline__ uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
    // make the initialised barrier visible to the async (TMA) proxy
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}

// dst, src and bytes must be multiples of 16 bytes.
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
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

// Bounded wait for the given phase; false (and DEVERR_TIMEOUT) if it did not
// complete within TMA_SPIN_LIMIT polls.
// The outcome is this thread's own: a caller whose threads go on to
// block-wide barriers or full-warp votes must agree on it first (see
// mbar_wait_cta).
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity, uint32_t *err) {
    uint32_t left = 0;
    while (true) {
        if (mbar_try_wait(bar, parity)) return true;
        if (spin_spend(left, err, TMA_SPIN_LIMIT)) break;
    }
    dev_fail(err, DEVERR_TIMEOUT);
    return false;
}

// Bounded wait by every thread of the CTA with one CTA-wide outcome: if any
// thread's wait ran out, every thread waits once more (bounded; the copies
// may still be landing in shared memory) and all of them get false, so the
// CTA retires as a whole instead of leaving some threads in later barriers.
// Must be called by all threads of the CTA.
__device__ __forceinline__ bool mbar_wait_cta(uint64_t *bar, uint32_t parity, uint32_t *err) {
    const bool ok = mbar_wait_bounded(bar, parity, err);
    if (__syncthreads_or(!ok)) {
        mbar_wait_bounded(bar, parity, err);
        return false;
    }
    return true;
}

}  // namespace psk
