// bulk_copy.cuh -- asynchronous global -> shared row staging with the bulk
// copy engine (cp.async.bulk, completion on an mbarrier), sm_90+ PTX used on
// sm_100a.
//
// A row of a per-vertex array (4-byte elements starting anywhere) is fetched
// as the 16-byte-aligned window that contains it: the copy starts at the row
// start rounded down to 16 bytes and its size is rounded up to a multiple of
// 16, as the bulk copy requires; the row then begins `off` elements into the
// shared buffer.  The source allocation must extend at least 12 bytes past
// the last row end (the caller pads it).  No multicast: every copy reads
// this GPU's own memory into this CTA's shared memory.
//
// Waits are bounded: a wait that does not see the copy complete within
// BULK_WAIT_SPINS polls reports failure and the caller sets an error flag
// instead of spinning forever.
#pragma once

#include <cstdint>

namespace csaw {

constexpr int BULK_WAIT_SPINS = 1 << 22;

__device__ __forceinline__ uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// One arrival (the issuing thread's) completes a phase once the bytes land.
__device__ __forceinline__ void mbar_init(uint64_t *bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bar)) : "memory");
}

// Makes barrier initialisation visible to the bulk copy engine (the async
// proxy); follow with a CTA barrier.
__device__ __forceinline__ void mbar_init_fence() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

// Orders this thread's earlier shared-memory accesses (generic proxy) before
// later bulk copies into the same memory (async proxy).
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// Starts copying `bytes` (a multiple of 16; both addresses 16-byte aligned)
// from global src to shared dst, completing the barrier's current phase.
__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}

// Three copies completing one phase together (sizes multiples of 16, 0 for
// none; addresses 16-byte aligned): one arrival expecting all their bytes.
__device__ __forceinline__ void bulk_copy_tx(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}

__device__ __forceinline__ void bulk_load3(void *d0, const void *s0, uint32_t b0, void *d1, const void *s1, uint32_t b1,
                                           void *d2, const void *s2, uint32_t b2, uint64_t *bar) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(b0 + b1 + b2)
                 : "memory");
    if (b0) bulk_copy_tx(d0, s0, b0, bar);
    if (b1) bulk_copy_tx(d1, s1, b1, bar);
    if (b2) bulk_copy_tx(d2, s2, b2, bar);
}

__device__ __forceinline__ bool mbar_test(uint64_t *bar, uint32_t parity) {
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

// Waits (bounded) for the phase with the given parity to complete.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
    for (int i = 0; i < BULK_WAIT_SPINS; ++i)
        if (mbar_test(bar, parity)) return true;
    return false;
}

// The 16-byte-aligned window holding elements [0, d) of row `src`: its
// start, the row's offset in it (elements) and its size in bytes.
struct RowWindow {
    const void *start;
    int off;
    uint32_t bytes;
};

__device__ __forceinline__ RowWindow row_window(const float *src, int d) {
    const uintptr_t a = (uintptr_t)src, a0 = a & ~(uintptr_t)15;
    RowWindow w;
    w.start = (const void *)a0;
    w.off = (int)((a - a0) >> 2);
    w.bytes = (uint32_t)(((uintptr_t)(w.off + d) * 4 + 15) & ~(uintptr_t)15);
    return w;
}

}  // namespace csaw
