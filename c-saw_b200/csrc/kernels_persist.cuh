// kernels_persist.cuh -- every level of a batched neighbor-sampling job in one
// persistent launch (sm_100a).
//
// The batched schedule otherwise launches, per level, the take-all pass
// (k_coop_fast), the warp-list, hub and pair selection passes, the refill
// pass and the CTA retry pass: six launches, each ending in a tail where most
// SMs idle, and small levels that cannot fill 148 SMs.  Here one cooperative
// launch (all CTAs resident) runs the same device bodies level after level;
// items pushed into the next-level queue are consumed in the same launch.
// Per level:
//   phase 1  classify every item, expand take-all items, fill the lists
//   phase 2  warp list, hub list and pair list, back to back (no barrier:
//            a warp that runs out of one list starts on the next)
//   phase 3  refill list (pair items that need a rebuild, a warp each) and
//            the retry list (hub rebuilds, a CTA each)
// separated by grid barriers.  A barrier counts arriving CTAs (a counter per
// barrier, zero at launch, so none is ever reset) and waits with a bounded
// spin: if it expires, the error flag is set and the warp goes on, so a
// failure ends the launch with an error instead of a hang.  Each level's
// counters live in a block of their own, cleared once before the launch.
// Host-buffer jobs post the running edge count after every level, as the
// per-level launches do.
#pragma once

#include "kernels_fast.cuh"

namespace csaw {

constexpr int PERSIST_MAX_LEVELS = 4;
constexpr int PERSIST_BARRIER_SPINS = 1 << 23;   // polls, ~128 ns apart: about a second

enum : uint32_t { PF_HUB = 1u, PF_PAIR = 2u, PF_RETRY = 4u };

// Counters of one level of a persistent job (cleared before the launch).
struct PersistLevelCtr {
    uint32_t n_out;      // items pushed for the next level
    uint32_t n_heavy;
    uint32_t n_sel;
    uint32_t n_cta[4];
    uint32_t n_retry;
    uint32_t n_hub;
    uint32_t n_pair;
    uint32_t n_refill;
    uint32_t n_thread;   // unused: a persistent job has no thread list
};

struct PersistArgs {
    LevelArgs lv[PERSIST_MAX_LEVELS];
    LevelArgs refill[PERSIST_MAX_LEVELS];   // lv with the refill list as its warp list
    LevelArgs retry[PERSIST_MAX_LEVELS];    // lv with the retry list as its CTA list
    uint32_t flags[PERSIST_MAX_LEVELS];
    unsigned long long *posts[PERSIST_MAX_LEVELS];   // page-locked slot for the edge count after level l, or null
    int D;
    unsigned *arrive;   // [3 * D] CTA arrivals per barrier
    int *err;
};

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned *p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Every CTA of the grid arrives at `arrive` (zero before the first
// arrival) once all its warps are done; returns once all CTAs have, or sets
// ERR_BARRIER after the bounded wait.
__device__ __forceinline__ void grid_barrier(unsigned *arrive, unsigned nblocks, int *err) {
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        atomicAdd(arrive, 1u);
        int spins = 0;
        while (ld_acquire_u32(arrive) < nblocks) {
            if (++spins > PERSIST_BARRIER_SPINS) {
                atomicOr(err, ERR_BARRIER);
                break;
            }
            __nanosleep(64);
        }
        __threadfence();
    }
    __syncthreads();
}

// Bytes of dynamic shared memory of k_persist: the pair pass's row windows,
// entry slots and barriers.
constexpr size_t PERSIST_SMEM =
    sizeof(float) * PAIR_HALVES * (PAIR_ROW + PAIR_ENT) + sizeof(uint64_t) * PAIR_HALVES;

// The passes: the frequent ones inlined into the one kernel, the hub and
// CTA-retry passes (rare, with large state of their own) as calls, so their
// registers do not weigh on the inlined loops.
template <typename I, int BIAS>
__device__ __forceinline__ void call_coop(const DevGraph &g, const LevelArgs &a) {
    coop_body<I, BIAS>(g, a);
}
template <typename I, int BIAS, bool CACHED>
__device__ __forceinline__ void call_select(const DevGraph &g, const LevelArgs &a) {
    select_fast_body<I, BIAS, CACHED>(g, a);
}
template <typename I, int BIAS>
__device__ __noinline__ void call_hub(const DevGraph &g, const LevelArgs &a) {
    hub_body<I, BIAS>(g, a);
}
template <typename I, int BIAS>
__device__ __forceinline__ void call_pair(const DevGraph &g, const LevelArgs &a, float *buf, float *ebuf,
                                       uint64_t *bar, uint32_t &parity) {
    pair_body<I, BIAS>(g, a, buf, ebuf, bar, parity);
}
template <typename I, int BIAS>
__device__ __noinline__ void call_heavy(const DevGraph &g, const LevelArgs &a) {
    heavy_body<I, BIAS>(g, a);
}

#ifndef CSAW_PERSIST_MIN_BLOCKS
#define CSAW_PERSIST_MIN_BLOCKS 4
#endif

template <typename I, int BIAS>
__global__ void __launch_bounds__(FAST_THREADS, CSAW_PERSIST_MIN_BLOCKS)
k_persist(const __grid_constant__ DevGraph g, const __grid_constant__ PersistArgs pa) {
    constexpr bool BIASED = BIAS != CSAW_BIAS_UNBIASED;
    extern __shared__ float s_heavy[];   // the same dynamic region heavy_body names (unused by it here)
    float *pairP = s_heavy;
    float *pairE = s_heavy + PAIR_HALVES * PAIR_ROW;
    uint64_t *bars = reinterpret_cast<uint64_t *>(pairE + PAIR_HALVES * PAIR_ENT);
    const int hid = threadIdx.x >> 4;
    if (BIASED) {
        if ((threadIdx.x & 15) == 0) mbar_init(bars + hid);
        mbar_init_fence();
    }
    __syncthreads();
    uint32_t parity = 0;
    const unsigned nblocks = gridDim.x;
    int k = 0;
    for (int l = 0; l < pa.D; ++l) {
        const uint32_t fl = pa.flags[l];
        call_coop<I, BIAS>(g, pa.lv[l]);
        grid_barrier(pa.arrive + k++, nblocks, pa.err);
        call_select<I, BIAS, BIASED>(g, pa.lv[l]);
        if (fl & PF_HUB) call_hub<I, BIAS>(g, pa.lv[l]);
        if (BIASED && (fl & PF_PAIR))
            call_pair<I, BIAS>(g, pa.lv[l], pairP + hid * PAIR_ROW, pairE + hid * PAIR_ENT, bars + hid, parity);
        grid_barrier(pa.arrive + k++, nblocks, pa.err);
        if (BIASED && (fl & PF_PAIR)) call_select<I, BIAS, true>(g, pa.refill[l]);
        if (fl & PF_RETRY) {
            __syncthreads();   // the whole CTA enters the retry pass
            call_heavy<I, BIAS>(g, pa.retry[l]);
        }
        if (l + 1 < pa.D || pa.posts[l]) grid_barrier(pa.arrive + k++, nblocks, pa.err);
        if (pa.posts[l] && blockIdx.x == 0 && threadIdx.x == 0) {   // this level's edges are final
            *(volatile unsigned long long *)pa.posts[l] = *(volatile unsigned long long *)pa.lv[l].o_count;
            __threadfence_system();
        }
    }
}

}  // namespace csaw
