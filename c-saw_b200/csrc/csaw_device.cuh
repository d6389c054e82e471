// csaw_device.cuh -- device primitives of the csaw-b200 sampler (sm_100a).
//
// Every float operation here is one IEEE round-to-nearest add, multiply or
// max, in the canonical order documented in csaw_internal.h, so the CUDA path
// is bit-identical to the CPU restatement of the same semantics.  The library
// is built with --fmad=false as a second guard against FMA contraction.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "csaw.h"
#include "csaw_api.cuh"
#include "csaw_internal.h"

namespace csaw {

constexpr unsigned FULL = 0xffffffffu;

// --------------------------------------------------------------- graph view
// Per-edge neighbor record (batched schedules): the column of edge e with the
// row begin and degree of that column vertex, one 16-byte record, so a
// selected edge costs one 32-byte sector and one 128-bit load for its
// neighbor, its adjacency range and its degree.
struct __align__(16) NbrRec {
    int32_t col;
    int32_t deg;
    long long beg;
};

static_assert(sizeof(NbrRec) == 16, "one 128-bit load per record");

__device__ __forceinline__ NbrRec load_rec(const NbrRec *r, int64_t e) {
    const int4 x = __ldg(reinterpret_cast<const int4 *>(r) + e);
    NbrRec o;
    o.col = x.x;
    o.deg = x.y;
    o.beg = (long long)(((unsigned long long)(uint32_t)x.w << 32) | (uint32_t)x.z);
    return o;
}

struct DevGraph {
    csaw_graph_view v;     // what the user hooks see
    const float *ebias;    // materialised neighbor degree per edge, or null
    const float *cdf;      // canonical per-vertex prefix of cdf_bias, or null
    const float *cdf1;     // cdf[32k + 31] (search index, level 1), with cdf
    const float *cdf2;     // cdf[1024u + 1023] (search index, level 2), with cdf
    int cdf_bias;          // bias kind the cdf was built for
    // Per-edge neighbor records (batched schedules): a selected neighbor
    // carries its own adjacency range, so the next expansion or walk step
    // skips the dependent rowptr loads.
    const NbrRec *nrec;    // [E] or null
    // Tile summaries of rows above TSC_MIN_DEG edges, with cdf (same bias):
    // for each 32-edge tile t of the row (row-aligned, as the canonical
    // prefix tiles it), x = the tile's Kogge-Stone total and y = the maximum
    // of its in-tile scan over the row's edges, at tsc_slot(beg, v) + t.
    const float2 *tsc;     // or null
};

// Rows with more edges than this have tile summaries (the rows a CTA retry
// can get: above the warp passes' shared-memory prefix of 512).
constexpr int64_t TSC_MIN_DEG = 512;

// First summary slot of row (v, beg).  Slots of different rows never meet:
// row v's last tile sits at or below (beg_next >> 5) + v, the next row's
// first at (beg_next >> 5) + v + 1 or above, so E / 32 + V + 1 slots cover
// every row.
__device__ __forceinline__ int64_t tsc_slot(int64_t beg, int32_t v) { return (beg >> 5) + (int64_t)v; }

template <typename I>
__device__ __forceinline__ int64_t row_begin(const DevGraph &g, int64_t v) {
    return (int64_t)__ldg(((const I *)g.v.rowptr) + v);
}

template <typename I>
__device__ __forceinline__ float degree_f(const DevGraph &g, int32_t u) {
    const I *r = (const I *)g.v.rowptr;
    return __ll2float_rn((long long)(__ldg(r + u + 1) - __ldg(r + u)));
}

// Bias of edge e (neighbor col[e]) for the bias kind BIAS.
template <typename I, int BIAS>
__device__ __forceinline__ float edge_bias(const DevGraph &g, int64_t e) {
    if constexpr (BIAS == CSAW_BIAS_EDGE_WEIGHT) {
        return __ldg(g.v.weight + e);
    } else if constexpr (BIAS == CSAW_BIAS_DEGREE) {
        if (g.nrec) return __int2float_rn(__ldg(&g.nrec[e].deg));
        if (g.ebias) return __ldg(g.ebias + e);
        return degree_f<I>(g, __ldg(g.v.col + e));
    } else {
        return EdgeBias(__ldg(g.v.col + e), e, &g.v);
    }
}

// ------------------------------------------------------------------- Philox
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC11).
__device__ __forceinline__ uint4 philox(uint4 c, uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        uint32_t hi0 = __umulhi(0xD2511F53u, c.x), lo0 = 0xD2511F53u * c.x;
        uint32_t hi1 = __umulhi(0xCD9E8D57u, c.z), lo1 = 0xCD9E8D57u * c.z;
        c = make_uint4(hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0);
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    return c;
}

__device__ __forceinline__ uint32_t word_of(uint4 b, int w) {
    return w == 0 ? b.x : (w == 1 ? b.y : (w == 2 ? b.z : b.w));
}

__device__ __forceinline__ float unit24(uint32_t x) {
    return __fmul_rn(__uint2float_rn(x >> 8), 5.9604644775390625e-8f);
}

__device__ __forceinline__ uint32_t mulhi(uint32_t x, uint32_t n) { return __umulhi(x, n); }

// t = unit(x) * T, kept strictly below T.
__device__ __forceinline__ float its_target(uint32_t x, float T) {
    float t = __fmul_rn(unit24(x), T);
    if (!(t < T)) t = __int_as_float(__float_as_int(T) - 1);
    return t;
}

// First i in [0, d) with P[i] > t (P monotone, P[d-1] > t).
__device__ __forceinline__ int64_t search_upper(const float *P, int64_t d, float t) {
    int64_t lo = 0, hi = d - 1;
    while (lo < hi) {
        int64_t mid = (lo + hi) >> 1;
        if (P[mid] > t) hi = mid; else lo = mid + 1;
    }
    return lo;
}

// search_upper for rows held in shared memory (d < 2^31): 32-bit indices.
__device__ __forceinline__ int search_upper32(const float *P, int d, float t) {
    int lo = 0, hi = d - 1;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (P[mid] > t) hi = mid; else lo = mid + 1;
    }
    return lo;
}

// The same index by binary lifting in a fixed LOG steps, for d <= 2^LOG: no
// data-dependent loop (lanes and half-warps searching rows of different
// lengths stay converged); the last element is never read.
template <int LOG>
__device__ __forceinline__ int search_upper_lift(const float *P, int d, float t) {
    int lo = 0;
#pragma unroll
    for (int step = 1 << (LOG - 1); step >= 1; step >>= 1) {
        const int idx = lo + step - 1;
        if (idx < d - 1 && !(P[idx] > t)) lo += step;
    }
    return lo;
}

// warp_search_upper over an array this CTA wrote earlier in the launch
// (shared or global memory): plain loads instead of the read-only path.
__device__ __forceinline__ int64_t warp_search_upper_rw(const float *P, int64_t d, float t, int lane) {
    int64_t lo = 0, hi = d;   // the answer lies in [lo, hi)
    while (hi - lo > 32) {
        const int64_t step = (hi - lo + 31) >> 5;
        const int64_t idx = lo + (int64_t)(lane + 1) * step - 1;
        const bool up = idx >= hi - 1 || P[idx] > t;
        const int k = __ffs(__ballot_sync(FULL, up)) - 1;
        const int64_t nlo = lo + (int64_t)k * step;
        hi = nlo + step < hi ? nlo + step : hi;
        lo = nlo;
    }
    const int64_t idx = lo + lane;
    const bool up = idx >= hi - 1 || P[idx] > t;
    return lo + __ffs(__ballot_sync(FULL, up)) - 1;
}

// The same index for one warp-uniform target, found by the whole warp with a
// 32-way search: each round probes the last element of 32 equal chunks of the
// remaining range and keeps the first chunk whose probe exceeds t, so a
// degree-d search takes about log32(d) dependent loads instead of log2(d).
__device__ __forceinline__ int64_t warp_search_upper(const float *P, int64_t d, float t, int lane) {
    int64_t lo = 0, hi = d;   // the answer lies in [lo, hi)
    while (hi - lo > 32) {
        const int64_t step = (hi - lo + 31) >> 5;
        const int64_t idx = lo + (int64_t)(lane + 1) * step - 1;
        const bool up = idx >= hi - 1 || __ldg(P + idx) > t;
        const int k = __ffs(__ballot_sync(FULL, up)) - 1;
        const int64_t nlo = lo + (int64_t)k * step;
        hi = nlo + step < hi ? nlo + step : hi;
        lo = nlo;
    }
    const int64_t idx = lo + lane;
    const bool up = idx >= hi - 1 || __ldg(P + idx) > t;
    return lo + (__ffs(__ballot_sync(FULL, up)) - 1);
}

// First i in [0, d) with P[i] > t for the row of global edge offset beg of a
// cached prefix, through its two index levels: a binary search of the
// row's 1024-edge groups in cdf2 (E/1024 floats, L2-resident), then of the
// group's 32-edge tiles in cdf1 and of the tile in cdf (each one 128-byte
// line).  Every probe lies inside the row; the last candidate of each level
// is known to exceed t (it ends the row, or ends the previous level's pick).
__device__ __forceinline__ int64_t cdf_search(const DevGraph &g, int64_t beg, int64_t d, float t) {
    const int64_t end = beg + d;
    const int64_t ua = beg >> 10, ub = (end - 1) >> 10;
    const int64_t u = ua + search_upper(g.cdf2 + ua, ub - ua + 1, t);
    const int64_t ka = (u << 5) > (beg >> 5) ? (u << 5) : (beg >> 5);
    const int64_t kb = (u << 5) + 31 < ((end - 1) >> 5) ? (u << 5) + 31 : ((end - 1) >> 5);
    const int64_t k = ka + search_upper(g.cdf1 + ka, kb - ka + 1, t);
    const int64_t ia = (k << 5) > beg ? (k << 5) : beg;
    const int64_t ib = (k << 5) + 31 < end - 1 ? (k << 5) + 31 : end - 1;
    return ia + search_upper(g.cdf + ia, ib - ia + 1, t) - beg;
}

// The same with one warp-uniform target, each level by warp_search_upper.
__device__ __forceinline__ int64_t warp_cdf_search(const DevGraph &g, int64_t beg, int64_t d, float t, int lane) {
    const int64_t end = beg + d;
    const int64_t ua = beg >> 10, ub = (end - 1) >> 10;
    const int64_t u = ua + warp_search_upper(g.cdf2 + ua, ub - ua + 1, t, lane);
    const int64_t ka = (u << 5) > (beg >> 5) ? (u << 5) : (beg >> 5);
    const int64_t kb = (u << 5) + 31 < ((end - 1) >> 5) ? (u << 5) + 31 : ((end - 1) >> 5);
    const int64_t k = ka + warp_search_upper(g.cdf1 + ka, kb - ka + 1, t, lane);
    const int64_t ia = (k << 5) > beg ? (k << 5) : beg;
    const int64_t ib = (k << 5) + 31 < end - 1 ? (k << 5) + 31 : end - 1;
    return ia + warp_search_upper(g.cdf + ia, ib - ia + 1, t, lane) - beg;
}

// ------------------------------------------------------------ warp scans
__device__ __forceinline__ float warp_ks_sum(float v, int lane) {
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        float up = __shfl_up_sync(FULL, v, off);
        if (lane >= off) v = __fadd_rn(v, up);
    }
    return v;
}

__device__ __forceinline__ float warp_max_scan(float v, int lane) {
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        float up = __shfl_up_sync(FULL, v, off);
        if (lane >= off) v = fmaxf(v, up);
    }
    return v;
}

// Canonical prefix of wfn(0..d) into P[0..d) computed by one warp; elements
// whose bit is set in zmask (if given) count as 0.  Returns T = P[d-1] on
// every lane.  P may live in shared or global memory.
template <typename WFn>
__device__ float warp_canon_prefix(WFn wfn, int64_t d, float *P, const uint32_t *zmask, int lane) {
    const int64_t ntiles = (d + 31) >> 5;
    float C = 0.f, runmax = 0.f;
    for (int64_t g0 = 0; g0 < ntiles; g0 += 32) {
        const int gt = (ntiles - g0) < 32 ? (int)(ntiles - g0) : 32;
        float my_tsum = 0.f;
        for (int tt = 0; tt < gt; ++tt) {
            int64_t i = ((g0 + tt) << 5) + lane;
            float w = 0.f;
            if (i < d) {
                w = wfn(i);
                if (zmask && ((zmask[i >> 5] >> (i & 31)) & 1u)) w = 0.f;
            }
            float v = warp_ks_sum(w, lane);
            if (i < d) P[i] = v;
            float s = __shfl_sync(FULL, v, 31);
            if (lane == tt) my_tsum = s;
        }
        float q = warp_ks_sum(my_tsum, lane);
        float qex = __shfl_up_sync(FULL, q, 1);
        if (lane == 0) qex = 0.f;
        float gtot = __shfl_sync(FULL, q, 31);
        __syncwarp();
        for (int tt = 0; tt < gt; ++tt) {
            int64_t i = ((g0 + tt) << 5) + lane;
            float qx = __shfl_sync(FULL, qex, tt);
            float p = 0.f;
            if (i < d) p = __fadd_rn(C, __fadd_rn(qx, P[i]));
            p = fmaxf(warp_max_scan(p, lane), runmax);
            if (i < d) P[i] = p;
            runmax = __shfl_sync(FULL, p, 31);
        }
        C = __fadd_rn(C, gtot);
    }
    __syncwarp();
    return runmax;
}

// Same canonical prefix computed by a whole CTA (all threads must call).
// Scratch: tsum[ntiles], gcar[ngroups] (shared or global).
template <typename WFn>
__device__ float cta_canon_prefix(WFn wfn, int64_t d, float *P, float *tsum, float *gcar,
                                  const uint32_t *zmask) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int64_t ntiles = (d + 31) >> 5, ngroups = (ntiles + 31) >> 5;
    for (int64_t t = warp; t < ntiles; t += nw) {
        int64_t i = (t << 5) + lane;
        float w = 0.f;
        if (i < d) {
            w = wfn(i);
            if (zmask && ((zmask[i >> 5] >> (i & 31)) & 1u)) w = 0.f;
        }
        float v = warp_ks_sum(w, lane);
        if (i < d) P[i] = v;
        if (lane == 31) tsum[t] = v;
    }
    __syncthreads();
    for (int64_t gg = warp; gg < ngroups; gg += nw) {
        int64_t t = (gg << 5) + lane;
        float s = t < ntiles ? tsum[t] : 0.f;
        float q = warp_ks_sum(s, lane);
        float qex = __shfl_up_sync(FULL, q, 1);
        if (lane == 0) qex = 0.f;
        __syncwarp();
        if (t < ntiles) tsum[t] = qex;
        if (lane == 31) gcar[gg] = q;
    }
    __syncthreads();
    if (warp == 0) {
        // serial carry across groups, in group order (C += total of group g):
        // the warp loads 32 group totals at a time and folds them by shuffles,
        // every lane carrying the same C; lane k keeps the carry into group g0+k
        float C = 0.f;
        for (int64_t g0 = 0; g0 < ngroups; g0 += 32) {
            const int64_t gg = g0 + lane;
            const float tot = gg < ngroups ? gcar[gg] : 0.f;
            const int m = ngroups - g0 < 32 ? (int)(ngroups - g0) : 32;
            float mine = 0.f;
            for (int k = 0; k < m; ++k) {
                if (lane == k) mine = C;
                C = __fadd_rn(C, __shfl_sync(FULL, tot, k));
            }
            if (gg < ngroups) gcar[gg] = mine;
        }
    }
    __syncthreads();
    for (int64_t t = warp; t < ntiles; t += nw) {
        int64_t i = (t << 5) + lane;
        float C = gcar[t >> 5], qx = tsum[t];
        float p = 0.f;
        if (i < d) p = __fadd_rn(C, __fadd_rn(qx, P[i]));
        p = warp_max_scan(p, lane);
        if (i < d) P[i] = p;
        __syncwarp();
        if (lane == 31) tsum[t] = p;
    }
    __syncthreads();
    {
        // exclusive running max of the tile maxima.  max is exact, so the
        // warps scan contiguous ranges in parallel: range maxima first, then
        // each range from the max of the ranges before it.
        __shared__ float s_rmax[32];
        const int64_t per = (ntiles + nw - 1) / nw;
        const int64_t t0 = (int64_t)warp * per, t1 = t0 + per < ntiles ? t0 + per : ntiles;
        float rmax = 0.f;
        for (int64_t t = t0 + lane; t < t1; t += 32) rmax = fmaxf(rmax, tsum[t]);
#pragma unroll
        for (int off = 16; off; off >>= 1) rmax = fmaxf(rmax, __shfl_xor_sync(FULL, rmax, off));
        if (lane == 0) s_rmax[warp] = rmax;
        __syncthreads();
        float carry = 0.f;
        for (int w = 0; w < warp; ++w) carry = fmaxf(carry, s_rmax[w]);
        for (int64_t base = t0; base < t1; base += 32) {
            const int64_t t = base + lane;
            const float m = t < t1 ? tsum[t] : 0.f;
            const float ms = warp_max_scan(m, lane);
            float ex = __shfl_up_sync(FULL, ms, 1);
            if (lane == 0) ex = 0.f;
            ex = fmaxf(ex, carry);
            __syncwarp();
            if (t < t1) tsum[t] = ex;
            carry = fmaxf(carry, __shfl_sync(FULL, ms, 31));
        }
    }
    __syncthreads();
    for (int64_t t = warp; t < ntiles; t += nw) {
        int64_t i = (t << 5) + lane;
        if (i < d) P[i] = fmaxf(P[i], tsum[t]);
    }
    __syncthreads();
    return P[d - 1];
}

// ------------------------------------------------------------- selection
// Draw words of one slot: word A of slot `slot` of item (p, s, l).
struct DrawCtx {
    uint32_t k0, k1, p, s, l;
};

struct SlotRng {
    uint4 blk;
    int blk_id = -1;
    __device__ __forceinline__ uint32_t word(const DrawCtx &dc, int slot, int A) {
        if ((A >> 2) != blk_id) {
            blk = philox(make_uint4(dc.p, dc.s, (TAG_SAMPLE << 24) | dc.l,
                                    ((uint32_t)slot << 16) | (uint32_t)(A >> 2)),
                         dc.k0, dc.k1);
            blk_id = A >> 2;
        }
        return word_of(blk, A & 3);
    }
};

// Resolver state of the warp-parallel sequential-order selection: lane j owns
// slot j.  j (current slot) and a (draws in this phase for slot j) are warp
// uniform; A (draws used by the lane's slot), cand and sel are per lane.
struct SelState {
    int j = 0, a = 1, A = 0;
    int cand = -1, sel = -1;
};

// cand_of(x, act) maps a draw word to a neighbor offset; it is called by all
// lanes together, and only lanes with act set use the result.
// Runs slots in order until all N are accepted (returns 0) or the current slot
// has exhausted its REJECT_ATTEMPTS draws in this phase (returns 1: rebuild).
// A slot that has used MAX_SLOT_DRAWS draws takes the smallest unselected
// index, so the loop always ends.
template <typename CandFn>
__device__ __forceinline__ int resolve_slots(SelState &st, int N, int lane, const DrawCtx &dc,
                                             SlotRng &rng, CandFn cand_of) {
    while (st.j < N) {
        // Accept in one step the run of slots j, j+1, ... whose current
        // candidates repeat no lower slot's value (lanes below j hold their
        // selections); the sequential order would accept each in turn.
        const int j0 = st.j;
        const int v = lane < j0 ? st.sel : (lane < N ? st.cand : -2 - lane);
        const unsigned same = __match_any_sync(FULL, v);
        const bool dup = lane >= j0 && lane < N && (same & ((1u << lane) - 1u)) != 0u;
        const unsigned db = __ballot_sync(FULL, dup);
        const int j = db ? __ffs(db) - 1 : N;
        if (lane >= j0 && lane < j) st.sel = v;
        if (j == N) {
            st.j = N;
            st.a = 1;
            return 0;
        }
        if (j > j0) st.a = 1;   // slot j rejects its first draw of this phase
        st.j = j;
        if (__shfl_sync(FULL, st.A, j) == MAX_SLOT_DRAWS) {
            int i = 0;
            while (__ballot_sync(FULL, lane < j && st.sel == i)) ++i;
            if (lane == j) st.sel = i;
            st.j = j + 1;
            st.a = 1;
            continue;
        }
        if (st.a == REJECT_ATTEMPTS) return 1;
        const bool me = lane == j;
        const uint32_t x = me ? rng.word(dc, lane, st.A) : 0u;
        const int nc = cand_of(x, me);  // warp-uniform call (may shuffle)
        if (me) {
            st.cand = nc;
            st.A++;
        }
        st.a++;
    }
    return 0;
}

// First draws of slots lanes [from, N): the lane `from` continues with its
// next draw index, later lanes (re)draw their index-0 word on the current
// prefix.  Warp-uniform.
template <typename CandFn>
__device__ __forceinline__ void draw_pending(SelState &st, int from, int N, int lane, const DrawCtx &dc,
                                             SlotRng &rng, CandFn cand_of) {
    const bool act = lane >= from && lane < N;
    const int A = lane == from ? st.A : 0;
    const uint32_t x = act ? rng.word(dc, lane, A) : 0u;
    const int c = cand_of(x, act);
    if (act) {
        st.cand = c;
        st.A = A + 1;
    }
    st.a = 1;
}

// Zero-mass fill: slots j..N-1 take the smallest indices not yet selected.
__device__ __forceinline__ void zero_fill(SelState &st, int N, int lane) {
    int i = 0;
    for (int jj = st.j; jj < N; ++jj) {
        while (__ballot_sync(FULL, lane < jj && st.sel == i)) ++i;
        if (lane == jj) st.sel = i;
        ++i;
    }
    st.j = N;
}

// Sorted copy of the selections of lanes < j into zs[0..j) (unbiased phases).
__device__ __forceinline__ void sort_selected(const SelState &st, int j, int *zs, int lane) {
    int rank = 0;
    for (int m = 0; m < j; ++m) {
        int sm = __shfl_sync(FULL, st.sel, m);
        if (sm < st.sel) ++rank;
    }
    __syncwarp();
    if (lane < j) zs[rank] = st.sel;
    __syncwarp();
}

// Index of the t-th (0-based) element of [0, d) not in the sorted zs[0..nZ).
__device__ __forceinline__ int kth_not_excluded(uint32_t t, const int *zs, int nZ) {
    for (int m = 0; m < nZ; ++m)
        if ((uint32_t)zs[m] <= t) ++t;
    return (int)t;
}

// ----------------------------------------------------------- staged output
// Per-warp staging of output edges in shared memory; one atomic per flush.
struct OutArgs {
    int32_t *src, *dst, *smp, *dep;
    unsigned long long *count;
    int64_t cap;
};

constexpr int STAGE = 64;

struct WarpStage {
    int32_t *s_src, *s_dst, *s_smp, *s_dep;  // STAGE entries each (shared)
    int cnt = 0;

    __device__ __forceinline__ void flush(const OutArgs &o, int lane) {
        if (cnt == 0) return;
        unsigned long long base = 0;
        if (lane == 0) base = atomicAdd(o.count, (unsigned long long)cnt);
        base = __shfl_sync(FULL, base, 0);
        for (int i = lane; i < cnt; i += 32) {
            int64_t pos = (int64_t)base + i;
            if (pos < o.cap) {
                o.src[pos] = s_src[i];
                o.dst[pos] = s_dst[i];
                if (o.smp) o.smp[pos] = s_smp[i];
                if (o.dep) o.dep[pos] = s_dep[i];
            }
        }
        cnt = 0;
        __syncwarp();
    }

    __device__ __forceinline__ void push(const OutArgs &o, bool act, int32_t u, int32_t v, int32_t s,
                                         int32_t l, int lane) {
        unsigned m = __ballot_sync(FULL, act);
        int n = __popc(m);
        if (n == 0) return;
        if (cnt + n > STAGE) flush(o, lane);
        if (act) {
            int pos = cnt + __popc(m & ((1u << lane) - 1u));
            s_src[pos] = u;
            s_dst[pos] = v;
            s_smp[pos] = s;
            s_dep[pos] = l;
        }
        cnt += n;
        __syncwarp();
    }
};

}  // namespace csaw
