// kernels_fast.cuh -- batched-form level expansion and walk kernels (sm_100a).
//
// Same output as kernels_sample.cuh (the canonical prefix, draw keys and slot
// resolver are shared), scheduled for latency.  On power-law graphs most
// frontier items have d <= N and take every neighbor, so the work is a chain
// of dependent loads, not arithmetic:
//   - queue items carry their own row begin and degree, and every edge has a
//     materialised neighbor record (row begin, degree of col[e]), so a pushed
//     child or a walk's next vertex needs no rowptr round trip;
//   - a warp takes a batch of up to 32 items (lane-parallel loads), reserves
//     output and next-queue space for the whole batch with one atomic each,
//     then expands all take-all items together: lanes stride over the batch's
//     edges, find the owning item by a shuffle binary search over the
//     inclusive prefix of degrees, and issue every column load at once;
//   - items with d > N are selected one at a time by the whole warp: biases,
//     prefix and column ids in registers when d <= 32 (shuffle scans and a
//     5-step shuffle search), biases preloaded into shared memory in batches
//     of 8 tiles when d <= WF, the CTA kernel beyond;
//   - batch size shrinks on small levels so every warp gets work.
#pragma once

#include "bulk_copy.cuh"
#include "kernels_sample.cuh"

namespace csaw {

constexpr int WF = 512;  // per-warp shared prefix capacity of the fast kernels
// Resident CTAs per SM the pair kernel is compiled for (register budget).
#ifndef CSAW_PAIR_MIN_BLOCKS
#define CSAW_PAIR_MIN_BLOCKS 4
#endif
// Cached items with N <= 16 and d >= this many times N go to the pair pass
// (3: a phase-1 rejection is rare enough that its refill stays cheap).
#ifndef CSAW_PAIR_MIN_RATIO
#define CSAW_PAIR_MIN_RATIO 3
#endif

constexpr int FAST_THREADS = 256;

// Canonical prefix of a single tile held one element per lane (w = 0 for
// lanes >= d): identical to warp_canon_prefix for d <= 32.
__device__ __forceinline__ float tile_prefix(float w, int d, int lane) {
    float v = warp_ks_sum(w, lane);
    float p = lane < d ? __fadd_rn(0.f, __fadd_rn(0.f, v)) : 0.f;
    return fmaxf(warp_max_scan(p, lane), 0.f);
}

// First lane whose P exceeds t (P monotone across lanes, P[31] > t).
__device__ __forceinline__ int shfl_search(float P, float t) {
    int lo = 0;
#pragma unroll
    for (int s = 16; s >= 1; s >>= 1) {
        float pv = __shfl_sync(FULL, P, lo + s - 1);
        if (!(pv > t)) lo += s;
    }
    return lo;
}

// First lane whose inclusive count exceeds e (incl monotone, incl[31] > e).
__device__ __forceinline__ int shfl_search_int(int incl, int e) {
    int lo = 0;
#pragma unroll
    for (int s = 16; s >= 1; s >>= 1) {
        int pv = __shfl_sync(FULL, incl, lo + s - 1);
        if (!(pv > e)) lo += s;
    }
    return lo;
}

__device__ __forceinline__ int warp_incl_scan(int x, int lane) {
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        int up = __shfl_up_sync(FULL, x, off);
        if (lane >= off) x += up;
    }
    return x;
}

// Neighbor of edge e with its row begin and degree: one 128-bit record load
// with the neighbor records, else the column and two rowptr loads.
template <typename I>
__device__ __forceinline__ NbrRec edge_rec(const DevGraph &g, int64_t e) {
    if (g.nrec) return load_rec(g.nrec, e);
    NbrRec r;
    r.col = __ldg(g.v.col + e);
    r.beg = row_begin<I>(g, r.col);
    r.deg = (int32_t)(row_begin<I>(g, r.col + 1) - r.beg);
    return r;
}

// Row begin and degree of u = Update(col[e]): the record's when Update kept
// the neighbor, else from rowptr.
template <typename I>
__device__ __forceinline__ void row_of(const DevGraph &g, const NbrRec &r, int32_t u, int64_t &beg, int32_t &deg) {
    if (u == r.col) {
        beg = r.beg;
        deg = r.deg;
    } else {
        beg = row_begin<I>(g, u);
        deg = (int32_t)(row_begin<I>(g, u + 1) - beg);
    }
}

// Loads the biases of edges [beg, beg+d) into W, 8 tiles per round trip.
template <typename I, int BIAS>
__device__ __forceinline__ void preload_bias(const DevGraph &g, int64_t beg, int d, float *W, int lane) {
    for (int i0 = 0; i0 < d; i0 += 256) {
        float r[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            int i = i0 + u * 32 + lane;
            r[u] = i < d ? edge_bias<I, BIAS>(g, beg + i) : 0.f;
        }
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            int i = i0 + u * 32 + lane;
            if (i < d) W[i] = r[u];
        }
    }
    __syncwarp();
}

// Speculative resolver of the batched kernels (same result as resolve_slots).
// A rejection phase allows REJECT_ATTEMPTS = 4 draws per slot, and the four
// words of one Philox block are exactly the next four draws of a slot, so
// every pending lane computes the candidates of its next four draws at once
// (four independent searches, overlapped) and a rejected draw costs one
// shuffle and one ballot instead of a serial search.
struct Spec4 {
    int j = 0, a = 1;   // warp uniform: current slot, draws it used in this window
    int have = 4;       // warp uniform: candidates computed ahead per lane (4, or 1 when lazy)
    int base = 0;       // lane: draw index of c0 (a multiple of 4)
    int sel = -1;
    int c0 = -1, c1 = -1, c2 = -1, c3 = -1;
    __device__ __forceinline__ int pick(int k) const { return k == 0 ? c0 : (k == 1 ? c1 : (k == 2 ? c2 : c3)); }
};

// Windows of lanes [from, N): lane `from` starts at draw from_base, later
// lanes at draw 0, all on the current prefix.  Warp-uniform.
// lazy: compute only the first candidate of each window; later ones are
// computed on demand for the rejected slot (for costly searches where a
// rejection is rare, e.g. d >= 4N).
template <typename CandFn>
__device__ __forceinline__ void spec_fill(Spec4 &st, int from, int N, int lane, const DrawCtx &dc, SlotRng &rng,
                                          CandFn cand_of, int from_base, bool lazy) {
    const bool act = lane >= from && lane < N;
    const int base = lane == from ? from_base : 0;
    if (lazy) {
        const uint32_t x0 = act ? rng.word(dc, lane, base) : 0u;
        const int n0 = cand_of(x0, act);
        if (act) {
            st.base = base;
            st.c0 = n0;
        }
        st.have = 1;
        st.a = 1;
        return;
    }
    uint32_t x0 = 0, x1 = 0, x2 = 0, x3 = 0;
    if (act) {
        x0 = rng.word(dc, lane, base);
        x1 = rng.word(dc, lane, base + 1);
        x2 = rng.word(dc, lane, base + 2);
        x3 = rng.word(dc, lane, base + 3);
    }
    const int n0 = cand_of(x0, act), n1 = cand_of(x1, act), n2 = cand_of(x2, act), n3 = cand_of(x3, act);
    if (act) {
        st.base = base;
        st.c0 = n0;
        st.c1 = n1;
        st.c2 = n2;
        st.c3 = n3;
    }
    st.have = 4;
    st.a = 1;
}

__device__ __forceinline__ void fill_smallest(Spec4 &st, int j, int lane) {
    int i = 0;
    while (__ballot_sync(FULL, lane < j && st.sel == i)) ++i;
    if (lane == j) st.sel = i;
}

// 0: all N slots accepted; 1: slot st.j needs a phase rebuild.
template <typename CandFn>
__device__ __forceinline__ int resolve4(Spec4 &st, int N, int lane, const DrawCtx &dc, SlotRng &rng, CandFn cand_of) {
    while (st.j < N) {
        const int j = st.j, a = st.a;
        int cj;
        if (a - 1 < st.have) {
            cj = st.pick(a - 1);
        } else {   // lazy window: the rejected slot's next draw, on its lane
            const bool me = lane == j;
            cj = cand_of(me ? rng.word(dc, lane, st.base + a - 1) : 0u, me);
        }
        // Accept in one step the run of slots j, j+1, ... whose current
        // candidates repeat no lower slot's value: lanes below j hold their
        // selections, lane j its draw a, lanes above their first draw (the
        // sequential order would accept each of them in turn).  f is the first
        // slot whose candidate repeats a lower one.
        const int v = lane < j ? st.sel : (lane == j ? cj : (lane < N ? st.c0 : -2 - lane));
        const unsigned same = __match_any_sync(FULL, v);
        const bool dup = lane >= j && lane < N && (same & ((1u << lane) - 1u)) != 0u;
        const unsigned db = __ballot_sync(FULL, dup);
        const int f = db ? __ffs(db) - 1 : N;
        if (lane >= j && lane < f) st.sel = v;
        if (f == N) {
            st.j = N;
            st.a = 1;
            return 0;
        }
        // slot f's current draw (draw a of slot j, or the first of a later slot) is rejected
        const int af = f == j ? a : 1;
        st.j = f;
        if (__shfl_sync(FULL, st.base, f) + af == MAX_SLOT_DRAWS) {
            fill_smallest(st, f, lane);
            st.j = f + 1;
            st.a = 1;
            continue;
        }
        st.a = af;
        if (af == REJECT_ATTEMPTS) return 1;
        st.a = af + 1;
    }
    return 0;
}

// Generic driver: cand_of(x, act) maps a draw word to a candidate (warp-
// uniform call); rebuild(st, j) zeroes the selections of slots < j out of the
// prefix and returns false when no positive mass is left.
// j0 > 0 resumes an item whose first phase failed at slot j0 (lane m < j0
// passes its accepted index in sel0): slot j0 has used its draws
// 0..REJECT_ATTEMPTS-1, so the run goes on exactly as it would after that
// phase -- rebuild without the j0 selections, slot j0 from draw
// REJECT_ATTEMPTS, later slots from draw 0.
template <typename CandFn, typename RebuildFn>
__device__ __forceinline__ int select_spec(int N, int lane, const DrawCtx &dc, bool zero, CandFn cand_of,
                                           RebuildFn rebuild, bool lazy = false, int j0 = 0, int sel0 = -1) {
    SlotRng rng;
    Spec4 st;
    if (j0 > 0) {
        st.j = j0;
        st.sel = lane < j0 ? sel0 : -1;
        if (!rebuild(st, j0)) zero = true;
        else spec_fill(st, j0, N, lane, dc, rng, cand_of, REJECT_ATTEMPTS, lazy);
    } else if (!zero) {
        spec_fill(st, 0, N, lane, dc, rng, cand_of, 0, lazy);
    }
    for (;;) {
        if (zero) {
            for (int jj = st.j; jj < N; ++jj) fill_smallest(st, jj, lane);
            break;
        }
        if (resolve4(st, N, lane, dc, rng, cand_of) == 0) break;
        const int j = st.j;
        const int next = __shfl_sync(FULL, st.base, j) + REJECT_ATTEMPTS;
        if (!rebuild(st, j)) {
            zero = true;
            continue;
        }
        spec_fill(st, j, N, lane, dc, rng, cand_of, next, lazy);
    }
    return st.sel;
}

// Selection for N < d <= 32 entirely in registers.
template <typename I, int BIAS>
__device__ __forceinline__ int select_reg(const DevGraph &g, int64_t beg, int d, int N, const DrawCtx &dc,
                                          int lane) {
    const float w = lane < d ? edge_bias<I, BIAS>(g, beg + lane) : 0.f;
    float P = tile_prefix(w, d, lane);
    float T = __shfl_sync(FULL, P, 31);
    auto cand_of = [&](uint32_t x, bool act) -> int {
        const float t = act ? its_target(x, T) : 0.f;
        return shfl_search(P, t);
    };
    auto rebuild = [&](const Spec4 &st, int j) -> bool {
        const unsigned zm = __reduce_or_sync(FULL, lane < j ? (1u << st.sel) : 0u);
        P = tile_prefix(((zm >> lane) & 1u) ? 0.f : w, d, lane);
        T = __shfl_sync(FULL, P, 31);
        return T > 0.f;
    };
    return select_spec(N, lane, dc, !(T > 0.f), cand_of, rebuild);
}

// Selection for 32 < d with the canonical prefix in P (shared or a cached
// CDF); W holds the raw biases for rebuilds (shared), zb a rebuild bitmap.
__device__ __forceinline__ int select_smem(const float *W, int d, int N, const DrawCtx &dc, float *P,
                                           uint32_t *zb, int lane) {
    auto wfn = [&](int64_t i) { return W[i]; };
    float T = warp_canon_prefix(wfn, d, P, nullptr, lane);
    auto cand_of = [&](uint32_t x, bool act) -> int {
        return act ? search_upper32(P, d, its_target(x, T)) : -1;
    };
    auto rebuild = [&](const Spec4 &st, int j) -> bool {
        const int nwords = (d + 31) >> 5;
        for (int w = lane; w < nwords; w += 32) zb[w] = 0u;
        __syncwarp();
        if (lane < j) atomicOr(&zb[st.sel >> 5], 1u << (st.sel & 31));
        __syncwarp();
        T = warp_canon_prefix(wfn, d, P, zb, lane);
        return T > 0.f;
    };
    return select_spec(N, lane, dc, !(T > 0.f), cand_of, rebuild, d >= 4 * N);
}

// Selection for 32 < d <= WF from the cached canonical prefix: the row's
// prefix is copied to shared P (one coalesced pass, no scan); a rebuild reads
// the raw biases from global memory.  Same draws and result as select_smem,
// since the cache holds exactly the prefix it would compute.
template <typename I, int BIAS>
__device__ __forceinline__ int select_cached(const DevGraph &g, int64_t beg, int d, int N, const DrawCtx &dc,
                                             float *P, uint32_t *zb, int lane, int j0 = 0, int sel0 = -1) {
    const float *cp = g.cdf + beg;
    // a resumed item (j0 > 0) starts with a rebuild, which writes all of P
    for (int i0 = 0; i0 < (j0 > 0 ? 0 : d); i0 += 256) {
        float r[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int i = i0 + u * 32 + lane;
            r[u] = i < d ? __ldg(cp + i) : 0.f;
        }
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int i = i0 + u * 32 + lane;
            if (i < d) P[i] = r[u];
        }
    }
    __syncwarp();
    float T = j0 > 0 ? 1.f : P[d - 1];
    auto cand_of = [&](uint32_t x, bool act) -> int {
        return act ? search_upper32(P, d, its_target(x, T)) : -1;
    };
    auto rebuild = [&](const Spec4 &st, int j) -> bool {
        const int nwords = (d + 31) >> 5;
        for (int w = lane; w < nwords; w += 32) zb[w] = 0u;
        __syncwarp();
        if (lane < j) atomicOr(&zb[st.sel >> 5], 1u << (st.sel & 31));
        __syncwarp();
        auto wfn = [&](int64_t i) { return edge_bias<I, BIAS>(g, beg + i); };
        T = warp_canon_prefix(wfn, d, P, zb, lane);
        return T > 0.f;
    };
    return select_spec(N, lane, dc, !(T > 0.f), cand_of, rebuild, d >= 4 * N, j0, sel0);
}

// Unbiased selection (no prefix): index ranks over the non-excluded range.
__device__ __forceinline__ int select_unbiased(int64_t d, int N, const DrawCtx &dc, int *zs, int lane) {
    int nZ = 0;
    auto cand_of = [&](uint32_t x, bool act) -> int {
        return act ? kth_not_excluded(mulhi(x, (uint32_t)(d - nZ)), zs, nZ) : -1;
    };
    auto rebuild = [&](const Spec4 &st, int j) -> bool {
        int rank = 0;
        for (int m = 0; m < j; ++m) {
            const int sm = __shfl_sync(FULL, st.sel, m);
            if (sm < st.sel) ++rank;
        }
        __syncwarp();
        if (lane < j) zs[rank] = st.sel;
        __syncwarp();
        nZ = j;
        return true;
    };
    return select_spec(N, lane, dc, false, cand_of, rebuild);
}

// Seeds -> level-0 queue with row begin and degree.
template <typename I>
__global__ void k_init_queue_fast(DevGraph g, const int32_t *seeds, uint32_t n, int F, int s0, int32_t *qv,
                                  int32_t *qs, uint32_t *qp, I *qb, int32_t *qd, uint32_t *qn, int *err) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) *qn = n;
    if (i >= n) return;
    int32_t v = seeds[i];
    if (v < 0 || v >= g.v.n_vertices) {
        atomicOr(err, ERR_SEED_RANGE);
        v = 0;
    }
    const int64_t b = row_begin<I>(g, v);
    qv[i] = v;
    qs[i] = s0 + (int32_t)(i / (uint32_t)F);
    qp[i] = i % (uint32_t)F;
    qb[i] = (I)b;
    qd[i] = (int32_t)(row_begin<I>(g, v + 1) - b);
}

// Emitting an edge: emit_load reads the selected neighbor (its record on
// inner levels), emit_finish writes the output edge and, on inner levels,
// the child queue item; emit_edge does both.
template <typename I>
__device__ __forceinline__ NbrRec emit_load(const DevGraph &g, const LevelArgs &a, int64_t e) {
    NbrRec r;
    if (a.push) r = edge_rec<I>(g, e);   // the child's adjacency range comes with it
    else r.col = __ldg(g.v.col + e);     // last level: the column alone (4-byte stride over a row)
    return r;
}

// The stores of an emitted edge whose neighbor (record) r was loaded by emit_load.
template <typename I>
__device__ __forceinline__ void emit_finish(const DevGraph &g, const LevelArgs &a, const NbrRec &r, int32_t v,
                                            int32_t s, uint32_t child_p, int64_t pos, uint32_t q) {
    int32_t dst = Update(&g.v, r.col, v);
    if (dst < 0 || dst >= g.v.n_vertices) {
        atomicOr(a.err, ERR_UPDATE_RANGE);
        dst = 0;
    }
    if (pos < a.cap) {
        a.o_src[pos] = v;
        a.o_dst[pos] = dst;
        if (a.o_smp) a.o_smp[pos] = s;
        if (a.o_dep) a.o_dep[pos] = a.depth;
    }
    if (a.push) {
        int64_t nb;
        int32_t nd;
        row_of<I>(g, r, dst, nb, nd);
        a.out_v[q] = dst;
        a.out_s[q] = s;
        a.out_p[q] = child_p;
        ((I *)a.out_beg)[q] = (I)nb;
        a.out_deg[q] = nd;
    }
}

template <typename I>
__device__ __forceinline__ void emit_edge(const DevGraph &g, const LevelArgs &a, int64_t e, int32_t v, int32_t s,
                                          uint32_t child_p, int64_t pos, uint32_t q) {
    emit_finish<I>(g, a, emit_load<I>(g, a, e), v, s, child_p, pos, q);
}

// Level expansion, part 1 (every item): batches of up to 32 items per warp,
// output and next-queue slots reserved for the whole batch, take-all items
// (d <= N) expanded cooperatively, items needing a draw appended with their
// reserved slots to the warp list (or the CTA list when biased and d > WF).
template <typename I, int BIAS>
__device__ __forceinline__ void coop_body(const DevGraph &g, const LevelArgs &a) {
    constexpr bool BIASED = BIAS != CSAW_BIAS_UNBIASED;
    const int lane = threadIdx.x & 31;
    const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
    const uint32_t n = __ldcg(a.n_in);
    const int N = a.N;
    const bool cached = BIASED && g.cdf && g.cdf_bias == BIAS;
    const bool routed = BIASED && a.sched && a.sched->mode != SCHED_THRESHOLD;
    const bool thr_ok = BIASED && a.thread_list != nullptr;
    const int nout = 2 + (a.o_smp != nullptr) + (a.o_dep != nullptr);
    const unsigned long long per_edge = 4ull + 4ull * nout + (a.push ? 12ull + 2 * (sizeof(I) + 4) : 0ull);
    uint32_t bs = (n + nw - 1) / nw;
    bs = bs < 1 ? 1 : (bs > 32 ? 32 : bs);
    unsigned long long my_bytes = 0, my_items = 0;
    for (uint32_t base = gw * bs; base < n; base += nw * bs) {
        const uint32_t it = base + lane;
        const bool valid = lane < (int)bs && it < n;
        int32_t v = 0, s = 0;
        uint32_t p = 0;
        int64_t beg = 0, d = 0;
        if (valid) {
            v = __ldcg(a.in_v + it);
            s = __ldcg(a.in_s + it);
            p = __ldcg(a.in_p + it);
            beg = (int64_t)__ldcg((const I *)a.in_beg + it);
            d = __ldcg(a.in_deg + it);
        }
        const int k = (valid && d > 0) ? (int)(d < N ? d : N) : 0;
        const bool drawn = k > 0 && d > N;
        // execution class of items that need draws: degree rule, or learned
        int cls = 1;
        if (drawn && BIASED) cls = rule_class(d, N, n, WF, cached, thr_ok, a.thread_force);
        if (routed && a.sched_tab) {   // trained model: one table load per item
            if (drawn) cls = table_class(a.sched_tab, d, a.sched->vstats[v], N, WF, cached);
        } else if (routed) {
            float2 st = make_float2(0.f, 0.f);
            if (drawn) st = a.sched->vstats[v];
            unsigned dm = __ballot_sync(FULL, drawn);
            while (dm) {
                const int b = __ffs(dm) - 1;
                dm &= dm - 1;
                const int64_t db = __shfl_sync(FULL, d, b);
                const float2 sb = make_float2(__shfl_sync(FULL, st.x, b), __shfl_sync(FULL, st.y, b));
                uint32_t hb = (uint32_t)__shfl_sync(FULL, s, b) * 0x9E3779B1u ^ __shfl_sync(FULL, p, b) * 0x85EBCA77u ^
                              (uint32_t)a.depth * 0xC2B2AE3Du ^ a.k0;
                hb ^= hb >> 15;
                hb *= 0x2C1B3C6Du;
                hb ^= hb >> 13;
                const int c = choose_class(a.sched, a.sched->wq, db, N, sb, n, a.depth, hb, WF, cached, thr_ok, lane);
                if (lane == b) cls = c;
            }
        }
        // thread class: one item per thread (valid only with a thread list)
        const bool thr = drawn && cls == CLS_THREAD;
        const bool heavy = drawn && cls >= 2 && !thr;
        // cached items with few slots and a rare rebuild run two per warp;
        // other warp-class items above WF search the cached prefix in their own list
        const bool pair = drawn && !heavy && !thr && cached && N <= 16 && d >= CSAW_PAIR_MIN_RATIO * N && a.pair_list;
        const bool hub = drawn && !heavy && !thr && cached && d > WF && !pair;
        const int incl = warp_incl_scan(k, lane);
        const int excl = incl - k;
        const int K = __shfl_sync(FULL, incl, 31);
        // Items that need draws go to one list each, with their reserved
        // slots.  Lane 0 reserves the batch's output and queue slots and its
        // range in every list at once: the atomics are independent, so their
        // round trips overlap instead of following one another.
        const bool to_sel = drawn && !heavy && !hub && !pair && !thr;
        const unsigned sm = __ballot_sync(FULL, to_sel);
        const unsigned tm = __ballot_sync(FULL, thr);
        const unsigned pbm = __ballot_sync(FULL, pair);
        const unsigned hbm = __ballot_sync(FULL, hub);
        unsigned cm[4];
#pragma unroll
        for (int c = 0; c < 4; ++c) cm[c] = __ballot_sync(FULL, heavy && cls == 2 + c);
        unsigned long long ob = 0;
        uint32_t qb = 0, ps = 0, pt = 0, pp = 0, ph = 0, pc[4] = {0u, 0u, 0u, 0u};
        if (lane == 0) {
            if (K) {
                ob = atomicAdd(a.o_count, (unsigned long long)K);
                if (a.push) qb = atomicAdd(a.n_out, (uint32_t)K);
            }
            if (sm) ps = atomicAdd(a.n_sel, (uint32_t)__popc(sm));
            if (tm) pt = atomicAdd(a.n_thread, (uint32_t)__popc(tm));
            if (pbm) pp = atomicAdd(a.n_pair, (uint32_t)__popc(pbm));
            if (hbm) ph = atomicAdd(a.n_hub, (uint32_t)__popc(hbm));
#pragma unroll
            for (int c = 0; c < 4; ++c)
                if (cm[c]) pc[c] = atomicAdd(&a.n_cta[c], (uint32_t)__popc(cm[c]));
        }
        ob = __shfl_sync(FULL, ob, 0);
        qb = __shfl_sync(FULL, qb, 0);
        const unsigned below = (1u << lane) - 1u;
        const SelEntry en{it, qb + (uint32_t)excl, ob + excl, v, s, p, (int32_t)d, (long long)beg, cls, 0};
        {
            const uint32_t pos_s = __shfl_sync(FULL, ps, 0), pos_t = __shfl_sync(FULL, pt, 0);
            const uint32_t pos_p = __shfl_sync(FULL, pp, 0), pos_h = __shfl_sync(FULL, ph, 0);
            uint32_t pos_c[4];
#pragma unroll
            for (int c = 0; c < 4; ++c) pos_c[c] = __shfl_sync(FULL, pc[c], 0);
            if (to_sel) {
                a.sel_list[pos_s + __popc(sm & below)] = en;
            } else if (thr) {
                a.thread_list[pos_t + __popc(tm & below)] = en;
            } else if (pair) {
                a.pair_list[pos_p + __popc(pbm & below)] = en;
            } else if (hub) {
                a.hub_list[pos_h + __popc(hbm & below)] = en;
            } else if (heavy) {
#pragma unroll
                for (int c = 0; c < 4; ++c)
                    if (cls == 2 + c) a.cta_list[c][pos_c[c] + __popc(cm[c] & below)] = en;
            }
        }
        if (valid) {
            my_items++;
            my_bytes += 12 + sizeof(I) + 4 + (k > 0 && d <= N ? per_edge * k : 0ull);
        }
        // take-all items: all lanes stride over their edges together
        const int ks = (k > 0 && d <= N) ? k : 0;
        const int incl_s = warp_incl_scan(ks, lane);
        const int Ks = __shfl_sync(FULL, incl_s, 31);
        for (int e0 = 0; e0 < Ks; e0 += 32) {
            const int e = e0 + lane;
            const bool act = e < Ks;
            const int b = shfl_search_int(incl_s, act ? e : 0);
            const int32_t vb = __shfl_sync(FULL, v, b);
            const int32_t sb = __shfl_sync(FULL, s, b);
            const uint32_t pb = __shfl_sync(FULL, p, b);
            const int64_t begb = __shfl_sync(FULL, beg, b);
            const int exb = __shfl_sync(FULL, excl, b);
            const int j = e - (__shfl_sync(FULL, incl_s, b) - __shfl_sync(FULL, ks, b));
            if (act)
                emit_edge<I>(g, a, begb + j, vb, sb, pb * (uint32_t)N + (uint32_t)j, (int64_t)ob + exb + j,
                             qb + (uint32_t)(exb + j));
        }
    }
#pragma unroll
    for (int off = 16; off; off >>= 1) {
        my_bytes += __shfl_xor_sync(FULL, my_bytes, off);
        my_items += __shfl_xor_sync(FULL, my_items, off);
    }
    if (lane == 0 && my_items) {
        atomicAdd(&a.bytes[0], my_bytes);
        atomicAdd(&a.items[0], my_items);
    }
}

template <typename I, int BIAS>
__global__ void __launch_bounds__(FAST_THREADS)
k_coop_fast(DevGraph g, LevelArgs a) {
    coop_body<I, BIAS>(g, a);
}

// Level expansion, part 2: one warp per listed item (N < d <= WF when
// biased); writes into the slots reserved by part 1.  CACHED: the graph holds
// the prefix cache for BIAS, so no shared copy of the raw biases is kept
// (half the shared memory, more resident warps).
template <typename I, int BIAS, bool CACHED>
__device__ __forceinline__ void select_fast_body(const DevGraph &g, const LevelArgs &a) {
    constexpr bool BIASED = BIAS != CSAW_BIAS_UNBIASED;
    constexpr int NW = FAST_THREADS / 32;
    __shared__ float s_W[BIASED && !CACHED ? NW * WF : 1];
    __shared__ float s_P[BIASED ? NW * WF : 1];
    __shared__ uint32_t s_z[BIASED ? NW * (WF / 32) : 1];
    __shared__ int s_zs[NW * 32];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
    float *W = s_W + (BIASED && !CACHED ? wib * WF : 0);
    float *P = s_P + (BIASED ? wib * WF : 0);
    uint32_t *zb = s_z + (BIASED ? wib * (WF / 32) : 0);
    int *zs = s_zs + wib * 32;
    const uint32_t n = __ldcg(a.n_sel);
    const uint32_t n_level = __ldcg(a.n_in);
    const int N = a.N;
    constexpr bool cached = BIASED && CACHED;
    const int nout = 2 + (a.o_smp != nullptr) + (a.o_dep != nullptr);
    unsigned long long my_bytes = 0, my_items = 0;
    for (uint32_t i = gw; i < n; i += nw) {
        const SelEntry en = load_sel(a.sel_list + i);
        const int32_t v = en.v, s = en.s;
        const uint32_t p = en.p;
        const int64_t beg = en.beg, d = en.d;
        const DrawCtx dc{a.k0, a.k1, p, (uint32_t)s, (uint32_t)a.depth};
        const bool rec = a.sched && a.sched->mode == SCHED_RECORD;
        long long t0 = 0;
        if (rec) t0 = clock64();
        int sel;
        if constexpr (!BIASED) {
            sel = select_unbiased(d, N, dc, zs, lane);
        } else {
            if (en.cls == 0) {
                sel = select_reg<I, BIAS>(g, beg, (int)d, N, dc, lane);
            } else if constexpr (CACHED) {
                if (d <= WF) {
                    // a pair item whose first phase failed (en.pad = its pair
                    // index + 1): its failing slot and accepted indices wait
                    // in the consumed pair entry
                    int j0 = 0, sel0 = -1;
                    if (en.pad > 0 && a.pair_list) {
                        const uint16_t *ps = reinterpret_cast<const uint16_t *>(a.pair_list + (en.pad - 1));
                        j0 = __ldcg(ps);
                        if (j0 >= N) j0 = 0;
                        if (lane < j0) sel0 = __ldcg(ps + 1 + lane);
                    }
                    sel = select_cached<I, BIAS>(g, beg, (int)d, N, dc, P, zb, lane, j0, sel0);
                } else {   // hubs are listed for k_select_hub; kept for completeness
                    sel = select_warp<I, BIAS>(g, beg, d, N, dc, P, zb, zs, lane, WF);
                    if (sel == -2) {   // needs a rebuild that does not fit: retried by the CTA pass
                        if (lane == 0) a.retry_list[atomicAdd(a.n_retry, 1u)] = en;
                        continue;
                    }
                }
            } else {
                preload_bias<I, BIAS>(g, beg, (int)d, W, lane);
                sel = select_smem(W, (int)d, N, dc, P, zb, lane);
            }
        }
        if (lane < N)
            emit_edge<I>(g, a, beg + sel, v, s, p * (uint32_t)N + (uint32_t)lane, (int64_t)en.ob + lane,
                         en.q + (uint32_t)lane);
        if (rec) {
            __syncwarp();
            if (lane == 0) record_profile(a.sched, d, N, a.sched->vstats[v], n_level, a.depth, en.cls, clock64() - t0);
        }
        if (lane == 0) {
            my_items++;
            my_bytes += 16 + (BIASED && !(cached && d > WF) ? 4ull * d : 0ull) +   // weights, or cached prefix row
                        (unsigned long long)N * (4ull + 4ull * nout + (a.push ? 12ull + 2 * (sizeof(I) + 4) : 0ull));
        }
    }
    if (lane == 0 && my_items) {
        atomicAdd(&a.bytes[5], my_bytes);
        atomicAdd(&a.items[5], my_items);
    }
}

template <typename I, int BIAS, bool CACHED>
__global__ void __launch_bounds__(FAST_THREADS, 4)
k_select_fast(DevGraph g, LevelArgs a) {
    select_fast_body<I, BIAS, CACHED>(g, a);
}

// ------------------------------------------------ thread-per-item selection
// One thread runs one item with N < d <= 32 (biased) through the whole
// selection, serially in slot order, exactly as the semantics define it:
// the row's canonical prefix lives in 32 registers (the same Kogge-Stone
// additions and running max as the warp's tile scan, so the same bits), a
// draw's index is the number of prefix values <= t (the prefix is monotone),
// selected indices are a 32-bit mask, a slot that has drawn REJECT_ATTEMPTS
// times in a phase rebuilds the prefix with the selected neighbors zeroed,
// and zero mass or MAX_SLOT_DRAWS takes the smallest unselected index.  The
// slots' indices go to shared memory and the edges are emitted afterwards,
// four slots at a time, so an item's neighbor gathers are in flight together
// instead of one per slot.  A warp thus carries 32 items instead of one.

constexpr int THREAD_SEL_SLOTS = 32;   // N < d <= 32

// Canonical prefix of the (at most 32) biases of row [beg, beg + d), the
// neighbors in zmask counted as zero; returns T.
template <typename I, int BIAS>
__device__ __forceinline__ float thread_tile_prefix(const DevGraph &g, int64_t beg, int d, uint32_t zmask,
                                                    float (&P)[32]) {
#pragma unroll
    for (int i = 0; i < 32; ++i) P[i] = (i < d && !((zmask >> i) & 1u)) ? edge_bias<I, BIAS>(g, beg + i) : 0.f;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
#pragma unroll
        for (int i = 31; i >= off; --i) P[i] = __fadd_rn(P[i], P[i - off]);
    }
    float m = 0.f;
#pragma unroll
    for (int i = 0; i < 32; ++i) {
        const float pi = i < d ? __fadd_rn(0.f, __fadd_rn(0.f, P[i])) : 0.f;
        m = fmaxf(m, pi);
        P[i] = m;
    }
    return P[31];
}

// Selects the item's N slots; slot j's neighbor index goes to sidx[j * stride].
template <typename I, int BIAS>
__device__ __forceinline__ void select_thread_item(const DevGraph &g, const LevelArgs &a, const SelEntry &en, int N,
                                                   uint8_t *sidx, int stride) {
    const int64_t beg = en.beg;
    const int d = en.d;
    const DrawCtx dc{a.k0, a.k1, en.p, (uint32_t)en.s, (uint32_t)a.depth};
    float P[32];
    float T = thread_tile_prefix<I, BIAS>(g, beg, d, 0u, P);
    uint32_t selmask = 0;
    for (int j = 0; j < N; ++j) {
        SlotRng rng;
        int A = 0, ph = 0, idx = 0;
        for (;;) {
            if (!(T > 0.f) || A == MAX_SLOT_DRAWS) {   // no mass left, or the slot's draw guard
                idx = __ffs(~selmask) - 1;
                break;
            }
            if (ph == REJECT_ATTEMPTS) {   // new phase: the selected neighbors zeroed out of the prefix
                T = thread_tile_prefix<I, BIAS>(g, beg, d, selmask, P);
                ph = 0;
                continue;
            }
            const float t = its_target(rng.word(dc, j, A), T);
            ++A;
            ++ph;
            idx = 0;
#pragma unroll
            for (int i = 0; i < 32; ++i) idx += P[i] <= t ? 1 : 0;
            if (!((selmask >> idx) & 1u)) break;
        }
        selmask |= 1u << idx;
        sidx[j * stride] = (uint8_t)idx;
    }
}

#ifndef CSAW_THREAD_SEL_MIN_BLOCKS
#define CSAW_THREAD_SEL_MIN_BLOCKS 3
#endif

template <typename I, int BIAS>
__device__ __forceinline__ void select_thread_body(const DevGraph &g, const LevelArgs &a) {
    __shared__ uint8_t s_idx[THREAD_SEL_SLOTS * FAST_THREADS];   // [slot][thread]
    const int lane = threadIdx.x & 31;
    const uint32_t n = __ldcg(a.n_thread);
    const uint32_t n_level = __ldcg(a.n_in);
    const int N = a.N;
    const int nout = 2 + (a.o_smp != nullptr) + (a.o_dep != nullptr);
    const bool rec = a.sched && a.sched->mode == SCHED_RECORD;
    uint8_t *sidx = s_idx + threadIdx.x;
    unsigned long long my_bytes = 0, my_items = 0;
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        long long t0 = 0;
        if (rec) t0 = clock64();
        select_thread_item<I, BIAS>(g, a, load_sel(a.thread_list + i), N, sidx, FAST_THREADS);
        // the entry again (an L1/L2 hit): its emission fields stay out of the
        // selection loop's registers
        const SelEntry en = load_sel(a.thread_list + i);
        for (int j0 = 0; j0 < N; j0 += 4) {
            NbrRec r[4];
#pragma unroll
            for (int u = 0; u < 4; ++u)
                if (j0 + u < N) r[u] = emit_load<I>(g, a, en.beg + sidx[(j0 + u) * FAST_THREADS]);
#pragma unroll
            for (int u = 0; u < 4; ++u)
                if (j0 + u < N)
                    emit_finish<I>(g, a, r[u], en.v, en.s, en.p * (uint32_t)N + (uint32_t)(j0 + u),
                                   (int64_t)en.ob + j0 + u, en.q + (uint32_t)(j0 + u));
        }
        if (rec) record_profile(a.sched, en.d, N, a.sched->vstats[en.v], n_level, a.depth, en.cls, clock64() - t0);
        my_items++;
        my_bytes += 16 + 4ull * en.d +
                    (unsigned long long)N * (4ull + 4ull * nout + (a.push ? 12ull + 2 * (sizeof(I) + 4) : 0ull));
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) {
        my_bytes += __shfl_xor_sync(FULL, my_bytes, o);
        my_items += __shfl_xor_sync(FULL, my_items, o);
    }
    if (lane == 0 && my_items) {
        atomicAdd(&a.bytes[10], my_bytes);
        atomicAdd(&a.items[10], my_items);
    }
}

template <typename I, int BIAS>
__global__ void __launch_bounds__(FAST_THREADS, CSAW_THREAD_SEL_MIN_BLOCKS)
k_select_thread(DevGraph g, LevelArgs a) {
    select_thread_body<I, BIAS>(g, a);
}

// Half-warp primitives: a warp runs two independent items, lanes 0-15 and
// 16-31, each with its own mask (the halves may diverge).
struct Half {
    unsigned mask;
    int base, sl;   // first lane of the half, lane within the half
    __device__ explicit Half(int lane) : mask(0xFFFFu << (lane & 16)), base(lane & 16), sl(lane & 15) {}
    __device__ int shfl(int v, int src) const { return __shfl_sync(mask, v, base + src); }
    __device__ unsigned ballot(bool p) const { return (__ballot_sync(mask, p) >> base) & 0xFFFFu; }
    __device__ unsigned match(int v) const { return (__match_any_sync(mask, v) >> base) & 0xFFFFu; }
};

// Draws of one item (N <= 16 slots) in a half-warp, slot j on lane j, the
// same draws and acceptance order as resolve_slots; cand_of(x) is a per-lane
// search.  Returns -1 when every slot is accepted, else the slot j whose
// draws of the first phase ran out (slots below j then hold their accepted
// indices in sel; the item needs a rebuild of its prefix, which a whole warp
// or CTA goes on with).  T <= 0: the slots take indices 0..N-1.
template <typename CandFn>
__device__ __forceinline__ int half_select(const Half &h, int N, const DrawCtx &dc, float T, CandFn cand_of,
                                           int &sel) {
    const int sl = h.sl;
    sel = sl;
    if (!(T > 0.f)) return -1;
    SlotRng rng;
    int cand = -1, A = 0;
    if (sl < N) {
        cand = cand_of(rng.word(dc, sl, 0));
        A = 1;
    }
    int j = 0, a = 1;
    while (j < N) {
        const int v = sl < j ? sel : (sl < N ? cand : -2 - sl);
        const unsigned same = h.match(v);
        const bool dup = sl >= j && sl < N && (same & ((1u << sl) - 1u)) != 0u;
        const unsigned db = h.ballot(dup);
        const int f = db ? __ffs(db) - 1 : N;
        if (sl >= j && sl < f) sel = v;
        if (f == N) break;
        if (f > j) a = 1;
        j = f;
        if (h.shfl(A, j) == MAX_SLOT_DRAWS) {   // termination guard: smallest unselected index
            int i = 0;
            while (h.ballot(sl < j && sel == i)) ++i;
            if (sl == j) sel = i;
            ++j;
            a = 1;
            continue;
        }
        if (a == REJECT_ATTEMPTS) return j;
        if (sl == j) {
            cand = cand_of(rng.word(dc, sl, A));
            ++A;
        }
        ++a;
    }
    return -1;
}

// What the pair kernel stages in shared memory for an item over a cached
// prefix: its whole prefix row (d <= WF), else the row's entries of the
// first prefix index level (cdf1, one per 32 edges) when they fit in WF
// floats, else those of the second level (cdf2, one per 1024 edges), else
// nothing (rows above ~512 K edges search the global index).
enum : int { STAGE_NONE = 0, STAGE_ROW = 1, STAGE_CDF1 = 2, STAGE_CDF2 = 3 };
struct StagePlan {
    int mode;
    const float *src;
    int count;
};

__device__ __forceinline__ StagePlan stage_plan(const DevGraph &g, int64_t beg, int d) {
    const int64_t end = beg + d;
    if (d <= WF) return StagePlan{STAGE_ROW, g.cdf + beg, d};
    const int64_t ka = beg >> 5, kb = (end - 1) >> 5;
    if (kb - ka + 1 <= WF) return StagePlan{STAGE_CDF1, g.cdf1 + ka, (int)(kb - ka + 1)};
    const int64_t ua = beg >> 10, ub = (end - 1) >> 10;
    if (ub - ua + 1 <= WF) return StagePlan{STAGE_CDF2, g.cdf2 + ua, (int)(ub - ua + 1)};
    return StagePlan{STAGE_NONE, nullptr, 0};
}

// cdf_search for an item whose index level is staged (STAGE_CDF1 /
// STAGE_CDF2), once the staged entries' search has given r: the remaining
// levels in global memory, one 32-entry line each, by fixed-step lifting.
// The same index as cdf_search (the first i with P[i] > t is unique); as
// there, no level reads its last candidate.
__device__ __forceinline__ int64_t staged_refine(const DevGraph &g, int mode, int r, int64_t beg, int64_t d, float t) {
    const int64_t end = beg + d;
    int64_t k;
    if (mode == STAGE_CDF1) {
        k = (beg >> 5) + r;
    } else {
        const int64_t u = (beg >> 10) + r;
        const int64_t ka = (u << 5) > (beg >> 5) ? (u << 5) : (beg >> 5);
        const int64_t kb = (u << 5) + 31 < ((end - 1) >> 5) ? (u << 5) + 31 : ((end - 1) >> 5);
        k = ka + search_upper_lift<5>(g.cdf1 + ka, (int)(kb - ka + 1), t);
    }
    const int64_t ia = (k << 5) > beg ? (k << 5) : beg;
    const int64_t ib = (k << 5) + 31 < end - 1 ? (k << 5) + 31 : end - 1;
    return ia + search_upper_lift<5>(g.cdf + ia, (int)(ib - ia + 1), t) - beg;
}

// Shared-memory copy of a work entry (three 16-byte loads).
__device__ __forceinline__ SelEntry load_sel_smem(const SelEntry *e) {
    const int4 *q = reinterpret_cast<const int4 *>(e);
    const int4 x = q[0], y = q[1], z = q[2];
    SelEntry r;
    r.it = (uint32_t)x.x;
    r.q = (uint32_t)x.y;
    r.ob = ((unsigned long long)(uint32_t)x.w << 32) | (uint32_t)x.z;
    r.v = y.x;
    r.s = y.y;
    r.p = (uint32_t)y.z;
    r.d = y.w;
    r.beg = (long long)(((unsigned long long)(uint32_t)z.y << 32) | (uint32_t)z.x);
    r.cls = z.z;
    r.pad = z.w;
    return r;
}

// Counted bytes of the prefix reads of one item (4 bytes per element staged
// or probed): the staged entries, plus per draw the probes of the levels
// searched in global memory (a 32-entry line: 5 probes each).
__device__ __forceinline__ unsigned long long staged_bytes(const StagePlan &sp, int64_t d, int N) {
    switch (sp.mode) {
        case STAGE_ROW: return 4ull * d;
        case STAGE_CDF1: return 4ull * sp.count + (unsigned long long)N * 4ull * 5;
        case STAGE_CDF2: return 4ull * sp.count + (unsigned long long)N * 4ull * 10;
        default: return (unsigned long long)N * 4ull * (64 - __clzll((unsigned long long)d));
    }
}

// Level expansion, part 2 for items over a cached prefix with N <= 16 and
// d >= 3N (a rebuild is rare): two items per warp, one per half-warp, lanes
// N..15 of a half idle instead of N..31 of a warp.  For each item the bulk
// copy engine stages, on one barrier: its work entry, the 16 bytes holding
// its prefix total T, and what its draws search (stage_plan: the prefix row
// up to WF edges, else the row's entries of the first or second prefix index
// level).  The next item's copies are requested as soon as the current
// item's draws are resolved, so they overlap the current item's edge
// emission (dependent neighbor-record gathers and stores).  Every draw
// searches the staged array in shared memory by fixed-step lifting; index
// entries then lead to one 32-entry line per remaining level in global
// memory, so rows and hubs share one resolver loop.  Items that need a
// rebuild go on from their failed first phase (its state kept in the
// consumed pair entry): rows up to WF edges by k_select_fast on the refill
// list (written over the consumed warp list), larger ones by the CTA pass.
constexpr int PAIR_ENT = 16;   // floats of a half's entry slot: the 48-byte entry and the 16-byte T window

template <typename I, int BIAS>
__device__ __forceinline__ void pair_body(const DevGraph &g, const LevelArgs &a, float *buf, float *ebuf,
                                          uint64_t *bar, uint32_t &parity) {
    const int lane = threadIdx.x & 31;
    const Half h(lane);
    const uint32_t gh = (blockIdx.x * blockDim.x + threadIdx.x) >> 4;
    const uint32_t nh = (gridDim.x * blockDim.x) >> 4;
    const uint32_t n = __ldcg(a.n_pair);
    const uint32_t n_level = __ldcg(a.n_in);
    const int N = a.N;
    const int nout = 2 + (a.o_smp != nullptr) + (a.o_dep != nullptr);
    unsigned long long my_bytes = 0;
    uint32_t my_items = 0;   // at most n per lane
    // requests the staged copies of item idx (row range rbeg, rd); returns the
    // offset of its staged array in the buffer
    auto request = [&](uint32_t idx, long long rbeg, int rd) -> int {
        const StagePlan sp = stage_plan(g, rbeg, rd);
        RowWindow w{nullptr, 0, 0u};
        if (sp.mode != STAGE_NONE) w = row_window(sp.src, sp.count);
        if (h.sl == 0) {
            const int64_t e = rbeg + rd - 1;   // T's element; the cache is padded past its last row
            fence_async_smem();                // this half's reads of buf precede the copies' writes
            bulk_load3(ebuf, a.pair_list + idx, (uint32_t)sizeof(SelEntry), ebuf + 12, g.cdf + (e & ~(int64_t)3), 16u,
                       buf, w.start, w.bytes, bar);
        }
        return w.off;
    };
    // The item loop is uniform across the warp (half h takes item base + h;
    // on the warp's last item the second half may idle), so the two halves
    // meet at a full-warp barrier after their draws and run the copy
    // request, the emission and the bookkeeping as one instruction stream.
    const uint32_t hw = lane >> 4;
    const uint32_t wstep = nh;   // two halves per warp
    uint32_t i = gh;
    bool dead = false;           // a copy wait expired: this half stops
    int off = 0;
    if (i < n) off = request(i, __ldcg(&a.pair_list[i].beg), __ldcg(&a.pair_list[i].d));
    for (uint32_t base = gh - hw; base < n; base += wstep, i += wstep) {
        const bool act = i < n && !dead;
        const uint32_t inext = i + wstep;
        long long nbeg = 0;
        int nd = 0;
        if (act && inext < n) {   // the next item's range: its load overlaps this item
            nbeg = __ldcg(&a.pair_list[inext].beg);
            nd = __ldcg(&a.pair_list[inext].d);
        }
        int jfail = -1;   // -1: all slots accepted; else the slot whose first phase failed
        SelEntry en{};
        StagePlan sp{STAGE_NONE, nullptr, 0};
        int sel = 0;
        long long t0 = 0;
        const bool rec = a.sched && a.sched->mode == SCHED_RECORD;
        if (act) {
            if (!mbar_wait(bar, parity)) {   // bounded: report instead of spinning on
                if (h.sl == 0) atomicOr(a.err, ERR_COPY_WAIT);
                mbar_wait(bar, parity);        // let the copies in flight land first
                dead = true;
            } else {
                parity ^= 1u;
            }
        }
        const bool run = act && !dead;
        if (run) {
            en = load_sel_smem(reinterpret_cast<const SelEntry *>(ebuf));
            const int64_t beg = en.beg, d = en.d;
            const float T = ebuf[12 + ((beg + d - 1) & 3)];
            const DrawCtx dc{a.k0, a.k1, en.p, (uint32_t)en.s, (uint32_t)a.depth};
            if (rec) t0 = clock64();
            sp = stage_plan(g, beg, (int)d);
            const float *S = buf + off;   // the staged row or index entries
            jfail = half_select(h, N, dc, T, [&](uint32_t x) -> int {
                const float t = its_target(x, T);
                if (sp.mode == STAGE_NONE) return (int)cdf_search(g, beg, d, t);
                const int r = search_upper_lift<9>(S, sp.count, t);
                return sp.mode == STAGE_ROW ? r : (int)staged_refine(g, sp.mode, r, beg, d, t);
            }, sel);
        }
        const bool ok = jfail < 0;
        __syncwarp();   // both halves: every read of the buffers is done, they are free
        if (run && inext < n) off = request(inext, nbeg, nd);
        const bool keep = en.d <= RESUME_MAX_DEG && i < 0x7FFFFFFFu;
        if (run && !ok && keep) {
            // a whole warp (rows) or CTA (hubs) goes on from the failed first
            // phase: the failing slot and the accepted indices (16-bit) go
            // into this item's pair entry, which nothing reads after its copy
            // has landed
            uint16_t *ps = reinterpret_cast<uint16_t *>(a.pair_list + i);
            if (h.sl < jfail) ps[1 + h.sl] = (uint16_t)sel;
            if (h.sl == 0) ps[0] = (uint16_t)jfail;
        }
        if (run && !ok && h.sl == 0) {   // rebuild needed: a whole warp or CTA goes on with the item
            if (keep) en.pad = (int32_t)(i + 1);   // where its first phase's state waits
            if (en.d <= WF) a.refill_list[atomicAdd(a.n_refill, 1u)] = en;
            else a.retry_list[atomicAdd(a.n_retry, 1u)] = en;
        }
        if (run && ok && h.sl < N)
            emit_edge<I>(g, a, en.beg + sel, en.v, en.s, en.p * (uint32_t)N + (uint32_t)h.sl, (int64_t)en.ob + h.sl,
                         en.q + (uint32_t)h.sl);
        if (run && ok && rec) {
            __syncwarp(h.mask);
            if (h.sl == 0)
                record_profile(a.sched, en.d, N, a.sched->vstats[en.v], n_level, a.depth, en.cls, clock64() - t0);
        }
        if (run && ok && h.sl == 0) {
            my_items++;
            const unsigned long long row = staged_bytes(sp, en.d, N);
            my_bytes += 16 + row + (unsigned long long)N * (4ull + 4ull * nout +
                                                            (a.push ? 12ull + 2 * (sizeof(I) + 4) : 0ull));
        }
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) {
        my_bytes += __shfl_xor_sync(FULL, my_bytes, o);
        my_items += __shfl_xor_sync(FULL, my_items, o);
    }
    if (lane == 0 && my_items) {
        atomicAdd(&a.bytes[7], my_bytes);
        atomicAdd(&a.items[7], (unsigned long long)my_items);
    }
}

// Shared staging buffers of the pair pass: one row window and one entry slot
// per half-warp, each half with its bulk-copy barrier.
constexpr int PAIR_HALVES = FAST_THREADS / 16;
constexpr int PAIR_ROW = WF + 4;   // floats: a row of up to WF plus its 16-byte alignment window

template <typename I, int BIAS>
__global__ void __launch_bounds__(FAST_THREADS, CSAW_PAIR_MIN_BLOCKS)
k_select_pair(DevGraph g, LevelArgs a) {
    __shared__ __align__(16) float s_P[PAIR_HALVES * PAIR_ROW];
    __shared__ __align__(16) float s_E[PAIR_HALVES * PAIR_ENT];
    __shared__ __align__(8) uint64_t s_bar[PAIR_HALVES];
    const int hid = threadIdx.x >> 4;
    if ((threadIdx.x & 15) == 0) mbar_init(s_bar + hid);
    mbar_init_fence();
    __syncthreads();
    uint32_t parity = 0;
    pair_body<I, BIAS>(g, a, s_P + hid * PAIR_ROW, s_E + hid * PAIR_ENT, s_bar + hid, parity);
}

// Level expansion, part 2 for hub items (d > WF) over a cached prefix: one
// warp per item, each draw a search of the prefix through its index
// (cdf_search) taken one attempt at a time, since a search costs dependent
// loads; no shared memory.  An item whose draws need a rebuild of its prefix
// goes to the retry list (the CTA pass rebuilds it in global scratch).
template <typename I, int BIAS>
__device__ __forceinline__ void hub_body(const DevGraph &g, const LevelArgs &a) {
    const int lane = threadIdx.x & 31;
    const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
    const uint32_t n = __ldcg(a.n_hub);
    const uint32_t n_level = __ldcg(a.n_in);
    const int N = a.N;
    const int nout = 2 + (a.o_smp != nullptr) + (a.o_dep != nullptr);
    unsigned long long my_bytes = 0, my_items = 0;
    for (uint32_t i = gw; i < n; i += nw) {
        const SelEntry en = load_sel(a.hub_list + i);
        const DrawCtx dc{a.k0, a.k1, en.p, (uint32_t)en.s, (uint32_t)a.depth};
        const bool rec = a.sched && a.sched->mode == SCHED_RECORD;
        long long t0 = 0;
        if (rec) t0 = clock64();
        const int sel = select_warp<I, BIAS>(g, en.beg, en.d, N, dc, nullptr, nullptr, nullptr, lane, 0);
        if (sel == -2) {
            if (lane == 0) a.retry_list[atomicAdd(a.n_retry, 1u)] = en;
            continue;
        }
        if (lane < N)
            emit_edge<I>(g, a, en.beg + sel, en.v, en.s, en.p * (uint32_t)N + (uint32_t)lane, (int64_t)en.ob + lane,
                         en.q + (uint32_t)lane);
        if (rec) {
            __syncwarp();
            if (lane == 0)
                record_profile(a.sched, en.d, N, a.sched->vstats[en.v], n_level, a.depth, en.cls, clock64() - t0);
        }
        if (lane == 0) {
            my_items++;
            // per draw: one 4-byte prefix probe per halving of the row (the
            // index levels split the same search), then the edge's records
            my_bytes += 16 + (unsigned long long)N * (4ull * (64 - __clzll((unsigned long long)en.d)) + 4ull +
                                                      4ull * nout + (a.push ? 12ull + 2 * (sizeof(I) + 4) : 0ull));
        }
    }
    if (lane == 0 && my_items) {
        atomicAdd(&a.bytes[6], my_bytes);
        atomicAdd(&a.items[6], my_items);
    }
}

template <typename I, int BIAS>
__global__ void __launch_bounds__(FAST_THREADS, 4)
k_select_hub(DevGraph g, LevelArgs a) {
    hub_body<I, BIAS>(g, a);
}

// Biased walks: one warp per walk.  A step with d <= 32 is one round trip:
// the biases, column ids and neighbor records of all neighbors load together,
// the prefix and search run in registers, and the chosen lane's record gives
// the next vertex's adjacency range.  Lane l computes the Philox block of step
// t0 + l, so one warp-wide Philox serves 32 steps, and lane l holds the edge
// of step t0 + l until 32 records are written out together.
template <typename I, int BIAS>
__global__ void __launch_bounds__(FAST_THREADS, 4)
k_walk_fast(DevGraph g, WalkArgs a) {
    constexpr int NW = FAST_THREADS / 32;
    __shared__ float s_W[NW * WF];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    float *W = s_W + wib * WF;
    const bool cached = BIAS != CSAW_BIAS_UNBIASED && g.cdf && g.cdf_bias == BIAS;
    const bool mat = BIAS == CSAW_BIAS_EDGE_WEIGHT || BIAS == CSAW_BIAS_DEGREE;
    const unsigned long long obytes = 4ull * (2 + (a.o_smp != nullptr) + (a.o_dep != nullptr));
    const unsigned long long rec = 4ull + sizeof(I) + 4ull;   // col + neighbor record
    unsigned long long steps = 0, bytes = 0;
    for (int w = gw; w < a.n; w += nw) {
        int32_t v = a.seeds[w];
        if (v < 0 || v >= g.v.n_vertices) {
            if (lane == 0) atomicOr(a.err, ERR_SEED_RANGE);
            continue;
        }
        int64_t beg = row_begin<I>(g, v);
        int32_t d = (int32_t)(row_begin<I>(g, v + 1) - beg);
        bytes += 2 * sizeof(I);
        uint32_t xw = 0;
        int32_t rs = 0, rd = 0;
        int t0 = 0, nrec = 0;
        auto flush = [&]() {
            if (nrec == 0) return;
            unsigned long long base = 0;
            if (lane == 0) base = atomicAdd(a.o_count, (unsigned long long)nrec);
            base = __shfl_sync(FULL, base, 0);
            const int64_t pos = (int64_t)base + lane;
            if (lane < nrec && pos < a.cap) {
                a.o_src[pos] = rs;
                a.o_dst[pos] = rd;
                if (a.o_smp) a.o_smp[pos] = a.base + w;
                if (a.o_dep) a.o_dep[pos] = t0 + lane;
            }
            nrec = 0;
        };
        for (int t = 0; t < a.len; ++t) {
            if ((t & 31) == 0) {
                flush();
                t0 = t;
                xw = philox(make_uint4(0u, (uint32_t)(a.base + w), (TAG_SAMPLE << 24) | (uint32_t)(t + lane), 0u), a.k0,
                            a.k1).x;
            }
            if (d <= 0) break;
            const uint32_t x = __shfl_sync(FULL, xw, t & 31);
            int64_t e = beg;
            int32_t u = 0, nd = 0;
            int64_t nb = 0;
            bool have = false;
            bytes += obytes + rec;
            if (d == 1) {
            } else if (BIAS == CSAW_BIAS_UNBIASED) {
                e = beg + mulhi(x, (uint32_t)d);
            } else if (d <= 32) {
                float wl = 0.f;
                int32_t ul = 0, dl = 0;
                int64_t bl = 0;
                if (lane < d) {
                    if (g.nrec) {   // one 128-bit record per lane, coalesced
                        const NbrRec r = load_rec(g.nrec, beg + lane);
                        ul = r.col;
                        dl = r.deg;
                        bl = r.beg;
                        wl = BIAS == CSAW_BIAS_DEGREE ? __int2float_rn(dl) : edge_bias<I, BIAS>(g, beg + lane);
                    } else {
                        wl = edge_bias<I, BIAS>(g, beg + lane);
                        ul = __ldg(g.v.col + beg + lane);
                    }
                }
                // canonical prefix of one tile; the first lane above t is the
                // same with or without the running max, and T is the max
                const float v = warp_ks_sum(wl, lane);
                const float P = lane < d ? __fadd_rn(0.f, __fadd_rn(0.f, v)) : 0.f;
                const float T = __uint_as_float(__reduce_max_sync(FULL, __float_as_uint(P)));
                int idx = 0;
                if (T > 0.f) idx = __ffs(__ballot_sync(FULL, P > its_target(x, T))) - 1;
                e = beg + idx;
                u = __shfl_sync(FULL, ul, idx);
                nb = __shfl_sync(FULL, bl, idx);
                nd = __shfl_sync(FULL, dl, idx);
                have = g.nrec != nullptr;
                bytes += (mat ? 4ull : 4ull + 2ull * sizeof(I)) * d + rec * (d - 1);
            } else if (cached) {
                const float *cp = g.cdf + beg;
                const float T = __ldg(cp + d - 1);
                const float tt = its_target(x, T);
                e = beg + (!(T > 0.f) ? 0 : (d > 1024 ? warp_cdf_search(g, beg, d, tt, lane)
                                                       : warp_search_upper(cp, d, tt, lane)));
                bytes += 4ull * 32 * ((68 - __clzll((unsigned long long)d)) / 5);   // 32 probes per round
            } else if (d <= WF) {
                preload_bias<I, BIAS>(g, beg, d, W, lane);
                auto wfn = [&](int64_t i) { return W[i]; };
                const float T = warp_canon_prefix(wfn, d, W, nullptr, lane);
                e = beg + (T > 0.f ? search_upper(W, d, its_target(x, T)) : 0);
                __syncwarp();
                bytes += (mat ? 4ull : 4ull + 2ull * sizeof(I)) * d;
            } else {
                if (d > a.scratch_stride) {
                    if (lane == 0) atomicOr(a.err, ERR_SCRATCH);
                    break;
                }
                float *buf = a.scratch + (int64_t)gw * a.scratch_stride;
                auto wfn = [&](int64_t i) { return edge_bias<I, BIAS>(g, beg + i); };
                const float T = warp_canon_prefix(wfn, d, buf, nullptr, lane);
                e = beg + (T > 0.f ? search_upper(buf, d, its_target(x, T)) : 0);
                bytes += (mat ? 4ull : 4ull + 2ull * sizeof(I)) * d;
            }
            if (!have) {
                if (g.nrec) {
                    const NbrRec r = load_rec(g.nrec, e);
                    u = r.col;
                    nb = r.beg;
                    nd = r.deg;
                } else {
                    u = __ldg(g.v.col + e);
                }
            }
            int32_t dst = Update(&g.v, u, v);
            if (dst < 0 || dst >= g.v.n_vertices) {
                if (lane == 0) atomicOr(a.err, ERR_UPDATE_RANGE);
                dst = 0;
            }
            if (!g.nrec || dst != u) {
                nb = row_begin<I>(g, dst);
                nd = (int32_t)(row_begin<I>(g, dst + 1) - nb);
            }
            if (lane == (t & 31)) {
                rs = v;
                rd = dst;
            }
            ++nrec;
            v = dst;
            beg = nb;
            d = nd;
            ++steps;
        }
        flush();
    }
    if (lane == 0 && steps) {
        atomicAdd(&a.bytes[2], bytes);
        atomicAdd(&a.items[2], steps);
    }
}

// Walks with one thread per walk, for many walks: unbiased steps take one
// round trip via the neighbor records; biased steps search the cached prefix
// (the graph must hold it for BIAS) by binary search through its index, so a
// warp keeps 32 walks in flight instead of one.  Same draws as the warp
// kernels: step t of walk w uses word x of Philox(0, w, t).
template <typename I, int BIAS>
__global__ void __launch_bounds__(WALK_THREADS)
k_walk_thread_fast(DevGraph g, WalkArgs a) {
    constexpr bool BIASED = BIAS != CSAW_BIAS_UNBIASED;
    __shared__ int32_t s_out[(WALK_THREADS / 32) * 4 * STAGE];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    WarpStage stg;
    stg.s_src = s_out + wib * 4 * STAGE;
    stg.s_dst = stg.s_src + STAGE;
    stg.s_smp = stg.s_dst + STAGE;
    stg.s_dep = stg.s_smp + STAGE;
    const OutArgs oa{a.o_src, a.o_dst, a.o_smp, a.o_dep, a.o_count, a.cap};
    const int stride = gridDim.x * blockDim.x;
    unsigned long long steps = 0, probes = 0;
    for (int base = blockIdx.x * blockDim.x; base < a.n; base += stride) {
        const int w = base + threadIdx.x;
        bool alive = w < a.n;
        int32_t v = 0;
        int64_t beg = 0;
        int32_t d = 0;
        if (alive) {
            v = a.seeds[w];
            if (v < 0 || v >= g.v.n_vertices) {
                atomicOr(a.err, ERR_SEED_RANGE);
                alive = false;
            } else {
                beg = row_begin<I>(g, v);
                d = (int32_t)(row_begin<I>(g, v + 1) - beg);
            }
        }
        for (int t = 0; t < a.len; ++t) {
            if (alive && d <= 0) alive = false;
            if (!__any_sync(FULL, alive)) break;
            int32_t dst = 0;
            if (alive) {
                uint32_t idx = 0;
                if (d > 1) {
                    uint4 b = philox(make_uint4(0u, (uint32_t)(a.base + w), (TAG_SAMPLE << 24) | (uint32_t)t, 0u), a.k0, a.k1);
                    if constexpr (BIASED) {
                        const float T = __ldg(g.cdf + beg + d - 1);
                        if (T > 0.f) idx = (uint32_t)cdf_search(g, beg, d, its_target(b.x, T));
                        probes += 1 + (64 - __clzll((unsigned long long)d));
                    } else {
                        idx = mulhi(b.x, (uint32_t)d);
                    }
                }
                const NbrRec r = edge_rec<I>(g, beg + idx);
                dst = Update(&g.v, r.col, v);
                if (dst < 0 || dst >= g.v.n_vertices) {
                    atomicOr(a.err, ERR_UPDATE_RANGE);
                    dst = 0;
                }
                int64_t nb;
                int32_t nd;
                row_of<I>(g, r, dst, nb, nd);
                beg = nb;
                d = nd;
                ++steps;
            }
            stg.push(oa, alive, v, dst, a.base + w, t, lane);
            if (alive) v = dst;
        }
    }
    stg.flush(oa, lane);
    unsigned long long tot = steps, pr = probes;
    for (int off = 16; off; off >>= 1) {
        tot += __shfl_xor_sync(FULL, tot, off);
        pr += __shfl_xor_sync(FULL, pr, off);
    }
    if (lane == 0) {
        unsigned long long per = 4 + sizeof(I) + 4 + 4ull * (2 + (a.o_smp != nullptr) + (a.o_dep != nullptr));
        atomicAdd(&a.bytes[8], tot * per + 4 * pr);   // + prefix probes (biased)
        atomicAdd(&a.items[8], tot);
    }
}

template <typename I>
__global__ void k_nbr_records(DevGraph g, NbrRec *rec) {
    const I *r = (const I *)g.v.rowptr;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < g.v.n_edges;
         e += (int64_t)gridDim.x * blockDim.x) {
        const int32_t u = __ldg(g.v.col + e);
        const I b = __ldg(r + u);
        const unsigned long long ub = (unsigned long long)(long long)b;
        reinterpret_cast<int4 *>(rec)[e] =
            make_int4(u, (int32_t)(__ldg(r + u + 1) - b), (int32_t)(uint32_t)ub, (int32_t)(uint32_t)(ub >> 32));
    }
}

}  // namespace csaw
