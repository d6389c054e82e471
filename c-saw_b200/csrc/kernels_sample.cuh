// kernels_sample.cuh -- sampling and walk kernels (sm_100a).
//
// C-SAW counterparts (non-stream/): check (main.cu:21-93) is the level
// expansion below; get_neighbors (functions.cuh:872-892), ITS/gpu_prefix
// (:112-176), binary_search (:11-43), bitmap_search (:45-70) and
// heur_normalize (:743-868) are the canonical prefix, inverse-transform search
// and slot resolver of csaw_device.cuh; frontier (:971-1011) is the staged
// output and queue push; check_layer + ITS_MDRW (main.cu:95-194,
// functions.cuh:1014-1060) is k_mdrw.
#pragma once

#include "csaw_device.cuh"
#include "sched_mlp.cuh"

namespace csaw {

// A listed frontier item, read around L1 (the list may have been written by
// other blocks earlier in the same launch).
__device__ __forceinline__ SelEntry load_sel(const SelEntry *e) {
    static_assert(sizeof(SelEntry) == 48, "three 16-byte loads");
    const int4 *q = reinterpret_cast<const int4 *>(e);
    const int4 x = __ldcg(q), y = __ldcg(q + 1), z = __ldcg(q + 2);
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

// Algorithmic bytes of one expansion (what the algorithm must touch; sector
// waste not counted): queue item 12 B, rowptr pair, bias reads when the
// prefix is scanned, the selected col entries, the output edges and the pushed
// children.
template <typename I, int BIAS>
__device__ __forceinline__ unsigned long long expansion_bytes(const DevGraph &g, int64_t d, int k,
                                                              bool scanned, const LevelArgs &a, bool push) {
    unsigned long long b = 12 + 2 * sizeof(I);
    if (scanned) {
        if (BIAS == CSAW_BIAS_EDGE_WEIGHT || (BIAS == CSAW_BIAS_DEGREE && g.ebias))
            b += 4ull * d + 4ull * k;
        else
            b += (4ull + 2ull * sizeof(I)) * d;  // col + neighbor rowptr pairs
    } else {
        b += 4ull * k;
    }
    b += 4ull * k * (2 + (a.o_smp != nullptr) + (a.o_dep != nullptr));
    if (push) b += 12ull * k;
    return b;
}

// -------------------------------------------------------------- queue init
static __global__ void k_init_queue(const int32_t *seeds, uint32_t n, int F, int s0, int64_t V,
                             int32_t *qv, int32_t *qs, uint32_t *qp, uint32_t *qn, int *err) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) *qn = n;
    if (i >= n) return;
    int32_t v = seeds[i];
    if (v < 0 || v >= V) {
        atomicOr(err, ERR_SEED_RANGE);
        v = 0;
    }
    qv[i] = v;
    qs[i] = s0 + (int32_t)(i / (uint32_t)F);
    qp[i] = i % (uint32_t)F;
}

// ------------------------------------------------------- warp selection
// Selection for one item with d > N by one warp; returns the lane's slot
// selection (lanes < N).  P/zb/zs: the warp's shared buffers, P holding `cap`
// floats.  With a CDF cache the first phase searches the cached prefix, so d
// may exceed cap; if such an item needs a phase rebuild (which must write a
// prefix of d floats) every lane returns -2 and the caller hands the whole
// item to the CTA path, which recomputes it with the same keys.
template <typename I, int BIAS>
__device__ __forceinline__ int select_warp(const DevGraph &g, int64_t beg, int64_t d, int N,
                                           const DrawCtx &dc, float *P, uint32_t *zb, int *zs,
                                           int lane, int64_t cap) {
    constexpr bool BIASED = BIAS != CSAW_BIAS_UNBIASED;
    auto wfn = [&](int64_t i) { return edge_bias<I, BIAS>(g, beg + i); };
    float T = 0.f;
    int nZ = 0;
    bool indexed = false;   // searching the cached prefix through its index
    if constexpr (BIASED) {
        if (g.cdf && g.cdf_bias == BIAS) {
            indexed = true;
            T = g.cdf[beg + d - 1];
        } else {
            T = warp_canon_prefix(wfn, d, P, nullptr, lane);
        }
    }
    SlotRng rng;
    SelState st;
    auto cand_of = [&](uint32_t x, bool act) -> int {
        if (!act) return -1;
        if constexpr (BIASED) {
            const float t = its_target(x, T);
            return indexed ? (int)cdf_search(g, beg, d, t) : (int)search_upper(P, d, t);
        } else {
            return kth_not_excluded(mulhi(x, (uint32_t)(d - nZ)), zs, nZ);
        }
    };
    bool zero = BIASED && !(T > 0.f);
    if (!zero) draw_pending(st, 0, N, lane, dc, rng, cand_of);
    for (;;) {
        if (zero) {
            zero_fill(st, N, lane);
            break;
        }
        if (resolve_slots(st, N, lane, dc, rng, cand_of) == 0) break;
        const int j = st.j;
        if constexpr (BIASED) {
            if (d > cap) return -2;
            const int nwords = (int)((d + 31) >> 5);
            for (int w = lane; w < nwords; w += 32) zb[w] = 0u;
            __syncwarp();
            if (lane < j) atomicOr(&zb[st.sel >> 5], 1u << (st.sel & 31));
            __syncwarp();
            T = warp_canon_prefix(wfn, d, P, zb, lane);
            indexed = false;
            if (!(T > 0.f)) {
                zero = true;
                continue;
            }
        } else {
            sort_selected(st, j, zs, lane);
            nZ = j;
        }
        draw_pending(st, j, N, lane, dc, rng, cand_of);
    }
    return st.sel;
}

// Streaming: the bias bases of a resident partition -- its weights, or its
// canonical prefix with the graph's resident index levels (raw weights, for
// a rebuild, read from page-locked host memory).
__device__ __forceinline__ void stream_bases(DevGraph &g, const LevelArgs &a, int part) {
    if (a.part_cdf) {
        g.cdf = a.part_w[part];
        g.cdf1 = a.cdf1_all;
        g.cdf2 = a.cdf2_all;
        g.v.weight = a.host_w;
    } else {
        g.v.weight = a.part_w[part];
    }
}

// ----------------------------------------------------- level expansion
// One warp per queue item (grid-stride, persistent grid).  Biased items whose
// degree exceeds WBUF are deferred to k_expand_heavy.  STREAM: each item
// reads the adjacency of its own partition (LevelArgs::part_col/part_w) and
// items of partitions not sampled this round are skipped.
template <typename I, int BIAS, bool STREAM = false>
__global__ void __launch_bounds__(EXPAND_THREADS)
k_expand_warp(DevGraph g0, LevelArgs a) {
    constexpr bool BIASED = BIAS != CSAW_BIAS_UNBIASED;
    constexpr int NW = EXPAND_THREADS / 32;
    __shared__ float s_P[BIASED ? NW * WBUF : 1];
    __shared__ uint32_t s_z[BIASED ? NW * (WBUF / 32) : 1];
    __shared__ int s_zs[NW * 32];
    __shared__ int32_t s_out[NW * 4 * STAGE];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
    float *P = s_P + (BIASED ? wib * WBUF : 0);
    uint32_t *zb = s_z + (BIASED ? wib * (WBUF / 32) : 0);
    int *zs = s_zs + wib * 32;
    WarpStage stg;
    stg.s_src = s_out + wib * 4 * STAGE;
    stg.s_dst = stg.s_src + STAGE;
    stg.s_smp = stg.s_dst + STAGE;
    stg.s_dep = stg.s_smp + STAGE;
    const OutArgs oa{a.o_src, a.o_dst, a.o_smp, a.o_dep, a.o_count, a.cap};
    const uint32_t n = *a.n_in;
    unsigned long long my_bytes = 0, my_items = 0;
    for (uint32_t it = gw; it < n; it += nw) {
        int32_t v = a.in_v[it];
        if (v < 0) continue;   // dropped by per-sample dedup
        DevGraph g = g0;
        if (STREAM) {
            const int part = v >> a.pbits;
            g.v.col = a.part_col[part];
            if (!g.v.col) continue;   // partition not resident this round
            stream_bases(g, a, part);
        }
        int l, N;
        bool push;
        item_level(a, it, l, N, push);
        const int32_t s = a.in_s[it];
        const uint32_t p = a.in_p[it];
        // STREAM: a walk step (N = 1) whose next vertex lies in a partition of
        // this round goes on in this warp instead of waiting for the next
        // round (same draw keys: the child of slot 0 keeps lineage p); at
        // most D steps
        for (;;) {
            const int64_t beg = row_begin<I>(g, v);
            const int64_t d = row_begin<I>(g, v + 1) - beg;
            if (d <= 0) {
                my_items++;
                my_bytes += 12 + 2 * sizeof(I);
                break;
            }
            if (BIASED && d > N && d > WBUF && !(g.cdf && g.cdf_bias == BIAS)) {
                // never a continued step (those have d <= WBUF), so `it` is this item
                if (lane == 0) {
                    uint32_t h = atomicAdd(a.n_heavy, 1u);
                    a.heavy[h] = it;
                }
                break;
            }
            my_items++;
            const int k = d < N ? (int)d : N;
            int sel = lane;
            bool scanned = false;
            if (d > N) {
                scanned = BIASED && !(g.cdf && g.cdf_bias == BIAS);
                const DrawCtx dc{a.k0, a.k1, p, (uint32_t)s, (uint32_t)l};
                sel = select_warp<I, BIAS>(g, beg, d, N, dc, P, zb, zs, lane, WBUF);
                if (sel == -2) {   // cached hub that needs a rebuild: the CTA path redoes it
                    // (only with a prefix cache, which streaming graphs do not have)
                    my_items--;
                    if (lane == 0) {
                        uint32_t h = atomicAdd(a.n_heavy, 1u);
                        a.heavy[h] = it;
                    }
                    break;
                }
            }
            bool act = lane < k;
            int32_t dst = 0;
            if (act) {
                dst = Update(&g.v, __ldg(g.v.col + beg + sel), v);
                if (dst < 0 || dst >= g.v.n_vertices) {
                    atomicOr(a.err, ERR_UPDATE_RANGE);
                    dst = 0;
                }
            }
            stg.push(oa, act, v, dst, s, l, lane);
            bool cont = false;
            int32_t nv = 0;
            if (STREAM && push && k == 1 && a.fan[l + 1] == 1) {
                nv = __shfl_sync(FULL, dst, 0);
                if (a.part_col[nv >> a.pbits]) {
                    const int64_t nd = row_begin<I>(g, nv + 1) - row_begin<I>(g, nv);
                    cont = !(BIASED && nd > 1 && nd > WBUF && !a.part_cdf);   // the warp path can take it
                }
            }
            if (push && !cont) {
                uint32_t q = 0;
                if (lane == 0) q = atomicAdd(a.n_out, (uint32_t)k);
                q = __shfl_sync(FULL, q, 0);
                if (act) {
                    a.out_v[q + lane] = dst;
                    a.out_s[q + lane] = s;
                    a.out_p[q + lane] = p * (uint32_t)N + (uint32_t)lane;
                    if (a.out_dep) a.out_dep[q + lane] = l + 1;
                }
            }
            my_bytes += expansion_bytes<I, BIAS>(g, d, k, scanned, a, push && !cont);
            if (!cont) break;
            v = nv;
            l += 1;
            N = 1;
            push = l + 1 < a.D;
            g.v.col = a.part_col[v >> a.pbits];
            stream_bases(g, a, v >> a.pbits);
        }
    }
    stg.flush(oa, lane);
    if (lane == 0) {
        atomicAdd(&a.bytes[0], my_bytes);
        atomicAdd(&a.items[0], my_items);
    }
}

// ------------------------------------------------ high-degree expansion
// Floats of prefix scratch a CTA rebuild of a degree-d row needs: the
// prefix, tile sums, group carries and the exclusion bitmap.
__host__ __device__ __forceinline__ int64_t heavy_need(int64_t d) {
    return d + (d >> 5) + (d >> 10) + (d >> 5) + 8;
}

// ------------------------------------------- incremental rebuild of a hub
// The canonical prefix of a row with the selected neighbors Z zeroed is, per
// edge i in tile t (32 edges, row-aligned) of group u (32 tiles):
//   P'[i] = C_u + (qex_t + a_t[i])      (then a running max)
// with a_t the tile's Kogge-Stone scan, qex_t the exclusive Kogge-Stone scan
// of the group's tile totals and C_u the in-order sum of the earlier groups'
// totals.  Only the tiles holding a zeroed neighbor change their scan; the
// others keep the totals and in-tile maxima of the tile-summary cache.  So a
// rebuild recomputes those tiles, rescans the tile totals of every group,
// carries across groups in order and keeps, per tile, the running max of
// M_t = C_u + (qex_t + max a_t), the tile's largest P' (rounding is monotone,
// so the largest a_t gives it).  The first i with P'[i] > x lies in the
// first tile whose running max exceeds x; that tile's P' values are
// recomputed from its 32 biases with the same additions.  Every value is
// the one the full rescan computes, and the search returns the same index,
// but a rebuild touches d/32 summaries instead of d biases and d prefix
// values.  Scratch (floats): RM, QEX, QA per tile, GC per group.
struct IncrView {
    float *RM, *QEX, *QA, *GC;
    int64_t ntiles, ngroups;
};

// Rows of up to this many groups (2 M edges) keep their group maxima in
// shared memory for the draws' first search level.
constexpr int INCR_SGROUPS = 2048;

__device__ __forceinline__ IncrView incr_view(float *P, int64_t d) {
    IncrView iv;
    iv.ntiles = (d + 31) >> 5;
    iv.ngroups = (iv.ntiles + 31) >> 5;
    iv.RM = P;
    iv.QEX = P + iv.ntiles;
    iv.QA = P + 2 * iv.ntiles;
    iv.GC = P + 3 * iv.ntiles;
    return iv;
}

// The rebuild, by the whole CTA (all threads call it; zs[0..nz) in shared
// memory are the zeroed edge offsets).  Returns the new total T.
template <typename WFn>
__device__ float incr_rebuild(const DevGraph &g, WFn wfn, int64_t beg, int32_t v, int64_t d, const int32_t *zs,
                              int nz, const IncrView &iv, float *sgm) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const float2 *ts = g.tsc + tsc_slot(beg, v);
    // per group: tile totals (recomputed where a neighbor is zeroed), their
    // exclusive scan, qex + max a per tile, the group total
    for (int64_t gg = warp; gg < iv.ngroups; gg += nw) {
        const int64_t t = (gg << 5) + lane;
        float tot = 0.f, amax = 0.f;
        if (t < iv.ntiles) {
            const float2 x = __ldg(ts + t);
            tot = x.x;
            amax = x.y;
        }
        bool touched = false;
        for (int k = 0; k < nz; ++k) touched |= (int64_t)(zs[k] >> 5) == t;
        unsigned tm = __ballot_sync(FULL, touched);
        while (tm) {
            const int b = __ffs(tm) - 1;
            tm &= tm - 1;
            const int64_t i = ((((gg << 5) + b)) << 5) + lane;
            float w = 0.f;
            if (i < d) {
                w = wfn(i);
                for (int k = 0; k < nz; ++k)
                    if ((int64_t)zs[k] == i) w = 0.f;
            }
            const float a = warp_ks_sum(w, lane);
            const float at = __shfl_sync(FULL, a, 31);
            float m = i < d ? a : 0.f;
#pragma unroll
            for (int off = 16; off; off >>= 1) m = fmaxf(m, __shfl_xor_sync(FULL, m, off));
            if (lane == b) {
                tot = at;
                amax = m;
            }
        }
        const float q = warp_ks_sum(tot, lane);
        float qex = __shfl_up_sync(FULL, q, 1);
        if (lane == 0) qex = 0.f;
        if (t < iv.ntiles) {
            iv.QEX[t] = qex;
            iv.QA[t] = __fadd_rn(qex, amax);
        }
        if (lane == 31) iv.GC[gg] = q;
    }
    __syncthreads();
    if (warp == 0) {   // carry into each group, in group order (as cta_canon_prefix)
        float C = 0.f;
        for (int64_t g0 = 0; g0 < iv.ngroups; g0 += 32) {
            const int64_t gg = g0 + lane;
            const float tot = gg < iv.ngroups ? iv.GC[gg] : 0.f;
            const int m = iv.ngroups - g0 < 32 ? (int)(iv.ngroups - g0) : 32;
            float mine = 0.f;
            for (int k = 0; k < m; ++k) {
                if (lane == k) mine = C;
                C = __fadd_rn(C, __shfl_sync(FULL, tot, k));
            }
            if (gg < iv.ngroups) iv.GC[gg] = mine;
        }
    }
    __syncthreads();
    for (int64_t t = threadIdx.x; t < iv.ntiles; t += blockDim.x) iv.RM[t] = __fadd_rn(iv.GC[t >> 5], iv.QA[t]);
    __syncthreads();
    {   // running max of the tile maxima (max is exact: ranges scanned in parallel)
        __shared__ float s_rm[32];
        const int64_t per = (iv.ntiles + nw - 1) / nw;
        const int64_t t0 = (int64_t)warp * per, t1 = t0 + per < iv.ntiles ? t0 + per : iv.ntiles;
        float rmax = 0.f;
        for (int64_t t = t0 + lane; t < t1; t += 32) rmax = fmaxf(rmax, iv.RM[t]);
#pragma unroll
        for (int off = 16; off; off >>= 1) rmax = fmaxf(rmax, __shfl_xor_sync(FULL, rmax, off));
        if (lane == 0) s_rm[warp] = rmax;
        __syncthreads();
        float carry = 0.f;
        for (int w = 0; w < warp; ++w) carry = fmaxf(carry, s_rm[w]);
        for (int64_t base = t0; base < t1; base += 32) {
            const int64_t t = base + lane;
            const float ms = fmaxf(warp_max_scan(t < t1 ? iv.RM[t] : 0.f, lane), carry);
            if (t < t1) iv.RM[t] = ms;
            carry = __shfl_sync(FULL, ms, 31);
        }
    }
    __syncthreads();
    if (iv.ngroups <= INCR_SGROUPS) {   // the running max at each group's last tile
        for (int64_t u = threadIdx.x; u < iv.ngroups; u += blockDim.x)
            sgm[u] = iv.RM[(u << 5) + 31 < iv.ntiles - 1 ? (u << 5) + 31 : iv.ntiles - 1];
        __syncthreads();
    }
    return iv.RM[iv.ntiles - 1];
}

// Draw searches after an incremental rebuild, by one warp (all lanes call):
// each lane with act set gets the first i with P'[i] > t.  Each lane finds
// its own tile, in parallel: its group among the running maxima at the
// groups' last tiles (sgm, shared memory, when the row has at most
// INCR_SGROUPS groups; else in RM), then the tile among the group's 32
// entries of RM; it stages the tile's biases (zeroed ones as 0) in its row of
// srow ([32][33] floats, shared) with the tile's carry and scan offset.  The
// warp then scans each staged tile in turn, with no memory access on that
// serial path.
template <typename WFn>
__device__ __forceinline__ int incr_search(WFn wfn, int64_t d, const int32_t *zs, int nz, const IncrView &iv,
                                           const float *sgm, float *srow, float t, bool act, int lane) {
    int64_t k = 0;
    float gc = 0.f, qx = 0.f;
    if (act) {
        int64_t u;
        if (iv.ngroups <= INCR_SGROUPS) {
            u = search_upper(sgm, iv.ngroups, t);
        } else {
            int64_t lo = 0, hi = iv.ngroups - 1;
            while (lo < hi) {
                const int64_t mid = (lo + hi) >> 1;
                const int64_t te = (mid << 5) + 31 < iv.ntiles - 1 ? (mid << 5) + 31 : iv.ntiles - 1;
                if (iv.RM[te] > t) hi = mid; else lo = mid + 1;
            }
            u = lo;
        }
        const int64_t k0 = u << 5;
        k = k0 + search_upper_lift<5>(iv.RM + k0, iv.ntiles - k0 < 32 ? (int)(iv.ntiles - k0) : 32, t);
        gc = iv.GC[u];
        qx = iv.QEX[k];
        uint32_t zm = 0;
        for (int z = 0; z < nz; ++z)
            if ((int64_t)(zs[z] >> 5) == k) zm |= 1u << (zs[z] & 31);
        float *row = srow + lane * 33;
        const int64_t i0 = k << 5;
#pragma unroll
        for (int m = 0; m < 32; ++m) row[m] = (i0 + m < d && !((zm >> m) & 1u)) ? wfn(i0 + m) : 0.f;
    }
    __syncwarp();
    int res = -1;
    unsigned am = __ballot_sync(FULL, act);
    while (am) {
        const int b = __ffs(am) - 1;
        am &= am - 1;
        const long long kb = __shfl_sync(FULL, (long long)k, b);
        const float tb = __shfl_sync(FULL, t, b), gb = __shfl_sync(FULL, gc, b), qb = __shfl_sync(FULL, qx, b);
        const float a = warp_ks_sum(srow[b * 33 + lane], lane);
        const float pv = __fadd_rn(gb, __fadd_rn(qb, a));
        const unsigned hit = __ballot_sync(FULL, ((int64_t)kb << 5) + lane < d && pv > tb);
        // hit is never empty: the tile's largest P' is its running max entry
        if (lane == b) res = (int)(((int64_t)kb << 5) + (hit ? __ffs(hit) - 1 : 0));
    }
    __syncwarp();   // the rows are free for the next call
    return res;
}

// One CTA per deferred item: the canonical prefix is built by the whole CTA in
// shared memory when the launch has room for the row (a.heavy_smem), else in
// global scratch (same canonical order, so bit-identical to the warp path);
// warp 0 runs the slot resolver; a rebuild is incremental over the tile
// summaries for a cached hub (incr_rebuild), else a CTA-wide rescan.
template <typename I, int BIAS, bool STREAM = false>
__device__ __forceinline__ void heavy_body(const DevGraph &g0, const LevelArgs &a) {
    __shared__ int s_flag, s_j, s_nz;
    __shared__ int32_t s_z[32];                 // zeroed neighbors of an incremental rebuild
    __shared__ float s_gm[INCR_SGROUPS];        // its group maxima
    __shared__ float s_row[32 * 33];            // its draws' staged tiles
    extern __shared__ float s_heavy[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    float *const P_global = a.heavy_scratch + (int64_t)blockIdx.x * a.heavy_stride;
    const uint32_t nh = __ldcg(a.n_heavy);
    unsigned long long my_bytes = 0, my_items = 0;
    for (uint32_t h = blockIdx.x; h < nh; h += gridDim.x) {
        const uint32_t it = a.heavy_list ? __ldcg(&a.heavy_list[h].it) : __ldcg(a.heavy + h);
        int l, N;
        bool push;
        item_level(a, it, l, N, push);
        const bool rec = a.sched && a.sched->mode == SCHED_RECORD;
        long long t0 = 0;
        if (rec && threadIdx.x == 0) t0 = clock64();
        const int32_t v = __ldcg(a.in_v + it);
        DevGraph g = g0;
        if (STREAM) {   // deferred by the warp pass, so its partition is resident
            const int part = v >> a.pbits;
            g.v.col = a.part_col[part];
            stream_bases(g, a, part);
        }
        const int32_t s = __ldcg(a.in_s + it);
        const uint32_t p = __ldcg(a.in_p + it);
        const int64_t beg = row_begin<I>(g, v);
        const int64_t d = row_begin<I>(g, v + 1) - beg;
        const bool in_smem = heavy_need(d) <= a.heavy_smem;
        if (!in_smem && heavy_need(d) > a.heavy_stride) {
            if (threadIdx.x == 0) atomicOr(a.err, ERR_SCRATCH);
            continue;
        }
        float *P = in_smem ? s_heavy : P_global;
        float *tsum = P + d;
        float *gcar = tsum + (d >> 5) + 1;
        uint32_t *zb = (uint32_t *)(gcar + (d >> 10) + 1);
        auto wfn = [&](int64_t i) { return edge_bias<I, BIAS>(g, beg + i); };
        bool indexed = g.cdf && g.cdf_bias == BIAS;   // cached prefix, searched through its index
        const bool indexed0 = indexed;
        unsigned long long rebuild_bytes = 0;         // counted prefix reads of the rebuilds
        // cached hub with tile summaries: rebuilds are incremental
        const bool incr = !STREAM && indexed && g.tsc && d > TSC_MIN_DEG;
        bool rebuilt = false;
        const IncrView iv = incr_view(P, d);
        float T = indexed ? g.cdf[beg + d - 1] : cta_canon_prefix(wfn, d, P, tsum, gcar, nullptr);
        const DrawCtx dc{a.k0, a.k1, p, (uint32_t)s, (uint32_t)l};
        SlotRng rng;
        SelState st;
        auto cand_of = [&](uint32_t x, bool act) -> int {
            const float t = act ? its_target(x, T) : 0.f;
            if (rebuilt) return incr_search(wfn, d, s_z, s_nz, iv, s_gm, s_row, t, act, lane);   // all lanes take part
            if (!act) return -1;
            return indexed ? (int)cdf_search(g, beg, d, t) : (int)search_upper(P, d, t);
        };
        bool zero = !(T > 0.f);
        // a pair item whose first phase failed at slot j0 (the entry's pad =
        // its pair index + 1; the slot and the accepted indices wait in the
        // consumed pair entry): the run goes on from there -- a rebuild
        // without the j0 selections, slot j0 from draw REJECT_ATTEMPTS
        int j0 = 0;
        if (a.heavy_list && a.pair_list && indexed && !zero) {
            const int pad = __ldcg(&a.heavy_list[h].pad);
            if (pad > 0 && d <= RESUME_MAX_DEG) {
                const uint16_t *ps = reinterpret_cast<const uint16_t *>(a.pair_list + (pad - 1));
                j0 = __ldcg(ps);
                if (j0 >= N) j0 = 0;
                if (warp == 0 && j0 > 0) {
                    st.j = j0;
                    if (lane < j0) st.sel = __ldcg(ps + 1 + lane);
                    if (lane == j0) st.A = REJECT_ATTEMPTS;
                }
            }
        }
        if (warp == 0 && !zero && j0 == 0) draw_pending(st, 0, N, lane, dc, rng, cand_of);
        for (bool resumed = j0 > 0;; resumed = false) {
            if (warp == 0) {
                int r = 0;
                if (resumed) r = 1;   // the rebuild after the failed first phase comes first
                else if (zero) zero_fill(st, N, lane);
                else r = resolve_slots(st, N, lane, dc, rng, cand_of);
                if (lane == 0) {
                    s_flag = r;
                    s_j = st.j;
                }
            }
            __syncthreads();
            const int need = s_flag, j = s_j;
            if (!need) break;
            if (incr) {
                if (warp == 0) {
                    if (lane < j) s_z[lane] = st.sel;
                    if (lane == 0) s_nz = j;
                }
                __syncthreads();
                T = incr_rebuild(g, wfn, beg, v, d, s_z, j, iv, s_gm);
                rebuilt = true;
                // the row's tile summaries, the touched tiles' biases, and per
                // later draw one line of running maxima and one tile of biases
                rebuild_bytes += 8ull * (unsigned long long)iv.ntiles + 128ull * (unsigned long long)j +
                                 256ull * (unsigned long long)N;
            } else {
                const int64_t nwords = (d + 31) >> 5;
                for (int64_t w = threadIdx.x; w < nwords; w += blockDim.x) zb[w] = 0u;
                __syncthreads();
                if (warp == 0 && lane < j) atomicOr(&zb[st.sel >> 5], 1u << (st.sel & 31));
                __syncthreads();
                T = cta_canon_prefix(wfn, d, P, tsum, gcar, zb);
                rebuild_bytes += 4ull * (unsigned long long)d;   // every bias of the row again
            }
            indexed = false;
            if (warp == 0) {
                if (!(T > 0.f)) zero = true;
                else draw_pending(st, j, N, lane, dc, rng, cand_of);
            }
        }
        if (warp == 0) {
            bool act = lane < N;
            int32_t dst = 0;
            if (act) {
                dst = Update(&g.v, __ldg(g.v.col + beg + st.sel), v);
                if (dst < 0 || dst >= g.v.n_vertices) {
                    atomicOr(a.err, ERR_UPDATE_RANGE);
                    dst = 0;
                }
            }
            unsigned long long ob = 0;
            uint32_t q = 0;
            if (a.heavy_list) {  // slots reserved by the batched first pass
                ob = __ldcg(&a.heavy_list[h].ob);
                q = __ldcg(&a.heavy_list[h].q);
            } else {
                if (lane == 0) {
                    ob = atomicAdd(a.o_count, (unsigned long long)N);
                    if (push) q = atomicAdd(a.n_out, (uint32_t)N);
                }
                ob = __shfl_sync(FULL, ob, 0);
                q = __shfl_sync(FULL, q, 0);
            }
            if (act) {
                int64_t pos = (int64_t)ob + lane;
                if (pos < a.cap) {
                    a.o_src[pos] = v;
                    a.o_dst[pos] = dst;
                    if (a.o_smp) a.o_smp[pos] = s;
                    if (a.o_dep) a.o_dep[pos] = l;
                }
                if (push) {
                    a.out_v[q + lane] = dst;
                    a.out_s[q + lane] = s;
                    a.out_p[q + lane] = p * (uint32_t)N + (uint32_t)lane;
                    if (a.out_dep) a.out_dep[q + lane] = l + 1;
                    if (a.out_beg) {
                        const int64_t nb = row_begin<I>(g, dst);
                        ((I *)a.out_beg)[q + lane] = (I)nb;
                        a.out_deg[q + lane] = (int32_t)(row_begin<I>(g, dst + 1) - nb);
                    }
                }
            }
        }
        my_items++;
        // a prefix built here reads every bias; a cached one is searched
        // through its index (about log2 d probes a draw)
        my_bytes += expansion_bytes<I, BIAS>(g, d, N, !indexed0, a, push) + rebuild_bytes +
                    (indexed0 ? (unsigned long long)N * 4ull * (64 - __clzll((unsigned long long)d)) : 0ull);
        __syncthreads();
        if (rec && threadIdx.x == 0)
            record_profile(a.sched, d, N, a.sched->vstats[v], __ldcg(a.n_in), l, 2 + a.cta_class, clock64() - t0);
    }
    if (threadIdx.x == 0) {
        atomicAdd(&a.bytes[1], my_bytes);
        atomicAdd(&a.items[1], my_items);
    }
}

template <typename I, int BIAS, bool STREAM = false>
__global__ void __launch_bounds__(1024)
k_expand_heavy(DevGraph g0, LevelArgs a) {
    heavy_body<I, BIAS, STREAM>(g0, a);
}

// ------------------------------------------------------------ walks
// Unbiased walks: one thread per walk (a step is a rowptr pair, one Philox
// word and one col read).  Equivalent to neighbor sampling with N = 1.
template <typename I>
__global__ void __launch_bounds__(WALK_THREADS)
k_walk_thread(DevGraph g, WalkArgs a) {
    __shared__ int32_t s_out[(WALK_THREADS / 32) * 4 * STAGE];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    WarpStage stg;
    stg.s_src = s_out + wib * 4 * STAGE;
    stg.s_dst = stg.s_src + STAGE;
    stg.s_smp = stg.s_dst + STAGE;
    stg.s_dep = stg.s_smp + STAGE;
    const OutArgs oa{a.o_src, a.o_dst, a.o_smp, a.o_dep, a.o_count, a.cap};
    const int stride = gridDim.x * blockDim.x;
    unsigned long long steps = 0;
    for (int base = blockIdx.x * blockDim.x; base < a.n; base += stride) {
        const int w = base + threadIdx.x;
        bool alive = w < a.n;
        int32_t v = 0;
        if (alive) {
            v = a.seeds[w];
            if (v < 0 || v >= g.v.n_vertices) {
                atomicOr(a.err, ERR_SEED_RANGE);
                alive = false;
            }
        }
        for (int t = 0; t < a.len; ++t) {
            if (!__any_sync(FULL, alive)) break;
            bool act = false;
            int32_t dst = 0;
            if (alive) {
                const int64_t beg = row_begin<I>(g, v), d = row_begin<I>(g, v + 1) - beg;
                if (d <= 0) {
                    alive = false;
                } else {
                    uint32_t idx = 0;
                    if (d > 1) {
                        uint4 b = philox(make_uint4(0u, (uint32_t)(a.base + w), (TAG_SAMPLE << 24) | (uint32_t)t, 0u),
                                         a.k0, a.k1);
                        idx = mulhi(b.x, (uint32_t)d);
                    }
                    dst = Update(&g.v, __ldg(g.v.col + beg + idx), v);
                    if (dst < 0 || dst >= g.v.n_vertices) {
                        atomicOr(a.err, ERR_UPDATE_RANGE);
                        dst = 0;
                    }
                    act = true;
                    ++steps;
                }
            }
            stg.push(oa, act, v, dst, a.base + w, t, lane);
            if (act) v = dst;
        }
    }
    stg.flush(oa, lane);
    unsigned long long tot = steps;
    for (int off = 16; off; off >>= 1) tot += __shfl_xor_sync(FULL, tot, off);
    if (lane == 0) {
        unsigned long long per = 2 * sizeof(I) + 4 + 4ull * (2 + (a.o_smp != nullptr) + (a.o_dep != nullptr));
        atomicAdd(&a.bytes[8], tot * per);
        atomicAdd(&a.items[8], tot);
    }
}

// Biased walks: one warp per walk; per step the warp builds the canonical
// prefix of the neighbor biases (shared memory up to WBUF, else per-warp
// global scratch) unless a CDF cache for this bias exists.
template <typename I, int BIAS>
__global__ void __launch_bounds__(WALK_THREADS)
k_walk_warp(DevGraph g, WalkArgs a) {
    constexpr int NW = WALK_THREADS / 32;
    __shared__ float s_P[NW * WBUF];
    __shared__ int32_t s_out[NW * 4 * STAGE];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    float *P = s_P + wib * WBUF;
    WarpStage stg;
    stg.s_src = s_out + wib * 4 * STAGE;
    stg.s_dst = stg.s_src + STAGE;
    stg.s_smp = stg.s_dst + STAGE;
    stg.s_dep = stg.s_smp + STAGE;
    const OutArgs oa{a.o_src, a.o_dst, a.o_smp, a.o_dep, a.o_count, a.cap};
    const bool cached = g.cdf && g.cdf_bias == BIAS;
    unsigned long long steps = 0, bytes = 0;
    const unsigned long long obytes = 4ull * (2 + (a.o_smp != nullptr) + (a.o_dep != nullptr));
    for (int w = gw; w < a.n; w += nw) {
        int32_t v = a.seeds[w];
        if (v < 0 || v >= g.v.n_vertices) {
            if (lane == 0) atomicOr(a.err, ERR_SEED_RANGE);
            continue;
        }
        for (int t = 0; t < a.len; ++t) {
            const int64_t beg = row_begin<I>(g, v), d = row_begin<I>(g, v + 1) - beg;
            if (d <= 0) break;
            int64_t idx = 0;
            bytes += 2 * sizeof(I) + 4 + obytes;
            if (d > 1) {
                const float *PP = nullptr;
                float T;
                if (cached) {
                    T = g.cdf[beg + d - 1];
                    bytes += 4ull * (64 - __clzll((unsigned long long)d));
                } else {
                    float *buf = P;
                    if (d > WBUF) {
                        if (d > a.scratch_stride) {
                            if (lane == 0) atomicOr(a.err, ERR_SCRATCH);
                            break;
                        }
                        buf = a.scratch + (int64_t)gw * a.scratch_stride;
                    }
                    auto wfn = [&](int64_t i) { return edge_bias<I, BIAS>(g, beg + i); };
                    T = warp_canon_prefix(wfn, d, buf, nullptr, lane);
                    PP = buf;
                    bytes += (BIAS == CSAW_BIAS_EDGE_WEIGHT || (BIAS == CSAW_BIAS_DEGREE && g.ebias))
                                 ? 4ull * d
                                 : (4ull + 2ull * sizeof(I)) * d;
                }
                if (T > 0.f) {
                    uint4 b = philox(make_uint4(0u, (uint32_t)(a.base + w), (TAG_SAMPLE << 24) | (uint32_t)t, 0u),
                                     a.k0, a.k1);
                    const float tt = its_target(b.x, T);
                    if (!cached) idx = search_upper(PP, d, tt);
                    else if (d > 1024) idx = warp_cdf_search(g, beg, d, tt, lane);
                    else idx = warp_search_upper(g.cdf + beg, d, tt, lane);
                }
            }
            int32_t dst = Update(&g.v, __ldg(g.v.col + beg + idx), v);
            if (dst < 0 || dst >= g.v.n_vertices) {
                if (lane == 0) atomicOr(a.err, ERR_UPDATE_RANGE);
                dst = 0;
            }
            stg.push(oa, lane == 0, v, dst, a.base + w, t, lane);
            v = dst;
            ++steps;
        }
    }
    stg.flush(oa, lane);
    if (lane == 0) {
        atomicAdd(&a.bytes[2], bytes);
        atomicAdd(&a.items[2], steps);
    }
}

// ------------------------------------------------------------- MDRW
// One warp per sample; frontier and its bias prefix in dynamic shared memory
// (F ints + F floats per warp).
template <typename I, int BIAS>
__global__ void k_mdrw(DevGraph g, WalkArgs a) {
    extern __shared__ int32_t s_dyn[];
    __shared__ int32_t s_out[(WALK_THREADS / 32) * 4 * STAGE];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    const int F = a.F;
    int32_t *f = s_dyn + (int64_t)wib * 2 * F;
    float *P = (float *)(f + F);
    WarpStage stg;
    stg.s_src = s_out + wib * 4 * STAGE;
    stg.s_dst = stg.s_src + STAGE;
    stg.s_smp = stg.s_dst + STAGE;
    stg.s_dep = stg.s_smp + STAGE;
    const OutArgs oa{a.o_src, a.o_dst, a.o_smp, a.o_dep, a.o_count, a.cap};
    unsigned long long steps = 0, bytes = 0;
    const unsigned long long obytes = 4ull * (2 + (a.o_smp != nullptr) + (a.o_dep != nullptr));
    for (int s = gw; s < a.n; s += nw) {
        for (int i = lane; i < F; i += 32) {
            int32_t v = a.seeds[(int64_t)s * F + i];
            if (v < 0 || v >= g.v.n_vertices) {
                atomicOr(a.err, ERR_SEED_RANGE);
                v = 0;
            }
            f[i] = v;
        }
        __syncwarp();
        for (int t = 0; t < a.len; ++t) {
            uint4 b = philox(make_uint4(0u, (uint32_t)(a.base + s), (TAG_MDRW << 24) | (uint32_t)t, 0u), a.k0, a.k1);
            int slot = 0;
            if (F > 1) {
                auto wfn = [&](int64_t i) -> float {
                    if constexpr (BIAS == CSAW_BIAS_UNBIASED) return 1.f;
                    else if constexpr (BIAS == CSAW_BIAS_DEGREE) return degree_f<I>(g, f[i]);
                    else return VertexBias(f[i], &g.v);
                };
                float T = warp_canon_prefix(wfn, F, P, nullptr, lane);
                if (T > 0.f) slot = (int)search_upper(P, F, its_target(b.x, T));
                bytes += BIAS == CSAW_BIAS_UNBIASED ? 0 : 2ull * sizeof(I) * F;
            }
            const int32_t v = f[slot];
            const int64_t beg = row_begin<I>(g, v), d = row_begin<I>(g, v + 1) - beg;
            bytes += 2 * sizeof(I);
            if (d > 0) {
                int32_t dst = Update(&g.v, __ldg(g.v.col + beg + mulhi(b.y, (uint32_t)d)), v);
                if (dst < 0 || dst >= g.v.n_vertices) {
                    if (lane == 0) atomicOr(a.err, ERR_UPDATE_RANGE);
                    dst = 0;
                }
                stg.push(oa, lane == 0, v, dst, a.base + s, t, lane);
                bytes += 4 + obytes;
                ++steps;
                __syncwarp();
                if (lane == 0) f[slot] = dst;
            }
            __syncwarp();
        }
    }
    stg.flush(oa, lane);
    if (lane == 0) {
        atomicAdd(&a.bytes[3], bytes);
        atomicAdd(&a.items[3], steps);
    }
}

// -------------------------------------------------------------- CDF cache
// Canonical prefix of every vertex's edge biases, written in place of the
// per-edge array cdf[E] (same canonical order, so searching it equals
// scanning on the fly).  One warp per vertex up to big_deg; vertices above go
// to k_cdf_build_big, one CTA each.
template <typename I, int BIAS>
__global__ void k_cdf_build(DevGraph g, float *cdf, int64_t big_deg, int64_t v0, int64_t v1) {
    const int lane = threadIdx.x & 31;
    const int64_t gw = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t v = v0 + gw; v < v1; v += nw) {
        const int64_t beg = row_begin<I>(g, v), d = row_begin<I>(g, v + 1) - beg;
        if (d <= 0 || d > big_deg) continue;
        auto wfn = [&](int64_t i) { return edge_bias<I, BIAS>(g, beg + i); };
        warp_canon_prefix(wfn, d, cdf + beg, nullptr, lane);
    }
}

template <typename I, int BIAS>
__global__ void k_cdf_build_big(DevGraph g, float *cdf, const int32_t *verts, int n, float *scratch,
                                int64_t stride) {
    float *tsum = scratch + (int64_t)blockIdx.x * stride;
    for (int k = blockIdx.x; k < n; k += gridDim.x) {
        const int32_t v = verts[k];
        const int64_t beg = row_begin<I>(g, v), d = row_begin<I>(g, v + 1) - beg;
        float *gcar = tsum + (d >> 5) + 1;
        auto wfn = [&](int64_t i) { return edge_bias<I, BIAS>(g, beg + i); };
        cta_canon_prefix(wfn, d, cdf + beg, tsum, gcar, nullptr);
    }
}

// Tile summaries (DevGraph::tsc) of the rows in verts: one CTA per row,
// a warp per tile, the same Kogge-Stone scan as the canonical prefix.
template <typename I, int BIAS>
__global__ void k_tile_summary(DevGraph g, float2 *out, const int32_t *verts, int n) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int k = blockIdx.x; k < n; k += gridDim.x) {
        const int32_t v = verts[k];
        const int64_t beg = row_begin<I>(g, v), d = row_begin<I>(g, v + 1) - beg;
        const int64_t ntiles = (d + 31) >> 5, base = tsc_slot(beg, v);
        for (int64_t t = warp; t < ntiles; t += nw) {
            const int64_t i = (t << 5) + lane;
            const float a = warp_ks_sum(i < d ? edge_bias<I, BIAS>(g, beg + i) : 0.f, lane);
            const float tot = __shfl_sync(FULL, a, 31);
            float m = i < d ? a : 0.f;
#pragma unroll
            for (int off = 16; off; off >>= 1) m = fmaxf(m, __shfl_xor_sync(FULL, m, off));
            if (lane == 0) out[base + t] = make_float2(tot, m);
        }
    }
}

// ------------------------------------------------------- per-sample dedup
// Hash set of (sample, vertex) keys with, per key, the smallest packed
// (level << 32 | lineage) of the items that carried it.  Open addressing,
// linear probing; the table holds at most half its slots.  A queue item is
// kept iff its packed value is the key's minimum, i.e. the vertex is new to
// its sample at this level and this item has the lowest lineage among the
// level's items that carry it.
constexpr unsigned long long DEDUP_EMPTY = ~0ull;

__device__ __forceinline__ unsigned long long dedup_key(int32_t s, int32_t v) {
    return ((unsigned long long)(uint32_t)s << 32) | (uint32_t)v;
}

__device__ __forceinline__ uint64_t dedup_slot(unsigned long long key, uint64_t mask) {
    unsigned long long h = key * 0x9E3779B97F4A7C15ull;
    h ^= h >> 29;
    return h & mask;
}

// Pass 1 over a level's queue (count *n): insert every item's key and fold
// its packed value in with atomicMin.
static __global__ void k_dedup_insert(const int32_t *qv, const int32_t *qs, const uint32_t *qp, const uint32_t *n,
                                      int level, unsigned long long *keys, unsigned long long *vals, uint64_t mask,
                                      int *err) {
    const uint32_t cnt = *n;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < cnt; i += gridDim.x * blockDim.x) {
        const int32_t v = qv[i];
        if (v < 0) continue;
        const unsigned long long key = dedup_key(qs[i], v);
        const unsigned long long val = ((unsigned long long)(uint32_t)level << 32) | qp[i];
        uint64_t h = dedup_slot(key, mask);
        bool done = false;
        for (uint64_t probe = 0; probe <= mask; ++probe) {
            const unsigned long long prev = atomicCAS(keys + h, DEDUP_EMPTY, key);
            if (prev == DEDUP_EMPTY || prev == key) {
                atomicMin(vals + h, val);
                done = true;
                break;
            }
            h = (h + 1) & mask;
        }
        if (!done) atomicOr(err, ERR_SCRATCH);
    }
}

// Pass 2: items that are not their key's minimum become empty (vertex -1,
// degree 0): the next level skips them; their edges were already emitted.
static __global__ void k_dedup_filter(int32_t *qv, const int32_t *qs, const uint32_t *qp, int32_t *qdeg,
                                      const uint32_t *n, int level, const unsigned long long *keys,
                                      const unsigned long long *vals, uint64_t mask) {
    const uint32_t cnt = *n;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < cnt; i += gridDim.x * blockDim.x) {
        const int32_t v = qv[i];
        if (v < 0) continue;
        const unsigned long long key = dedup_key(qs[i], v);
        const unsigned long long val = ((unsigned long long)(uint32_t)level << 32) | qp[i];
        uint64_t h = dedup_slot(key, mask);
        bool keep = false;
        for (uint64_t probe = 0; probe <= mask; ++probe) {
            const unsigned long long k = keys[h];
            if (k == key) {
                keep = vals[h] == val;
                break;
            }
            if (k == DEDUP_EMPTY) break;
            h = (h + 1) & mask;
        }
        if (!keep) {
            qv[i] = -1;
            if (qdeg) qdeg[i] = 0;
        }
    }
}

// Search index of a built prefix cache: c1[k] = cdf[32k + 31] and
// c2[u] = cdf[1024u + 1023] where those edges exist (others are never read).
// The index entries whose edge lies in [e0, e1): cdf1[k] = cdf[32k + 31],
// cdf2[u] = cdf[1024u + 1023] (cdf indexed by global edge; entries past the
// last edge are left as they are, zero).
static __global__ void k_cdf_index_range(const float *cdf, int64_t e0, int64_t e1, float *c1, float *c2) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t k = (e0 >> 5) + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k <= (e1 - 1) >> 5; k += stride) {
        const int64_t i = (k << 5) + 31;
        if (i >= e0 && i < e1) c1[k] = cdf[i];
    }
    for (int64_t u = (e0 >> 10) + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; u <= (e1 - 1) >> 10; u += stride) {
        const int64_t j = (u << 10) + 1023;
        if (j >= e0 && j < e1) c2[u] = cdf[j];
    }
}

static __global__ void k_cdf_index(const float *cdf, int64_t E, float *c1, int64_t n1, float *c2, int64_t n2) {
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n1; k += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = (k << 5) + 31;
        c1[k] = i < E ? cdf[i] : 0.f;
        if (k < n2) {
            const int64_t j = (k << 10) + 1023;
            c2[k] = j < E ? cdf[j] : 0.f;
        }
    }
}

// -------------------------------------------------------------- utilities
static __global__ void k_make_seeds(const int32_t *nonisolated, uint32_t n_non, int64_t n, uint32_t k0,
                             uint32_t k1, int32_t *out) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        uint4 b = philox(make_uint4((uint32_t)i, (uint32_t)(i >> 32), TAG_SEED << 24, 0u), k0, k1);
        out[i] = nonisolated[mulhi(b.x, n_non)];
    }
}

template <typename I>
__global__ void k_edge_degree(DevGraph g, float *ebias) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < g.v.n_edges;
         e += (int64_t)gridDim.x * blockDim.x)
        ebias[e] = degree_f<I>(g, __ldg(g.v.col + e));
}

}  // namespace csaw
