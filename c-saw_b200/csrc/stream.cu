// stream.cu -- partitioned ("streaming") sampling for graphs whose adjacency
// does not fit the device budget.
//
// Replaces C-SAW's streaming sampler (streaming/streaming_sampling.cu): its
// kernel (:199-384) consumed per-partition queues and pushed children into
// the queue of the child's partition (:359-371); its host loop (:597-714)
// copied 4 fixed partitions on 4 streams per round (with byte counts missing
// sizeof, :602, over a graph already fully copied by gpu_graph, :474) and
// synchronised the device between rounds.  Here:
//   - row offsets stay resident; column ids (and weights when the bias needs
//     them) stay in page-locked host memory, split into vertex-range
//     partitions of 2^k vertices;
//   - resident partitions live in one device arena of the byte budget, each
//     in a region of its own size (first fit), so many small partitions fit
//     beside a few large ones;
//   - the frontier is asynchronous: every pending item carries its depth,
//     and pending items are kept sorted by (partition, depth) (histogram,
//     scan, scatter).  A round processes all pending items of the resident
//     partitions, whatever their depth; only when no resident partition has
//     pending items are new ones loaded: the not-yet-visited partitions of
//     the current sweep with the most pending items per byte, as many as fit
//     once partitions without pending items are evicted.  A sweep ends when
//     every partition with pending items has been visited.  Walks that stay
//     within resident partitions advance many steps per load;
//   - copies run on a copy stream; each partition has a ready event (copy
//     done) and a free event (last kernel using it done), so an eviction
//     waits only for that partition's kernels;
//   - the expansion kernel runs once per round over all pending items,
//     whatever their depths (each item carries its depth; its fanout and
//     whether it pushes children follow from it): each item reads the
//     column/weight bases of its partition from a per-round table (re-based
//     onto the partition's region, so col[e] of any edge of the partition is
//     read from HBM), and items of partitions not in the round are skipped;
//     a walk step whose next vertex is in a partition of the round goes on
//     in the same warp;
//   - walks are neighbor sampling with N = 1 (same keys, same output).
// Because every draw is keyed by (sample, depth, lineage, slot, draw), the
// output equals the in-memory output exactly, whatever the processing order.
#include <cuda_runtime.h>

#include <algorithm>
#include <map>
#include <string>
#include <vector>

#include "csaw.h"
#include "csaw_host.h"
#include "csaw_internal.h"
#include "kernels_sample.cuh"

using namespace csaw;

namespace {

constexpr int STREAM_GROUPS = 4;   // launches a loading round is split into (copy/compute overlap)

struct StreamCounters {
    unsigned long long out_count;
    unsigned long long bytes[8];
    unsigned long long items[8];
    uint32_t n_next;      // unsorted new items (children)
    uint32_t n_heavy;
    int err;
    uint32_t n_pend;      // pending items, sorted by (partition, depth)
};

// Pending-set histogram over (partition, depth) keys; items of partitions
// flagged in skip (processed this round) are left out.
__global__ void k_key_hist(const int32_t *v, const int32_t *dep, const uint32_t *n, int pbits, int D,
                           const uint8_t *skip, uint32_t *counts) {
    const uint32_t m = *n;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
        const int part = v[i] >> pbits;
        if (skip && skip[part]) continue;
        atomicAdd(&counts[part * D + dep[i]], 1u);
    }
}

__global__ void k_key_scatter(const int32_t *v, const int32_t *s, const uint32_t *p, const int32_t *dep,
                              const uint32_t *n, int pbits, int D, const uint8_t *skip, uint32_t *cursor, int32_t *ov,
                              int32_t *os, uint32_t *op, int32_t *od) {
    const uint32_t m = *n;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
        const int part = v[i] >> pbits;
        if (skip && skip[part]) continue;
        const uint32_t pos = atomicAdd(&cursor[part * D + dep[i]], 1u);
        ov[pos] = v[i];
        os[pos] = s[i];
        op[pos] = p[i];
        od[pos] = dep[i];
    }
}


// Exclusive scan of n counts into offsets[0..n] and a cursor copy (one block).
__global__ void k_part_scan(const uint32_t *counts, int npart, uint32_t *offsets, uint32_t *cursor) {
    __shared__ uint32_t carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int base = 0; base < npart; base += blockDim.x) {
        const int i = base + threadIdx.x;
        const uint32_t c = i < npart ? counts[i] : 0u;
        // block-wide inclusive scan by warps
        uint32_t x = c;
        const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
        for (int off = 1; off < 32; off <<= 1) {
            uint32_t up = __shfl_up_sync(0xffffffffu, x, off);
            if (lane >= off) x += up;
        }
        __shared__ uint32_t wsum[32];
        if (lane == 31) wsum[w] = x;
        __syncthreads();
        if (w == 0) {
            uint32_t y = lane < (int)(blockDim.x >> 5) ? wsum[lane] : 0u;
            for (int off = 1; off < 32; off <<= 1) {
                uint32_t up = __shfl_up_sync(0xffffffffu, y, off);
                if (lane >= off) y += up;
            }
            wsum[lane] = y;
        }
        __syncthreads();
        const uint32_t incl = x + (w ? wsum[w - 1] : 0u) + carry;
        if (i < npart) {
            offsets[i] = incl - c;
            cursor[i] = incl - c;
        }
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) carry = incl;
        __syncthreads();
    }
    if (threadIdx.x == 0) offsets[npart] = carry;
}

struct Buf {
    void *p = nullptr;
    size_t n = 0;
};

int grow(Buf &b, size_t bytes) {
    if (b.n >= bytes) return 0;
    cudaFree(b.p);
    b.p = nullptr;
    b.n = 0;
    if (cudaMalloc(&b.p, bytes) != cudaSuccess) {
        cudaGetLastError();
        return csaw_host_fail(CSAW_ERR_NOMEM, "streaming workspace allocation failed");
    }
    b.n = bytes;
    return 0;
}

}  // namespace

struct csaw_stream_graph_s {
    int device = 0, sm_count = 148;
    int64_t V = 0, E = 0, max_pedges = 0, maxdeg = 0;
    int idx64 = 0, pbits = 20, npart = 0;
    std::vector<int64_t> pbeg;        // first edge of each partition, npart + 1
    void *d_rowptr = nullptr;
    const int32_t *h_col = nullptr;
    const float *h_w = nullptr;
    bool reg_col = false, reg_w = false;
    int nslots = 0;                   // largest partitions the budget holds (reported)
    unsigned char *arena = nullptr;   // resident partitions, one region each
    int64_t arena_bytes = 0;
    std::map<int64_t, int64_t> free_regions;   // offset -> bytes
    std::vector<int64_t> res_off;     // per partition: region offset, or -1
    std::vector<int64_t> res_bytes;
    std::vector<char> res_w;          // what the region holds beside the columns (a Second)
    std::vector<int> resident;        // resident partitions, in load order
    std::vector<cudaEvent_t> ready, freed;   // per partition, created on first load
    cudaStream_t copy = nullptr;
    Buf q[3][4], counts, offsets, cursor, heavy, hscratch, ctr, skip, ptab;
    // Prefix cache per bias kind (csaw_stream_graph_cache): the canonical
    // prefix of every row in page-locked host memory, streamed in place of the
    // weights, and its two index levels resident on the device.
    float *h_cdf[4] = {};
    float *d_idx[4] = {};             // cdf1 [(E + 31) / 32], then cdf2 [(E + 1023) / 1024]
    StreamCounters *hctr = nullptr;
    int64_t loads = 0, hits = 0, bytes_h2d = 0, launches = 0;
    // Read in place (CSAW_STREAM_OPT_READ_IN_PLACE): device addresses of the
    // page-locked host arrays, null where not mapped
    bool read_in_place = true;
    const int32_t *dv_col = nullptr;
    const float *dv_w = nullptr, *dv_cdf[4] = {};
    int64_t host_items = 0;           // pending items served from host memory
};

namespace {

#define SCK(x)                                                                      \
    do {                                                                            \
        cudaError_t e_ = (x);                                                       \
        if (e_ != cudaSuccess) {                                                    \
            cudaGetLastError();                                                     \
            return csaw_host_fail(CSAW_ERR_CUDA, (std::string(#x) + ": " + cudaGetErrorString(e_)).c_str()); \
        }                                                                           \
    } while (0)

#define STRY(x)              \
    do {                     \
        int rc_ = (x);       \
        if (rc_) return rc_; \
    } while (0)

// What a partition's region holds beside its columns: nothing, its weights,
// or its rows' canonical prefix for bias kind b (SECOND_CDF + b).
enum : int { SECOND_NONE = 0, SECOND_W = 1, SECOND_CDF = 2 };

int64_t region_bytes(const csaw_stream_graph_s *g, int part, int second) {
    const int64_t ne = g->pbeg[part + 1] - g->pbeg[part];
    const int64_t colb = (4 * std::max<int64_t>(ne, 1) + 255) & ~255ll;
    return second != SECOND_NONE ? 2 * colb : colb;
}

// First-fit region of `bytes` in the arena, or -1.
int64_t region_alloc(csaw_stream_graph_s *g, int64_t bytes) {
    for (auto it = g->free_regions.begin(); it != g->free_regions.end(); ++it) {
        if (it->second < bytes) continue;
        const int64_t off = it->first, rem = it->second - bytes;
        g->free_regions.erase(it);
        if (rem > 0) g->free_regions[off + bytes] = rem;
        return off;
    }
    return -1;
}

void region_free(csaw_stream_graph_s *g, int64_t off, int64_t bytes) {
    auto it = g->free_regions.emplace(off, bytes).first;
    auto nx = std::next(it);
    if (nx != g->free_regions.end() && it->first + it->second == nx->first) {
        it->second += nx->second;
        g->free_regions.erase(nx);
    }
    if (it != g->free_regions.begin()) {
        auto pv = std::prev(it);
        if (pv->first + pv->second == it->first) {
            pv->second += it->second;
            g->free_regions.erase(it);
        }
    }
}

// Drops partition `part` from the device; later copies into its region wait
// for its last kernel.
int evict(csaw_stream_graph_s *g, int part) {
    SCK(cudaStreamWaitEvent(g->copy, g->freed[part], 0));
    region_free(g, g->res_off[part], g->res_bytes[part]);
    g->res_off[part] = -1;
    g->resident.erase(std::find(g->resident.begin(), g->resident.end(), part));
    return 0;
}

// Makes `part` resident (with the second array `second` the job needs),
// evicting partitions that are neither protected nor have pending items,
// oldest first; *ok is false (nothing changed) when it does not fit without
// evicting those.
int make_resident(csaw_stream_graph_s *g, int part, int second, const std::vector<char> &protect,
                  const std::vector<int64_t> &pend, bool *ok) {
    *ok = false;
    const bool with_w = second != SECOND_NONE;
    if (g->res_off[part] >= 0) {
        if (!with_w || g->res_w[part] == second) {
            g->hits++;
            *ok = true;
            return 0;
        }
        STRY(evict(g, part));   // resident without the array this job needs: reload
    }
    const int64_t bytes = region_bytes(g, part, second);
    int64_t off = region_alloc(g, bytes);
    while (off < 0) {
        int victim = -1;
        for (int q : g->resident)   // nothing pending there, oldest first
            if (!protect[q] && pend[q] == 0) {
                victim = q;
                break;
            }
        if (victim < 0)
            for (int q : g->resident)   // or unusable by this job (weights missing)
                if (!protect[q] && with_w && g->res_w[q] != second) {
                    victim = q;
                    break;
                }
        if (victim < 0) return 0;
        STRY(evict(g, victim));
        off = region_alloc(g, bytes);
    }
    if (!g->ready[part]) {
        SCK(cudaEventCreateWithFlags(&g->ready[part], cudaEventDisableTiming));
        SCK(cudaEventCreateWithFlags(&g->freed[part], cudaEventDisableTiming));
    }
    const int64_t e0 = g->pbeg[part], ne = g->pbeg[part + 1] - e0;
    if (ne > 0) {
        SCK(cudaMemcpyAsync(g->arena + off, g->h_col + e0, sizeof(int32_t) * ne, cudaMemcpyHostToDevice, g->copy));
        g->bytes_h2d += 4 * ne;
        if (with_w) {
            const float *src2 = second == SECOND_W ? g->h_w : g->h_cdf[second - SECOND_CDF];
            SCK(cudaMemcpyAsync(g->arena + off + bytes / 2, src2 + e0, sizeof(float) * ne, cudaMemcpyHostToDevice,
                                g->copy));
            g->bytes_h2d += 4 * ne;
        }
    }
    SCK(cudaEventRecord(g->ready[part], g->copy));
    g->res_off[part] = off;
    g->res_bytes[part] = bytes;
    g->res_w[part] = (char)second;
    g->resident.push_back(part);
    g->loads++;
    *ok = true;
    return 0;
}



template <typename I, int BIAS>
int run_stream(csaw_stream_graph_s *g, const csaw_params *p, const int fan[], const int32_t *seeds, int32_t *src,
               int32_t *dst, int32_t *smp, int32_t *dep, int64_t cap, cudaStream_t st) {
    constexpr bool BIASED = BIAS != CSAW_BIAS_UNBIASED;
    // the prefix cache of this bias (if built) is streamed in place of the
    // weights; otherwise the weights, when the bias reads them
    const bool cached = BIASED && g->h_cdf[BIAS];
    const int second = cached ? SECOND_CDF + BIAS
                              : (((BIAS == CSAW_BIAS_EDGE_WEIGHT || BIAS == CSAW_BIAS_HOOK) && g->h_w) ? SECOND_W
                                                                                                     : SECOND_NONE);
    const int S = p->n_samples, F = p->mode == CSAW_MODE_WALK ? 1 : p->frontier_size, D = p->depth;
    // pending items at once: at most every item of every level
    double per = F, lvl = F;
    for (int l = 0; l + 1 < D; ++l) {
        lvl *= fan[l];
        per += lvl;
    }
    if (lvl > 4294967295.0) return csaw_host_fail(CSAW_ERR_INVALID, "lineage items exceed 2^32");
    if (per * S > 2.0e9) return csaw_host_fail(CSAW_ERR_INVALID, "the frontier exceeds 2e9 items");
    const int64_t qcap = (int64_t)(per * S) + 32;
    const int nbins = g->npart * D;
    for (auto &qq : g->q)
        for (auto &b : qq) STRY(grow(b, sizeof(int32_t) * (size_t)qcap));
    STRY(grow(g->counts, sizeof(uint32_t) * (size_t)nbins));
    STRY(grow(g->cursor, sizeof(uint32_t) * (size_t)nbins));
    STRY(grow(g->offsets, sizeof(uint32_t) * (size_t)(nbins + 1)));
    STRY(grow(g->ctr, sizeof(StreamCounters)));
    STRY(grow(g->skip, (size_t)g->npart));
    STRY(grow(g->ptab, sizeof(void *) * 2 * (size_t)g->npart * STREAM_GROUPS));
    int hblocks = 0;
    int64_t hstride = 0;
    if (BIASED && g->maxdeg > WBUF) {
        STRY(grow(g->heavy, sizeof(uint32_t) * (size_t)qcap));
        hstride = (g->maxdeg + 2 * ((g->maxdeg >> 5) + 1) + (g->maxdeg >> 10) + 1 + 8 + 63) & ~63ll;
        hblocks = g->sm_count;
        while (hblocks > 1 && (int64_t)hblocks * hstride * 4 > (1ll << 30)) hblocks /= 2;
        STRY(grow(g->hscratch, sizeof(float) * (size_t)(hstride * hblocks)));
    }
    StreamCounters *c = (StreamCounters *)g->ctr.p;
    uint32_t *d_counts = (uint32_t *)g->counts.p;
    uint8_t *d_skip = (uint8_t *)g->skip.p;
    SCK(cudaMemsetAsync(c, 0, sizeof(StreamCounters), st));
    auto qv = [&](int k, int a) { return (int32_t *)g->q[k][a].p; };
    const int U = 2;      // unsorted new items
    int A = 0, B = 1;     // sorted pending / scratch for the next sorted pending
    const int bgrid = g->sm_count * 4;
    // pending := (pending items of partitions not flagged in skip) + new items,
    // sorted by (partition, depth); new := empty
    auto rebin = [&](bool use_skip) -> int {
        const uint8_t *sk = use_skip ? d_skip : nullptr;
        SCK(cudaMemsetAsync(d_counts, 0, sizeof(uint32_t) * (size_t)nbins, st));
        k_key_hist<<<bgrid, 256, 0, st>>>(qv(A, 0), qv(A, 3), &c->n_pend, g->pbits, D, sk, d_counts);
        k_key_hist<<<bgrid, 256, 0, st>>>(qv(U, 0), qv(U, 3), &c->n_next, g->pbits, D, nullptr, d_counts);
        k_part_scan<<<1, 1024, 0, st>>>(d_counts, nbins, (uint32_t *)g->offsets.p, (uint32_t *)g->cursor.p);
        k_key_scatter<<<bgrid, 256, 0, st>>>(qv(A, 0), qv(A, 1), (const uint32_t *)qv(A, 2), qv(A, 3), &c->n_pend,
                                             g->pbits, D, sk, (uint32_t *)g->cursor.p, qv(B, 0), qv(B, 1),
                                             (uint32_t *)qv(B, 2), qv(B, 3));
        k_key_scatter<<<bgrid, 256, 0, st>>>(qv(U, 0), qv(U, 1), (const uint32_t *)qv(U, 2), qv(U, 3), &c->n_next,
                                             g->pbits, D, nullptr, (uint32_t *)g->cursor.p, qv(B, 0), qv(B, 1),
                                             (uint32_t *)qv(B, 2), qv(B, 3));
        SCK(cudaMemcpyAsync(&c->n_pend, (uint32_t *)g->offsets.p + nbins, sizeof(uint32_t), cudaMemcpyDeviceToDevice,
                            st));
        SCK(cudaMemsetAsync(&c->n_next, 0, sizeof(uint32_t), st));
        std::swap(A, B);
        g->launches += 5;
        return 0;
    };
    const uint32_t n0 = (uint32_t)((int64_t)S * F);
    k_init_queue<<<(n0 + 255) / 256, 256, 0, st>>>(seeds, n0, F, (int)p->sample_base, g->V, qv(U, 0), qv(U, 1),
                                                   (uint32_t *)qv(U, 2), &c->n_next, &c->err);
    SCK(cudaMemsetAsync(qv(U, 3), 0, sizeof(int32_t) * (size_t)n0, st));
    g->launches++;
    STRY(rebin(false));
    int grid = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&grid, k_expand_warp<I, BIAS, true>, EXPAND_THREADS, 0);
    grid = (grid > 0 ? grid : 1) * g->sm_count;
    std::vector<uint32_t> h_counts((size_t)nbins);
    std::vector<int64_t> h_off((size_t)nbins + 1), pend((size_t)g->npart);
    std::vector<uint8_t> h_skip((size_t)g->npart);
    std::vector<const void *> h_tab(2 * (size_t)g->npart);
    std::vector<char> visited((size_t)g->npart, 0), in_round((size_t)g->npart, 0);
    // Read in place: every round processes every pending item; partitions in
    // the arena are read from HBM, the others from their page-locked host
    // arrays through the device's mapping (a hop then moves one prefix line
    // and one column over the link instead of its whole partition).  Free
    // arena space still takes the partitions of most pending items per byte,
    // which serve the rounds and jobs after their copies land; nothing is
    // evicted for them.
    const float *dv_second =
        second == SECOND_NONE ? nullptr : (second == SECOND_W ? g->dv_w : g->dv_cdf[second - SECOND_CDF]);
    const bool rip = g->read_in_place && g->dv_col && (second == SECOND_NONE || dv_second);
    const std::vector<char> protect_all((size_t)g->npart, 1);
    std::vector<int> served;
    for (;;) {
        SCK(cudaMemcpyAsync(h_counts.data(), d_counts, sizeof(uint32_t) * (size_t)nbins, cudaMemcpyDeviceToHost, st));
        SCK(cudaStreamSynchronize(st));
        h_off[0] = 0;
        for (int k = 0; k < nbins; ++k) h_off[k + 1] = h_off[k] + h_counts[k];
        if (h_off[nbins] == 0) break;
        for (int q = 0; q < g->npart; ++q) {
            pend[q] = 0;
            for (int l = 0; l < D; ++l) pend[q] += h_counts[(size_t)q * D + l];
        }
        // this round: the resident partitions with pending items (with the
        // weights this job needs); if none, the next partitions of the sweep.
        // Read in place: every partition with pending items.
        std::vector<int> round;
        bool loading = false;   // this round copies partitions in
        if (rip) {
            std::vector<int> cand;
            for (int q = 0; q < g->npart; ++q) {
                if (pend[q] > 0) round.push_back(q);
                if (pend[q] > 0 && g->res_off[q] < 0) cand.push_back(q);
            }
            std::stable_sort(cand.begin(), cand.end(), [&](int x, int y) {
                return (double)pend[x] * (double)region_bytes(g, y, second) >
                       (double)pend[y] * (double)region_bytes(g, x, second);
            });
            for (int q : cand) {   // into free space only
                bool ok = false;
                STRY(make_resident(g, q, second, protect_all, pend, &ok));
            }
        } else {
            for (int q : g->resident)
                if (pend[q] > 0 && (second == SECOND_NONE || g->res_w[q] == second)) round.push_back(q);
        }
        std::fill(in_round.begin(), in_round.end(), 0);
        if (round.empty()) {
            std::vector<int> cand;
            for (int q = 0; q < g->npart; ++q)
                if (pend[q] > 0 && !visited[q]) cand.push_back(q);
            if (cand.empty()) {   // a new sweep
                std::fill(visited.begin(), visited.end(), 0);
                for (int q = 0; q < g->npart; ++q)
                    if (pend[q] > 0) cand.push_back(q);
            }
            // most pending items per byte first
            std::stable_sort(cand.begin(), cand.end(), [&](int x, int y) {
                return (double)pend[x] * (double)region_bytes(g, y, second) >
                       (double)pend[y] * (double)region_bytes(g, x, second);
            });
            for (int q : cand) {
                bool ok = false;
                STRY(make_resident(g, q, second, in_round, pend, &ok));
                if (!ok) break;
                in_round[q] = 1;
                visited[q] = 1;
                round.push_back(q);
            }
            if (round.empty()) return csaw_host_fail(CSAW_ERR_INVALID, "no partition fits the device budget");
            loading = true;
        }
        // Launches over all pending items, each with a table of some of the
        // round's partitions (every other partition's items are skipped and
        // stay pending).  A loading round is split, in load order, into up
        // to STREAM_GROUPS groups, each launched as soon as its own
        // partitions have arrived, so the copies of later groups overlap the
        // sampling of earlier ones; a round of resident partitions is one
        // launch.
        std::fill(h_skip.begin(), h_skip.end(), 0);
        for (int part : round) h_skip[part] = 1;
        const int ngroups = loading ? std::min<int>(STREAM_GROUPS, (int)round.size()) : 1;
        for (int k = 0; k < ngroups; ++k) {
            const size_t lo = round.size() * k / ngroups, hi = round.size() * (k + 1) / ngroups;
            std::fill(h_tab.begin(), h_tab.end(), nullptr);
            served.clear();
            if (rip) {   // every partition: its copy in the arena once landed, else the host array
                bool pending_copy = false;
                for (int q = 0; q < g->npart; ++q) {
                    bool dev = g->res_off[q] >= 0 && (second == SECOND_NONE || g->res_w[q] == second);
                    if (dev && cudaEventQuery(g->ready[q]) != cudaSuccess) {
                        dev = false;
                        pending_copy = true;
                    }
                    if (dev) {
                        unsigned char *base = g->arena + g->res_off[q];
                        h_tab[q] = (const int32_t *)base - g->pbeg[q];
                        if (g->res_w[q]) h_tab[g->npart + q] = (const float *)(base + g->res_bytes[q] / 2) - g->pbeg[q];
                        served.push_back(q);
                    } else {
                        h_tab[q] = g->dv_col;
                        h_tab[g->npart + q] = dv_second;
                        g->host_items += pend[q];
                    }
                }
                if (pending_copy) cudaGetLastError();   // "not ready" is no error
            }
            for (size_t r = lo; r < hi && !rip; ++r) {
                const int part = round[r];
                SCK(cudaStreamWaitEvent(st, g->ready[part], 0));
                unsigned char *base = g->arena + g->res_off[part];
                h_tab[part] = (const int32_t *)base - g->pbeg[part];
                if (g->res_w[part])
                    h_tab[g->npart + part] = (const float *)(base + g->res_bytes[part] / 2) - g->pbeg[part];
                served.push_back(part);
            }
            const void **tab = (const void **)g->ptab.p + (size_t)k * 2 * g->npart;
            SCK(cudaMemcpyAsync(tab, h_tab.data(), sizeof(void *) * h_tab.size(), cudaMemcpyHostToDevice, st));
            DevGraph dg{};
            dg.v.rowptr = g->d_rowptr;
            dg.v.rowptr_is_64 = g->idx64;
            dg.v.n_vertices = g->V;
            dg.v.n_edges = g->E;
            dg.cdf_bias = cached ? BIAS : -1;
            LevelArgs a{};
            a.in_v = qv(A, 0);
            a.in_s = qv(A, 1);
            a.in_p = (const uint32_t *)qv(A, 2);
            a.in_dep = qv(A, 3);
            a.n_in = &c->n_pend;
            a.part_col = (const int32_t *const *)tab;
            a.part_w = (const float *const *)(tab + g->npart);
            a.pbits = g->pbits;
            a.part_cdf = cached ? 1 : 0;
            if (cached) {
                a.cdf1_all = g->d_idx[BIAS];
                a.cdf2_all = g->d_idx[BIAS] + ((g->E + 31) >> 5);
                a.host_w = g->reg_w ? g->h_w : nullptr;   // page-locked in place: device-readable
            }
            a.out_v = qv(U, 0);
            a.out_s = qv(U, 1);
            a.out_p = (uint32_t *)qv(U, 2);
            a.out_dep = qv(U, 3);
            a.n_out = &c->n_next;
            a.heavy = (uint32_t *)g->heavy.p;
            a.n_heavy = &c->n_heavy;
            a.heavy_scratch = (float *)g->hscratch.p;
            a.heavy_stride = hstride;
            a.o_src = src;
            a.o_dst = dst;
            a.o_smp = smp;
            a.o_dep = dep;
            a.o_count = &c->out_count;
            a.cap = cap;
            a.bytes = c->bytes;
            a.items = c->items;
            a.err = &c->err;
            a.k0 = (uint32_t)p->seed;
            a.k1 = (uint32_t)(p->seed >> 32);
            a.D = D;
            for (int l = 0; l < D; ++l) a.fan[l] = (uint8_t)fan[l];
            if (hblocks) SCK(cudaMemsetAsync(&c->n_heavy, 0, sizeof(uint32_t), st));
            k_expand_warp<I, BIAS, true><<<grid, EXPAND_THREADS, 0, st>>>(dg, a);
            g->launches++;
            if (hblocks) {
                k_expand_heavy<I, BIAS, true><<<hblocks, HEAVY_THREADS, 0, st>>>(dg, a);
                g->launches++;
            }
            for (int part : served) SCK(cudaEventRecord(g->freed[part], st));
        }
        SCK(cudaMemcpyAsync(d_skip, h_skip.data(), (size_t)g->npart, cudaMemcpyHostToDevice, st));
        STRY(rebin(true));
    }
    SCK(cudaGetLastError());
    SCK(cudaMemcpyAsync(g->hctr, c, sizeof(StreamCounters), cudaMemcpyDeviceToHost, st));
    SCK(cudaStreamSynchronize(st));
    return 0;
}

int check_stream_params(const csaw_params *p, int fan[CSAW_MAX_DEPTH]) {
    if (!p) return csaw_host_fail(CSAW_ERR_INVALID, "params is NULL");
    if (p->mode == CSAW_MODE_MDRW)
        return csaw_host_fail(CSAW_ERR_INVALID, "streaming runs neighbor sampling and walks");
    if (p->mode != CSAW_MODE_NEIGHBOR && p->mode != CSAW_MODE_WALK)
        return csaw_host_fail(CSAW_ERR_INVALID, "unknown mode");
    if (p->bias < CSAW_BIAS_UNBIASED || p->bias > CSAW_BIAS_HOOK) return csaw_host_fail(CSAW_ERR_INVALID, "unknown bias");
    if (p->flags) return csaw_host_fail(CSAW_ERR_INVALID, "params flags (dedup) are not supported by the streaming graph");
    if (p->n_samples < 0 || p->frontier_size < 1 || p->depth < 0 || p->depth > CSAW_MAX_DEPTH)
        return csaw_host_fail(CSAW_ERR_INVALID, "bad n_samples / frontier_size / depth (streaming depth <= 64)");
    if (p->sample_base < 0 || p->sample_base + p->n_samples > INT32_MAX)
        return csaw_host_fail(CSAW_ERR_INVALID, "sample ids must fit int32");
    for (int l = 0; l < p->depth; ++l) {
        fan[l] = p->mode == CSAW_MODE_WALK ? 1 : (p->fanout[l] ? p->fanout[l] : p->neighbor_size);
        if (fan[l] < 1 || fan[l] > MAX_FANOUT) return csaw_host_fail(CSAW_ERR_INVALID, "NeighborSize must be in [1, 32]");
    }
    return 0;
}

}  // namespace

extern "C" int csaw_stream_graph_create(const void *rowptr, int rowptr_is_64, const int32_t *col, const float *weights,
                                        int64_t n_vertices, int64_t n_edges, int partition_bits,
                                        int64_t slot_budget_bytes, csaw_stream_graph *out) {
    if (!out) return csaw_host_fail(CSAW_ERR_INVALID, "out is NULL");
    *out = nullptr;
    if (!rowptr || n_vertices < 1 || n_edges < 0 || (n_edges > 0 && !col))
        return csaw_host_fail(CSAW_ERR_INVALID, "bad CSR arguments");
    if (n_vertices >= (1ll << 31)) return csaw_host_fail(CSAW_ERR_INVALID, "vertex ids must fit int32");
    if (partition_bits < 4 || partition_bits > 30) return csaw_host_fail(CSAW_ERR_INVALID, "partition_bits in [4, 30]");
    if (!rowptr_is_64 && n_edges >= (1ll << 31)) return csaw_host_fail(CSAW_ERR_INVALID, "E >= 2^31 needs int64 rowptr");
    auto rp = [&](int64_t v) -> int64_t {
        return rowptr_is_64 ? ((const int64_t *)rowptr)[v] : (int64_t)((const int32_t *)rowptr)[v];
    };
    if (rp(0) != 0 || rp(n_vertices) != n_edges) return csaw_host_fail(CSAW_ERR_INVALID, "rowptr[0] != 0 or rowptr[V] != E");
    int64_t maxdeg = 0;
    for (int64_t v = 0; v < n_vertices; ++v) {
        const int64_t d = rp(v + 1) - rp(v);
        if (d < 0) return csaw_host_fail(CSAW_ERR_INVALID, "rowptr is not monotone");
        maxdeg = std::max(maxdeg, d);
    }
    for (int64_t e = 0; e < n_edges; ++e)
        if (col[e] < 0 || col[e] >= n_vertices) return csaw_host_fail(CSAW_ERR_INVALID, "col entry out of range");
    auto *g = new csaw_stream_graph_s();
    cudaGetDevice(&g->device);
    cudaDeviceGetAttribute(&g->sm_count, cudaDevAttrMultiProcessorCount, g->device);
    g->V = n_vertices;
    g->E = n_edges;
    g->idx64 = rowptr_is_64 ? 1 : 0;
    g->maxdeg = maxdeg;
    g->pbits = partition_bits;
    g->npart = (int)((n_vertices + (1ll << partition_bits) - 1) >> partition_bits);
    g->pbeg.resize((size_t)g->npart + 1);
    for (int q = 0; q <= g->npart; ++q) g->pbeg[q] = rp(std::min<int64_t>((int64_t)q << partition_bits, n_vertices));
    for (int q = 0; q < g->npart; ++q) g->max_pedges = std::max(g->max_pedges, g->pbeg[q + 1] - g->pbeg[q]);
    g->h_col = col;
    g->h_w = weights;
    auto bail = [&](const char *msg, int code) {
        csaw_stream_graph_destroy(g);
        return csaw_host_fail(code, msg);
    };
    const size_t rsz = (size_t)(n_vertices + 1) * (rowptr_is_64 ? 8 : 4);
    if (cudaMalloc(&g->d_rowptr, rsz) != cudaSuccess) return bail("rowptr allocation failed", CSAW_ERR_NOMEM);
    if (cudaMemcpy(g->d_rowptr, rowptr, rsz, cudaMemcpyHostToDevice) != cudaSuccess)
        return bail("rowptr copy failed", CSAW_ERR_CUDA);
    // page-lock the caller's arrays in place so partition copies are async DMA
    if (n_edges > 0) {
        g->reg_col = cudaHostRegister((void *)col, sizeof(int32_t) * n_edges, cudaHostRegisterDefault) == cudaSuccess;
        if (weights)
            g->reg_w = cudaHostRegister((void *)weights, sizeof(float) * n_edges, cudaHostRegisterDefault) == cudaSuccess;
        cudaGetLastError();
        // device addresses of the registered arrays, for reads in place
        void *dp = nullptr;
        if (g->reg_col && cudaHostGetDevicePointer(&dp, (void *)col, 0) == cudaSuccess) g->dv_col = (const int32_t *)dp;
        if (g->reg_w && cudaHostGetDevicePointer(&dp, (void *)weights, 0) == cudaSuccess) g->dv_w = (const float *)dp;
        cudaGetLastError();
    }
    const int64_t per_max = std::max<int64_t>(g->max_pedges, 1) * (weights ? 8 : 4);
    int64_t ns = slot_budget_bytes / per_max;
    if (ns > g->npart) ns = g->npart;
    if (ns < std::min(2, g->npart)) return bail("slot budget holds fewer than 2 partitions", CSAW_ERR_INVALID);
    g->nslots = (int)ns;
    // regions are 256-byte aligned: room for the padding of two largest ones
    g->arena_bytes = ((slot_budget_bytes + 255) & ~255ll) + 1024;
    int64_t all = 0;   // no larger than every partition at once
    for (int q = 0; q < g->npart; ++q) all += (((4 * std::max<int64_t>(g->pbeg[q + 1] - g->pbeg[q], 1) + 255) & ~255ll)) *
                                               (weights ? 2 : 1);
    if (g->arena_bytes > all) g->arena_bytes = all;
    if (cudaMalloc((void **)&g->arena, (size_t)g->arena_bytes) != cudaSuccess)
        return bail("partition arena allocation failed", CSAW_ERR_NOMEM);
    g->free_regions[0] = g->arena_bytes;
    g->res_off.assign((size_t)g->npart, -1);
    g->res_bytes.assign((size_t)g->npart, 0);
    g->res_w.assign((size_t)g->npart, 0);
    g->ready.assign((size_t)g->npart, nullptr);
    g->freed.assign((size_t)g->npart, nullptr);
    if (cudaStreamCreateWithFlags(&g->copy, cudaStreamNonBlocking) != cudaSuccess)
        return bail("copy stream creation failed", CSAW_ERR_CUDA);
    if (cudaMallocHost((void **)&g->hctr, sizeof(StreamCounters)) != cudaSuccess)
        return bail("pinned counters failed", CSAW_ERR_NOMEM);
    *out = g;
    return 0;
}

extern "C" int csaw_stream_graph_destroy(csaw_stream_graph g) {
    if (!g) return 0;
    cudaSetDevice(g->device);
    if (g->copy) cudaStreamSynchronize(g->copy);
    cudaDeviceSynchronize();
    cudaFree(g->d_rowptr);
    cudaFree(g->arena);
    for (auto &qq : g->q)
        for (auto &b : qq) cudaFree(b.p);
    for (Buf *b : {&g->counts, &g->offsets, &g->cursor, &g->heavy, &g->hscratch, &g->ctr, &g->skip, &g->ptab})
        cudaFree(b->p);
    for (auto e : g->ready)
        if (e) cudaEventDestroy(e);
    for (auto e : g->freed)
        if (e) cudaEventDestroy(e);
    if (g->copy) cudaStreamDestroy(g->copy);
    if (g->hctr) cudaFreeHost(g->hctr);
    if (g->reg_col) cudaHostUnregister((void *)g->h_col);
    if (g->reg_w) cudaHostUnregister((void *)g->h_w);
    for (int b = 0; b < 4; ++b) {
        if (g->h_cdf[b]) cudaFreeHost(g->h_cdf[b]);
        if (g->d_idx[b]) cudaFree(g->d_idx[b]);
    }
    cudaGetLastError();
    delete g;
    return 0;
}

namespace {

// Builds the prefix cache of bias kind BIAS: partition by partition, the
// columns (and weights) go to device staging, every row's canonical prefix is
// computed there (a warp per row, any degree: the same bits as the in-memory
// cache, which builds large rows a CTA each), the index entries of the
// partition's edges are written into the resident index levels, and the
// prefix is copied to page-locked host memory.
template <typename I, int BIAS>
int build_stream_cdf(csaw_stream_graph_s *g) {
    if (g->h_cdf[BIAS]) return 0;
    const bool reads_w = BIAS == CSAW_BIAS_EDGE_WEIGHT || BIAS == CSAW_BIAS_HOOK;
    if (reads_w && !(g->h_w && g->reg_w))
        return csaw_host_fail(CSAW_ERR_INVALID,
                              "the prefix cache of this bias needs page-locked weights (rebuilds read them)");
    const int64_t E = g->E, n1 = (E + 31) >> 5, n2 = (E + 1023) >> 10, maxp = std::max<int64_t>(g->max_pedges, 1);
    float *h = nullptr, *idx = nullptr, *stage_w = nullptr, *stage_cdf = nullptr;
    int32_t *stage_col = nullptr;
    auto cleanup = [&]() {
        cudaFree(stage_col);
        cudaFree(stage_w);
        cudaFree(stage_cdf);
        cudaGetLastError();
    };
    if (cudaHostAlloc((void **)&h, sizeof(float) * (size_t)std::max<int64_t>(E, 1), cudaHostAllocDefault) != cudaSuccess) {
        cudaGetLastError();
        return csaw_host_fail(CSAW_ERR_NOMEM, "page-locked prefix cache allocation failed");
    }
    if (cudaMalloc((void **)&idx, sizeof(float) * (size_t)(n1 + n2)) != cudaSuccess ||
        cudaMalloc((void **)&stage_col, sizeof(int32_t) * (size_t)maxp) != cudaSuccess ||
        (reads_w && cudaMalloc((void **)&stage_w, sizeof(float) * (size_t)maxp) != cudaSuccess) ||
        cudaMalloc((void **)&stage_cdf, sizeof(float) * (size_t)maxp) != cudaSuccess) {
        cudaGetLastError();
        cleanup();
        cudaFree(idx);
        cudaFreeHost(h);
        return csaw_host_fail(CSAW_ERR_NOMEM, "prefix cache staging allocation failed");
    }
    cudaStream_t st = g->copy;
    int rc = 0;
    auto ck = [&](cudaError_t e, const char *what) {
        if (e != cudaSuccess && !rc) {
            cudaGetLastError();
            rc = csaw_host_fail(CSAW_ERR_CUDA, (std::string(what) + ": " + cudaGetErrorString(e)).c_str());
        }
    };
    ck(cudaMemsetAsync(idx, 0, sizeof(float) * (size_t)(n1 + n2), st), "index clear");
    for (int q = 0; q < g->npart && !rc; ++q) {
        const int64_t e0 = g->pbeg[q], e1 = g->pbeg[q + 1], ne = e1 - e0;
        if (ne == 0) continue;
        ck(cudaMemcpyAsync(stage_col, g->h_col + e0, sizeof(int32_t) * ne, cudaMemcpyHostToDevice, st), "columns");
        if (reads_w) ck(cudaMemcpyAsync(stage_w, g->h_w + e0, sizeof(float) * ne, cudaMemcpyHostToDevice, st), "weights");
        DevGraph dg{};
        dg.v.rowptr = g->d_rowptr;
        dg.v.rowptr_is_64 = g->idx64;
        dg.v.n_vertices = g->V;
        dg.v.n_edges = g->E;
        dg.v.col = stage_col - e0;   // re-based: col[e] is edge e of this partition
        dg.v.weight = reads_w ? stage_w - e0 : nullptr;
        dg.cdf_bias = -1;
        const int64_t v0 = (int64_t)q << g->pbits, v1 = std::min<int64_t>(g->V, (int64_t)(q + 1) << g->pbits);
        k_cdf_build<I, BIAS><<<g->sm_count * 8, 256, 0, st>>>(dg, stage_cdf - e0, INT64_MAX, v0, v1);
        k_cdf_index_range<<<g->sm_count * 2, 256, 0, st>>>(stage_cdf - e0, e0, e1, idx, idx + n1);
        g->launches += 2;
        ck(cudaGetLastError(), "prefix build launch");
        ck(cudaMemcpyAsync(h + e0, stage_cdf, sizeof(float) * ne, cudaMemcpyDeviceToHost, st), "prefix copy");
        ck(cudaStreamSynchronize(st), "prefix build");   // the staging buffers are reused
    }
    cleanup();
    if (rc) {
        cudaFree(idx);
        cudaFreeHost(h);
        return rc;
    }
    g->h_cdf[BIAS] = h;
    g->d_idx[BIAS] = idx;
    void *dp = nullptr;
    if (cudaHostGetDevicePointer(&dp, h, 0) == cudaSuccess) g->dv_cdf[BIAS] = (const float *)dp;
    cudaGetLastError();
    return 0;
}

}  // namespace

extern "C" int csaw_stream_graph_cache(csaw_stream_graph g, int bias) {
    if (!g) return csaw_host_fail(CSAW_ERR_INVALID, "graph is NULL");
    if (bias < CSAW_BIAS_DEGREE || bias > CSAW_BIAS_HOOK) return csaw_host_fail(CSAW_ERR_INVALID, "bias must be biased");
    if (bias == CSAW_BIAS_EDGE_WEIGHT && !g->h_w) return csaw_host_fail(CSAW_ERR_INVALID, "graph has no weights");
    if (cudaSetDevice(g->device) != cudaSuccess) return csaw_host_fail(CSAW_ERR_CUDA, "cudaSetDevice failed");
    if (cudaStreamSynchronize(g->copy) != cudaSuccess) {
        cudaGetLastError();
        return csaw_host_fail(CSAW_ERR_CUDA, "copy stream failed");
    }
#define CSAW_STREAM_CACHE(I)                                                  \
    switch (bias) {                                                           \
        case CSAW_BIAS_DEGREE: return build_stream_cdf<I, CSAW_BIAS_DEGREE>(g); \
        case CSAW_BIAS_EDGE_WEIGHT: return build_stream_cdf<I, CSAW_BIAS_EDGE_WEIGHT>(g); \
        default: return build_stream_cdf<I, CSAW_BIAS_HOOK>(g);               \
    }
    if (g->idx64) {
        CSAW_STREAM_CACHE(int64_t)
    }
    CSAW_STREAM_CACHE(int32_t)
#undef CSAW_STREAM_CACHE
}

extern "C" int csaw_stream_sample(csaw_stream_graph g, const csaw_params *p, const int32_t *seeds, int32_t *out_src,
                                  int32_t *out_dst, int32_t *out_sample, int32_t *out_depth, int64_t capacity,
                                  int64_t *n_out, void *stream) {
    int fan[CSAW_MAX_DEPTH];
    if (!g || !n_out) return csaw_host_fail(CSAW_ERR_INVALID, "NULL argument");
    *n_out = 0;
    STRY(check_stream_params(p, fan));
    if (p->bias == CSAW_BIAS_EDGE_WEIGHT && !g->h_w)
        return csaw_host_fail(CSAW_ERR_INVALID, "edge-weight bias needs a graph with weights");
    if (capacity < 0 || (capacity > 0 && (!out_src || !out_dst)))
        return csaw_host_fail(CSAW_ERR_INVALID, "bad output buffers");
    if (p->n_samples > 0 && !seeds) return csaw_host_fail(CSAW_ERR_INVALID, "seeds is NULL");
    if (p->n_samples == 0 || p->depth == 0) return 0;
    SCK(cudaSetDevice(g->device));
    cudaStream_t st = (cudaStream_t)stream;
    int rc;
#define CSAW_STREAM_RUN(I)                                                                                  \
    switch (p->bias) {                                                                                      \
        case CSAW_BIAS_UNBIASED: rc = run_stream<I, CSAW_BIAS_UNBIASED>(g, p, fan, seeds, out_src, out_dst, out_sample, out_depth, capacity, st); break; \
        case CSAW_BIAS_DEGREE: rc = run_stream<I, CSAW_BIAS_DEGREE>(g, p, fan, seeds, out_src, out_dst, out_sample, out_depth, capacity, st); break; \
        case CSAW_BIAS_EDGE_WEIGHT: rc = run_stream<I, CSAW_BIAS_EDGE_WEIGHT>(g, p, fan, seeds, out_src, out_dst, out_sample, out_depth, capacity, st); break; \
        default: rc = run_stream<I, CSAW_BIAS_HOOK>(g, p, fan, seeds, out_src, out_dst, out_sample, out_depth, capacity, st); break; \
    }
    if (g->idx64) {
        CSAW_STREAM_RUN(int64_t)
    } else {
        CSAW_STREAM_RUN(int32_t)
    }
#undef CSAW_STREAM_RUN
    if (rc) {
        cudaStreamSynchronize(st);
        return rc;
    }
    const StreamCounters &k = *g->hctr;
    *n_out = (int64_t)k.out_count;
    if (k.err & ERR_SEED_RANGE) return csaw_host_fail(CSAW_ERR_INVALID, "a seed vertex is out of range");
    if (k.err) return csaw_host_fail(CSAW_ERR_DEVICE, "kernel error flag set");
    if ((int64_t)k.out_count > capacity) return csaw_host_fail(CSAW_ERR_CAPACITY, "output capacity too small");
    return 0;
}

extern "C" int csaw_stream_stats(csaw_stream_graph g, csaw_stream_info *out) {
    if (!g || !out) return csaw_host_fail(CSAW_ERR_INVALID, "NULL argument");
    out->n_partitions = g->npart;
    out->n_slots = g->nslots;
    out->partition_loads = g->loads;
    out->partition_hits = g->hits;
    out->bytes_h2d = g->bytes_h2d;
    out->kernel_launches = g->launches;
    out->host_pinned_in_place = (g->reg_col ? 1 : 0) | (g->reg_w ? 2 : 0);
    out->items_read_in_place = g->host_items;
    return 0;
}

extern "C" int csaw_stream_graph_set_option(csaw_stream_graph g, int option, int64_t value) {
    if (!g) return csaw_host_fail(CSAW_ERR_INVALID, "stream graph is NULL");
    switch (option) {
        case CSAW_STREAM_OPT_READ_IN_PLACE:
            g->read_in_place = value != 0;
            return 0;
        default:
            return csaw_host_fail(CSAW_ERR_INVALID, "unknown stream graph option");
    }
}
