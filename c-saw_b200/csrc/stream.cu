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
//   - a fixed number of device slots (from the byte budget) hold partitions;
//     a level's partition order is known, so the victim is the slot whose
//     partition is needed farthest ahead (or never);
//   - copies run on a copy stream, each slot has a ready event (copy done)
//     and a free event (last kernel using it done); the next partition's copy
//     is issued before the current partition's kernels, so transfer overlaps
//     sampling;
//   - frontier items are binned by partition each level (histogram, scan,
//     scatter); the level-expansion kernel runs once per resident partition
//     on that partition's items with the column/weight pointers re-based onto
//     the slot, so col[e] of any edge of the partition is read from HBM;
//   - walks are neighbor sampling with N = 1 (same keys, same output).
// Because every draw is keyed by (sample, depth, lineage, slot, draw), the
// output equals the in-memory output exactly, whatever the partition order.
#include <cuda_runtime.h>

#include <algorithm>
#include <string>
#include <vector>

#include "csaw.h"
#include "csaw_host.h"
#include "csaw_internal.h"
#include "kernels_sample.cuh"

using namespace csaw;

namespace {

struct StreamCounters {
    unsigned long long out_count;
    unsigned long long bytes[8];
    unsigned long long items[8];
    uint32_t n_next;      // unsorted next-level items
    uint32_t n_heavy;
    int err;
    uint32_t pad;
};

__global__ void k_part_hist(const int32_t *v, const uint32_t *n, int pbits, uint32_t *counts) {
    const uint32_t m = *n;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x)
        atomicAdd(&counts[v[i] >> pbits], 1u);
}

// Exclusive scan of npart counts into offsets[0..npart] and a cursor copy
// (one block; npart is at most a few thousand).
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

__global__ void k_part_scatter(const int32_t *v, const int32_t *s, const uint32_t *p, const uint32_t *n, int pbits,
                               uint32_t *cursor, int32_t *ov, int32_t *os, uint32_t *op) {
    const uint32_t m = *n;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
        const uint32_t pos = atomicAdd(&cursor[v[i] >> pbits], 1u);
        ov[pos] = v[i];
        os[pos] = s[i];
        op[pos] = p[i];
    }
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
    int nslots = 0;
    int32_t *slot_col = nullptr;
    float *slot_w = nullptr;          // null when the graph has no weights
    std::vector<int> slot_part;
    std::vector<char> slot_has_w;     // the slot holds its partition's weights too
    std::vector<cudaEvent_t> slot_ready, slot_free;
    cudaStream_t copy = nullptr;
    Buf q[3][3], counts, offsets, cursor, heavy, hscratch, ctr;
    StreamCounters *hctr = nullptr;
    int64_t loads = 0, hits = 0, bytes_h2d = 0, launches = 0;
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

// Makes partition `part` resident and returns its slot.  On a miss the victim
// is the slot whose partition is needed farthest ahead in `order` (from
// position `from`), or never; `keep` is never evicted.  The copy waits for the
// victim's last kernel; for a use (not a prefetch) the compute stream -- which
// may be the legacy default stream, handle 0 -- waits for the copy.
int make_resident(csaw_stream_graph_s *g, int part, bool need_w, const std::vector<int> &order, size_t from,
                  int keep, bool use, cudaStream_t compute, int *slot_out) {
    for (int s = 0; s < g->nslots; ++s)
        if (g->slot_part[s] == part) {
            if (need_w && g->slot_w && !g->slot_has_w[s]) {   // resident without its weights: add them
                const int64_t e0 = g->pbeg[part], ne = g->pbeg[part + 1] - e0;
                SCK(cudaStreamWaitEvent(g->copy, g->slot_free[s], 0));
                if (ne > 0) {
                    SCK(cudaMemcpyAsync(g->slot_w + (size_t)s * g->max_pedges, g->h_w + e0, sizeof(float) * ne,
                                        cudaMemcpyHostToDevice, g->copy));
                    g->bytes_h2d += 4 * ne;
                }
                SCK(cudaEventRecord(g->slot_ready[s], g->copy));
                g->slot_has_w[s] = 1;
            }
            if (use) {   // a use (not a prefetch): wait for the copy
                g->hits++;
                SCK(cudaStreamWaitEvent(compute, g->slot_ready[s], 0));
            }
            *slot_out = s;
            return 0;
        }
    // victim: an empty slot, else the partition needed farthest ahead (or never)
    int victim = -1;
    size_t far = 0;
    for (int s = 0; s < g->nslots; ++s) {
        if (s == keep) continue;
        size_t nu = SIZE_MAX;
        if (g->slot_part[s] >= 0) {
            nu = SIZE_MAX - 1;
            for (size_t k = from; k < order.size(); ++k)
                if (order[k] == g->slot_part[s]) {
                    nu = k;
                    break;
                }
        }
        if (victim < 0 || nu > far) {
            victim = s;
            far = nu;
        }
    }
    if (victim < 0) return csaw_host_fail(CSAW_ERR_INVALID, "no free partition slot");
    const int64_t e0 = g->pbeg[part], ne = g->pbeg[part + 1] - e0;
    SCK(cudaStreamWaitEvent(g->copy, g->slot_free[victim], 0));
    if (ne > 0) {
        SCK(cudaMemcpyAsync(g->slot_col + (size_t)victim * g->max_pedges, g->h_col + e0, sizeof(int32_t) * ne,
                            cudaMemcpyHostToDevice, g->copy));
        g->bytes_h2d += 4 * ne;
        if (need_w && g->slot_w) {
            SCK(cudaMemcpyAsync(g->slot_w + (size_t)victim * g->max_pedges, g->h_w + e0, sizeof(float) * ne,
                                cudaMemcpyHostToDevice, g->copy));
            g->bytes_h2d += 4 * ne;
        }
    }
    SCK(cudaEventRecord(g->slot_ready[victim], g->copy));
    g->slot_part[victim] = part;
    g->slot_has_w[victim] = need_w && g->slot_w ? 1 : 0;
    g->loads++;
    if (use) SCK(cudaStreamWaitEvent(compute, g->slot_ready[victim], 0));
    *slot_out = victim;
    return 0;
}

#define STRY(x)              \
    do {                     \
        int rc_ = (x);       \
        if (rc_) return rc_; \
    } while (0)

template <typename I, int BIAS>
int run_stream(csaw_stream_graph_s *g, const csaw_params *p, const int fan[], const int32_t *seeds, int32_t *src,
               int32_t *dst, int32_t *smp, int32_t *dep, int64_t cap, cudaStream_t st) {
    constexpr bool BIASED = BIAS != CSAW_BIAS_UNBIASED;
    const bool need_w = (BIAS == CSAW_BIAS_EDGE_WEIGHT || BIAS == CSAW_BIAS_HOOK) && g->h_w;
    const int S = p->n_samples, F = p->mode == CSAW_MODE_WALK ? 1 : p->frontier_size, D = p->depth;
    double per = F, lvl = F;
    for (int l = 0; l + 1 < D; ++l) {
        lvl *= fan[l];
        per = std::max(per, lvl);
    }
    if (per > 4294967295.0) return csaw_host_fail(CSAW_ERR_INVALID, "lineage items exceed 2^32");
    if (per * S > 2.0e9) return csaw_host_fail(CSAW_ERR_INVALID, "a frontier level exceeds 2e9 items");
    const int64_t qcap = (int64_t)(per * S) + 32;
    for (auto &qq : g->q)
        for (auto &b : qq) STRY(grow(b, sizeof(int32_t) * (size_t)qcap));
    STRY(grow(g->counts, sizeof(uint32_t) * (size_t)g->npart));
    STRY(grow(g->cursor, sizeof(uint32_t) * (size_t)g->npart));
    STRY(grow(g->offsets, sizeof(uint32_t) * (size_t)(g->npart + 1)));
    STRY(grow(g->ctr, sizeof(StreamCounters)));
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
    SCK(cudaMemsetAsync(c, 0, sizeof(StreamCounters), st));
    auto qv = [&](int k, int a) { return (int32_t *)g->q[k][a].p; };
    const int U = 2;           // unsorted next-level items
    int A = 0, B = 1;          // sorted current / next
    const int bgrid = g->sm_count * 4;
    auto bin = [&](int into) -> int {
        SCK(cudaMemsetAsync(d_counts, 0, sizeof(uint32_t) * g->npart, st));
        k_part_hist<<<bgrid, 256, 0, st>>>(qv(U, 0), &c->n_next, g->pbits, d_counts);
        k_part_scan<<<1, 1024, 0, st>>>(d_counts, g->npart, (uint32_t *)g->offsets.p, (uint32_t *)g->cursor.p);
        k_part_scatter<<<bgrid, 256, 0, st>>>(qv(U, 0), qv(U, 1), (const uint32_t *)qv(U, 2), &c->n_next, g->pbits,
                                              (uint32_t *)g->cursor.p, qv(into, 0), qv(into, 1),
                                              (uint32_t *)qv(into, 2));
        g->launches += 3;
        return 0;
    };
    const uint32_t n0 = (uint32_t)((int64_t)S * F);
    k_init_queue<<<(n0 + 255) / 256, 256, 0, st>>>(seeds, n0, F, (int)p->sample_base, g->V, qv(U, 0), qv(U, 1),
                                                   (uint32_t *)qv(U, 2), &c->n_next, &c->err);
    g->launches++;
    STRY(bin(A));
    int grid = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&grid, k_expand_warp<I, BIAS>, EXPAND_THREADS, 0);
    grid = (grid > 0 ? grid : 1) * g->sm_count;
    std::vector<uint32_t> h_counts((size_t)g->npart);
    std::vector<int64_t> h_off((size_t)g->npart + 1);
    for (int l = 0; l < D; ++l) {
        SCK(cudaMemcpyAsync(h_counts.data(), d_counts, sizeof(uint32_t) * g->npart, cudaMemcpyDeviceToHost, st));
        SCK(cudaStreamSynchronize(st));
        h_off[0] = 0;
        for (int q = 0; q < g->npart; ++q) h_off[q + 1] = h_off[q] + h_counts[q];
        // resident partitions first, then the others in id order
        std::vector<int> order;
        for (int s2 = 0; s2 < g->nslots; ++s2)
            if (g->slot_part[s2] >= 0 && h_counts[g->slot_part[s2]] > 0) order.push_back(g->slot_part[s2]);
        for (int q = 0; q < g->npart; ++q)
            if (h_counts[q] > 0 && std::find(order.begin(), order.end(), q) == order.end()) order.push_back(q);
        SCK(cudaMemsetAsync(&c->n_next, 0, sizeof(uint32_t), st));
        for (size_t k = 0; k < order.size(); ++k) {
            const int part = order[k];
            int slot = -1;
            STRY(make_resident(g, part, need_w, order, k, -1, true, st, &slot));
            if (k + 1 < order.size() && g->nslots >= 2) {   // prefetch the next partition
                int pslot = -1;
                STRY(make_resident(g, order[k + 1], need_w, order, k + 1, slot, false, nullptr, &pslot));
            }
            DevGraph dg{};
            dg.v.rowptr = g->d_rowptr;
            dg.v.rowptr_is_64 = g->idx64;
            dg.v.col = g->slot_col + (size_t)slot * g->max_pedges - g->pbeg[part];
            dg.v.weight = g->slot_w ? g->slot_w + (size_t)slot * g->max_pedges - g->pbeg[part] : nullptr;
            dg.v.n_vertices = g->V;
            dg.v.n_edges = g->E;
            LevelArgs a{};
            a.in_v = qv(A, 0) + h_off[part];
            a.in_s = qv(A, 1) + h_off[part];
            a.in_p = (const uint32_t *)qv(A, 2) + h_off[part];
            a.n_in = d_counts + part;
            a.out_v = qv(U, 0);
            a.out_s = qv(U, 1);
            a.out_p = (uint32_t *)qv(U, 2);
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
            a.depth = l;
            a.N = fan[l];
            a.push = l + 1 < D;
            if (hblocks) SCK(cudaMemsetAsync(&c->n_heavy, 0, sizeof(uint32_t), st));
            k_expand_warp<I, BIAS><<<grid, EXPAND_THREADS, 0, st>>>(dg, a);
            g->launches++;
            if (hblocks) {
                k_expand_heavy<I, BIAS><<<hblocks, HEAVY_THREADS, 0, st>>>(dg, a);
                g->launches++;
            }
            SCK(cudaEventRecord(g->slot_free[slot], st));
        }
        if (l + 1 < D) {
            STRY(bin(B));
            std::swap(A, B);
        }
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
    }
    const int64_t per_slot = std::max<int64_t>(g->max_pedges, 1) * (weights ? 8 : 4);
    int64_t ns = slot_budget_bytes / per_slot;
    if (ns > g->npart) ns = g->npart;
    if (ns < std::min(2, g->npart)) return bail("slot budget holds fewer than 2 partitions", CSAW_ERR_INVALID);
    g->nslots = (int)ns;
    if (cudaMalloc((void **)&g->slot_col, sizeof(int32_t) * (size_t)std::max<int64_t>(g->max_pedges, 1) * ns) != cudaSuccess)
        return bail("slot allocation failed", CSAW_ERR_NOMEM);
    if (weights &&
        cudaMalloc((void **)&g->slot_w, sizeof(float) * (size_t)std::max<int64_t>(g->max_pedges, 1) * ns) != cudaSuccess)
        return bail("slot allocation failed", CSAW_ERR_NOMEM);
    g->slot_part.assign((size_t)ns, -1);
    g->slot_has_w.assign((size_t)ns, 0);
    g->slot_ready.resize((size_t)ns);
    g->slot_free.resize((size_t)ns);
    for (int64_t k = 0; k < ns; ++k) {
        cudaEventCreateWithFlags(&g->slot_ready[k], cudaEventDisableTiming);
        cudaEventCreateWithFlags(&g->slot_free[k], cudaEventDisableTiming);
    }
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
    cudaFree(g->slot_col);
    cudaFree(g->slot_w);
    for (auto &qq : g->q)
        for (auto &b : qq) cudaFree(b.p);
    for (Buf *b : {&g->counts, &g->offsets, &g->cursor, &g->heavy, &g->hscratch, &g->ctr}) cudaFree(b->p);
    for (auto e : g->slot_ready) cudaEventDestroy(e);
    for (auto e : g->slot_free) cudaEventDestroy(e);
    if (g->copy) cudaStreamDestroy(g->copy);
    if (g->hctr) cudaFreeHost(g->hctr);
    if (g->reg_col) cudaHostUnregister((void *)g->h_col);
    if (g->reg_w) cudaHostUnregister((void *)g->h_w);
    cudaGetLastError();
    delete g;
    return 0;
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
    return 0;
}
