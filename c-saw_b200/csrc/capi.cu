// capi.cu -- host driver and C ABI of the csaw-b200 sampler.
//
// Replaces C-SAW's host driver Sampler() (non-stream/main.cu:196-308), its
// gpu_graph residency (gpu_graph.cuh:25-66) and its Sampling/Wv/Cd/Si device
// state classes (sample_class.cuh:10-185) with: a graph handle that owns the
// resident CSR, a grow-only workspace (frontier queues, high-degree scratch),
// one small counter block, and level-by-level kernel launches on the caller's
// stream.  Errors are returned as status codes with a per-thread message.
#include <cuda_runtime.h>

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "csaw.h"
#include "csaw_internal.h"
#include "kernels_sample.cuh"

using namespace csaw;

namespace {

thread_local std::string g_err = "no error";

int fail(int code, const std::string &msg) {
    g_err = msg;
    return code;
}

#define CK(x)                                                                              \
    do {                                                                                   \
        cudaError_t e_ = (x);                                                              \
        if (e_ != cudaSuccess) {                                                           \
            cudaGetLastError();                                                            \
            return fail(e_ == cudaErrorMemoryAllocation ? CSAW_ERR_NOMEM : CSAW_ERR_CUDA,  \
                        std::string(#x) + ": " + cudaGetErrorString(e_));                  \
        }                                                                                  \
    } while (0)

#define TRY(x)                 \
    do {                       \
        int rc_ = (x);         \
        if (rc_) return rc_;   \
    } while (0)

enum { KK_EXPAND = 0, KK_HEAVY = 1, KK_WALK = 2, KK_MDRW = 3, KK_INIT = 4, KK_COUNT = 8 };

struct Counters {
    unsigned long long out_count;
    unsigned long long bytes[KK_COUNT];
    unsigned long long items[KK_COUNT];
    uint32_t nq[2];
    uint32_t n_heavy;
    int err;
};

struct DevBuf {
    void *p = nullptr;
    size_t n = 0;
};

int ensure(DevBuf &b, size_t bytes) {
    if (b.n >= bytes) return 0;
    if (b.p) cudaFree(b.p);
    b.p = nullptr;
    b.n = 0;
    if (bytes == 0) return 0;
    cudaError_t e = cudaMalloc(&b.p, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        b.p = nullptr;
        return fail(CSAW_ERR_NOMEM, "workspace allocation of " + std::to_string(bytes) +
                                        " bytes failed: " + cudaGetErrorString(e));
    }
    b.n = bytes;
    return 0;
}

constexpr int64_t QUEUE_ITEM_BUDGET = 32ll << 20;   // items per ping-pong queue
constexpr int64_t SCRATCH_BUDGET = 1ll << 30;        // bytes of high-degree scratch
constexpr int MDRW_MAX_F = 4096;

}  // namespace

struct csaw_graph_s {
    int device = 0, sm_count = 148;
    int64_t V = 0, E = 0, maxdeg = 0, n_non = 0;
    int idx64 = 0;
    void *rowptr = nullptr;
    int32_t *col = nullptr;
    float *weight = nullptr;
    float *ebias = nullptr;
    float *cdf = nullptr;
    int cdf_bias = -1;
    int32_t *nonisolated = nullptr;
    int64_t dev_bytes = 0;
    DevBuf q[2][3], heavy, hscratch, wscratch, seeds_in, out_dev;
    Counters *ctr = nullptr, *hctr = nullptr;
    int64_t launches = 0;
    csaw_stats last{};
    bool prof = false;
    double kms[KK_COUNT] = {};
    int64_t klaunch[KK_COUNT] = {};
    unsigned long long kbytes[KK_COUNT] = {}, kitems[KK_COUNT] = {};
    std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> pending;
    std::vector<cudaEvent_t> event_pool;
};

namespace {

DevGraph dev_view(const csaw_graph_s *g) {
    DevGraph d;
    d.v.rowptr = g->rowptr;
    d.v.rowptr_is_64 = g->idx64;
    d.v.col = g->col;
    d.v.weight = g->weight;
    d.v.n_vertices = g->V;
    d.v.n_edges = g->E;
    d.ebias = g->ebias;
    d.cdf = g->cdf;
    d.cdf_bias = g->cdf_bias;
    return d;
}

cudaEvent_t take_event(csaw_graph_s *g) {
    if (!g->event_pool.empty()) {
        cudaEvent_t e = g->event_pool.back();
        g->event_pool.pop_back();
        return e;
    }
    cudaEvent_t e;
    cudaEventCreate(&e);
    return e;
}

// Wraps one launch: counts it, and with profiling on brackets it with events.
struct LaunchScope {
    csaw_graph_s *g;
    int kind;
    cudaStream_t st;
    cudaEvent_t a = nullptr, b = nullptr;
    LaunchScope(csaw_graph_s *g_, int kind_, cudaStream_t st_) : g(g_), kind(kind_), st(st_) {
        g->launches++;
        if (g->prof) {
            a = take_event(g);
            b = take_event(g);
            cudaEventRecord(a, st);
        }
    }
    ~LaunchScope() {
        if (g->prof) {
            cudaEventRecord(b, st);
            g->pending.push_back({kind, {a, b}});
        }
    }
};

void drain_profile(csaw_graph_s *g) {
    for (auto &pe : g->pending) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, pe.second.first, pe.second.second);
        g->kms[pe.first] += ms;
        g->klaunch[pe.first] += 1;
        g->event_pool.push_back(pe.second.first);
        g->event_pool.push_back(pe.second.second);
    }
    g->pending.clear();
}

template <typename K>
int grid_for(K kernel, int threads, size_t dyn_smem, int sm_count) {
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, dyn_smem);
    if (per_sm < 1) per_sm = 1;
    return per_sm * sm_count;
}

int check_params(const csaw_graph_s *g, const csaw_params *p, int fan[CSAW_MAX_DEPTH]) {
    if (!p) return fail(CSAW_ERR_INVALID, "params is NULL");
    if (p->mode < CSAW_MODE_NEIGHBOR || p->mode > CSAW_MODE_MDRW)
        return fail(CSAW_ERR_INVALID, "unknown mode");
    if (p->bias < CSAW_BIAS_UNBIASED || p->bias > CSAW_BIAS_HOOK)
        return fail(CSAW_ERR_INVALID, "unknown bias");
    if (p->n_samples < 0) return fail(CSAW_ERR_INVALID, "n_samples < 0");
    if (p->depth < 0 || p->depth > (p->mode == CSAW_MODE_NEIGHBOR ? CSAW_MAX_DEPTH : (1 << 24) - 1))
        return fail(CSAW_ERR_INVALID, "depth out of range");
    if (p->frontier_size < 1) return fail(CSAW_ERR_INVALID, "frontier_size < 1");
    if (p->bias == CSAW_BIAS_EDGE_WEIGHT && !g->weight)
        return fail(CSAW_ERR_INVALID, "edge-weight bias needs a graph with weights");
    if (p->mode == CSAW_MODE_MDRW && p->bias == CSAW_BIAS_EDGE_WEIGHT)
        return fail(CSAW_ERR_INVALID, "MDRW picks frontier vertices: use a vertex bias");
    if (p->mode == CSAW_MODE_MDRW && p->frontier_size > MDRW_MAX_F)
        return fail(CSAW_ERR_INVALID, "MDRW frontier_size above 4096");
    if (p->mode == CSAW_MODE_NEIGHBOR) {
        for (int l = 0; l < p->depth; ++l) {
            fan[l] = p->fanout[l] ? p->fanout[l] : p->neighbor_size;
            if (fan[l] < 1 || fan[l] > MAX_FANOUT)
                return fail(CSAW_ERR_INVALID, "NeighborSize must be in [1, 32] for every hop");
        }
    }
    return 0;
}

template <typename I, int BIAS>
int run_neighbor_t(csaw_graph_s *g, const csaw_params *p, const int fan[], const int32_t *seeds,
                   const OutArgs &o, cudaStream_t st) {
    constexpr bool BIASED = BIAS != CSAW_BIAS_UNBIASED;
    const int S = p->n_samples, F = p->frontier_size, D = p->depth;
    // largest level of one sample's tree, and the lineage bound
    double per_sample = F, lvl = F;
    for (int l = 0; l + 1 < D; ++l) {
        lvl *= fan[l];
        if (lvl > per_sample) per_sample = lvl;
    }
    if (per_sample > 4294967295.0)
        return fail(CSAW_ERR_INVALID, "FrontierSize * prod(NeighborSize) exceeds 2^32 lineage items");
    if (per_sample > (double)QUEUE_ITEM_BUDGET)
        return fail(CSAW_ERR_INVALID, "one sample's frontier exceeds the queue budget");
    int64_t B = (int64_t)((double)QUEUE_ITEM_BUDGET / per_sample);
    if (B > S) B = S;
    if (B < 1) B = 1;
    const int64_t qcap = (int64_t)(B * per_sample) + 32;
    for (int k = 0; k < 2; ++k)
        for (int a = 0; a < 3; ++a) TRY(ensure(g->q[k][a], sizeof(int32_t) * qcap));
    int hblocks = 0;
    int64_t hstride = 0;
    if (BIASED && g->maxdeg > WBUF && !(g->cdf && g->cdf_bias == BIAS)) {
        TRY(ensure(g->heavy, sizeof(uint32_t) * qcap));
        hstride = g->maxdeg + 2 * ((g->maxdeg >> 5) + 1) + (g->maxdeg >> 10) + 1 + 8;
        hstride = (hstride + 63) & ~63ll;
        hblocks = g->sm_count * 2;
        while (hblocks > 1 && (int64_t)hblocks * hstride * 4 > SCRATCH_BUDGET) hblocks /= 2;
        TRY(ensure(g->hscratch, sizeof(float) * hstride * hblocks));
    }
    const DevGraph dg = dev_view(g);
    const uint64_t seed = p->seed;
    const int grid = grid_for(k_expand_warp<I, BIAS>, EXPAND_THREADS, 0, g->sm_count);
    for (int64_t s0 = 0; s0 < S; s0 += B) {
        const int64_t nb = (S - s0 < B) ? S - s0 : B;
        const uint32_t n0 = (uint32_t)(nb * F);
        {
            LaunchScope ls(g, KK_INIT, st);
            k_init_queue<<<(n0 + 255) / 256, 256, 0, st>>>(
                seeds + s0 * F, n0, F, (int)s0, g->V, (int32_t *)g->q[0][0].p, (int32_t *)g->q[0][1].p,
                (uint32_t *)g->q[0][2].p, &g->ctr->nq[0], &g->ctr->err);
        }
        for (int l = 0; l < D; ++l) {
            const int cur = l & 1, nxt = cur ^ 1;
            CK(cudaMemsetAsync(&g->ctr->nq[nxt], 0, sizeof(uint32_t), st));
            CK(cudaMemsetAsync(&g->ctr->n_heavy, 0, sizeof(uint32_t), st));
            LevelArgs a;
            a.in_v = (const int32_t *)g->q[cur][0].p;
            a.in_s = (const int32_t *)g->q[cur][1].p;
            a.in_p = (const uint32_t *)g->q[cur][2].p;
            a.n_in = &g->ctr->nq[cur];
            a.out_v = (int32_t *)g->q[nxt][0].p;
            a.out_s = (int32_t *)g->q[nxt][1].p;
            a.out_p = (uint32_t *)g->q[nxt][2].p;
            a.n_out = &g->ctr->nq[nxt];
            a.heavy = (uint32_t *)g->heavy.p;
            a.n_heavy = &g->ctr->n_heavy;
            a.heavy_scratch = (float *)g->hscratch.p;
            a.heavy_stride = hstride;
            a.o_src = o.src;
            a.o_dst = o.dst;
            a.o_smp = o.smp;
            a.o_dep = o.dep;
            a.o_count = o.count;
            a.cap = o.cap;
            a.bytes = g->ctr->bytes;
            a.items = g->ctr->items;
            a.err = &g->ctr->err;
            a.k0 = (uint32_t)seed;
            a.k1 = (uint32_t)(seed >> 32);
            a.depth = l;
            a.N = fan[l];
            a.push = l + 1 < D;
            {
                LaunchScope ls(g, KK_EXPAND, st);
                k_expand_warp<I, BIAS><<<grid, EXPAND_THREADS, 0, st>>>(dg, a);
            }
            if (hblocks) {
                LaunchScope ls(g, KK_HEAVY, st);
                k_expand_heavy<I, BIAS><<<hblocks, HEAVY_THREADS, 0, st>>>(dg, a);
            }
        }
    }
    CK(cudaGetLastError());
    return 0;
}

template <typename I, int BIAS>
int run_walk_t(csaw_graph_s *g, const csaw_params *p, const int32_t *seeds, const OutArgs &o,
               cudaStream_t st) {
    const DevGraph dg = dev_view(g);
    WalkArgs a{};
    a.seeds = seeds;
    a.n = p->n_samples;
    a.len = p->depth;
    a.F = 1;
    a.o_src = o.src;
    a.o_dst = o.dst;
    a.o_smp = o.smp;
    a.o_dep = o.dep;
    a.o_count = o.count;
    a.cap = o.cap;
    a.bytes = g->ctr->bytes;
    a.items = g->ctr->items;
    a.err = &g->ctr->err;
    a.k0 = (uint32_t)p->seed;
    a.k1 = (uint32_t)(p->seed >> 32);
    if (BIAS == CSAW_BIAS_UNBIASED) {
        int grid = (p->n_samples + WALK_THREADS - 1) / WALK_THREADS;
        int gmax = grid_for(k_walk_thread<I>, WALK_THREADS, 0, g->sm_count);
        if (grid > gmax) grid = gmax;
        LaunchScope ls(g, KK_WALK, st);
        k_walk_thread<I><<<grid, WALK_THREADS, 0, st>>>(dg, a);
    } else {
        int gmax = grid_for(k_walk_warp<I, BIAS>, WALK_THREADS, 0, g->sm_count);
        int grid = (p->n_samples + (WALK_THREADS / 32) - 1) / (WALK_THREADS / 32);
        if (grid > gmax) grid = gmax;
        if (g->maxdeg > WBUF && !(g->cdf && g->cdf_bias == BIAS)) {
            int64_t stride = (g->maxdeg + 63) & ~63ll;
            while (grid > 1 && (int64_t)grid * (WALK_THREADS / 32) * stride * 4 > SCRATCH_BUDGET) grid /= 2;
            TRY(ensure(g->wscratch, sizeof(float) * stride * grid * (WALK_THREADS / 32)));
            a.scratch = (float *)g->wscratch.p;
            a.scratch_stride = stride;
        }
        LaunchScope ls(g, KK_WALK, st);
        k_walk_warp<I, BIAS><<<grid, WALK_THREADS, 0, st>>>(dg, a);
    }
    CK(cudaGetLastError());
    return 0;
}

template <typename I, int BIAS>
int run_mdrw_t(csaw_graph_s *g, const csaw_params *p, const int32_t *seeds, const OutArgs &o,
               cudaStream_t st) {
    const DevGraph dg = dev_view(g);
    WalkArgs a{};
    a.seeds = seeds;
    a.n = p->n_samples;
    a.len = p->depth;
    a.F = p->frontier_size;
    a.o_src = o.src;
    a.o_dst = o.dst;
    a.o_smp = o.smp;
    a.o_dep = o.dep;
    a.o_count = o.count;
    a.cap = o.cap;
    a.bytes = g->ctr->bytes;
    a.items = g->ctr->items;
    a.err = &g->ctr->err;
    a.k0 = (uint32_t)p->seed;
    a.k1 = (uint32_t)(p->seed >> 32);
    const size_t per_warp = (size_t)8 * a.F;
    int wpb = (int)(96 * 1024 / per_warp);
    if (wpb > WALK_THREADS / 32) wpb = WALK_THREADS / 32;
    if (wpb < 1) wpb = 1;
    const size_t dyn = per_warp * wpb;
    CK(cudaFuncSetAttribute(k_mdrw<I, BIAS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn));
    int gmax = grid_for(k_mdrw<I, BIAS>, 32 * wpb, dyn, g->sm_count);
    int grid = (p->n_samples + wpb - 1) / wpb;
    if (grid > gmax) grid = gmax;
    LaunchScope ls(g, KK_MDRW, st);
    k_mdrw<I, BIAS><<<grid, 32 * wpb, dyn, st>>>(dg, a);
    CK(cudaGetLastError());
    return 0;
}

template <typename I>
int dispatch_bias(csaw_graph_s *g, const csaw_params *p, const int fan[], const int32_t *seeds,
                  const OutArgs &o, cudaStream_t st) {
#define CSAW_MODES(BIAS)                                                        \
    switch (p->mode) {                                                          \
        case CSAW_MODE_NEIGHBOR: return run_neighbor_t<I, BIAS>(g, p, fan, seeds, o, st); \
        case CSAW_MODE_WALK: return run_walk_t<I, BIAS>(g, p, seeds, o, st);    \
        default: return run_mdrw_t<I, BIAS>(g, p, seeds, o, st);                \
    }
    switch (p->bias) {
        case CSAW_BIAS_UNBIASED: CSAW_MODES(CSAW_BIAS_UNBIASED)
        case CSAW_BIAS_DEGREE: CSAW_MODES(CSAW_BIAS_DEGREE)
        case CSAW_BIAS_EDGE_WEIGHT:
            if (p->mode == CSAW_MODE_MDRW) return fail(CSAW_ERR_INVALID, "MDRW edge-weight bias");
            if (p->mode == CSAW_MODE_NEIGHBOR)
                return run_neighbor_t<I, CSAW_BIAS_EDGE_WEIGHT>(g, p, fan, seeds, o, st);
            return run_walk_t<I, CSAW_BIAS_EDGE_WEIGHT>(g, p, seeds, o, st);
        default: CSAW_MODES(CSAW_BIAS_HOOK)
    }
#undef CSAW_MODES
}

int sample_impl(csaw_graph_s *g, const csaw_params *p, const int32_t *seeds, int32_t *src, int32_t *dst,
                int32_t *smp, int32_t *dep, int64_t cap, int64_t *n_out, cudaStream_t st) {
    int fan[CSAW_MAX_DEPTH];
    if (!g) return fail(CSAW_ERR_INVALID, "graph is NULL");
    if (!n_out) return fail(CSAW_ERR_INVALID, "n_out is NULL");
    TRY(check_params(g, p, fan));
    if (cap < 0) return fail(CSAW_ERR_INVALID, "capacity < 0");
    if (cap > 0 && (!src || !dst)) return fail(CSAW_ERR_INVALID, "out_src/out_dst are NULL");
    if (p->n_samples > 0 && !seeds) return fail(CSAW_ERR_INVALID, "seeds is NULL");
    CK(cudaSetDevice(g->device));
    CK(cudaMemsetAsync(g->ctr, 0, sizeof(Counters), st));
    OutArgs o{src, dst, smp, dep, &g->ctr->out_count, cap};
    if (p->n_samples > 0 && p->depth > 0) {
        int rc = g->idx64 ? dispatch_bias<int64_t>(g, p, fan, seeds, o, st)
                          : dispatch_bias<int32_t>(g, p, fan, seeds, o, st);
        if (rc) {
            cudaStreamSynchronize(st);
            drain_profile(g);
            return rc;
        }
    }
    CK(cudaMemcpyAsync(g->hctr, g->ctr, sizeof(Counters), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    drain_profile(g);
    const Counters &c = *g->hctr;
    g->last.last_edges = (int64_t)c.out_count;
    int64_t items = 0, bytes = 0;
    for (int k = 0; k < KK_COUNT; ++k) {
        items += (int64_t)c.items[k];
        bytes += (int64_t)c.bytes[k];
        g->kbytes[k] += c.bytes[k];
        g->kitems[k] += c.items[k];
    }
    g->last.last_items = items;
    g->last.last_bytes = bytes;
    *n_out = (int64_t)c.out_count;
    if (c.err & ERR_SEED_RANGE) return fail(CSAW_ERR_INVALID, "a seed vertex is out of range");
    if (c.err & ERR_UPDATE_RANGE) return fail(CSAW_ERR_DEVICE, "Update() returned a vertex out of range");
    if (c.err) return fail(CSAW_ERR_DEVICE, "kernel error flag " + std::to_string(c.err));
    if ((int64_t)c.out_count > cap)
        return fail(CSAW_ERR_CAPACITY, "output capacity " + std::to_string(cap) + " < " +
                                           std::to_string(c.out_count) + " edges");
    return 0;
}

}  // namespace

// ===================================================================== C ABI

extern "C" const char *csaw_last_error(void) { return g_err.c_str(); }

extern "C" const char *csaw_version(void) { return "csaw-b200 0.1 (sm_100a)"; }

extern "C" int csaw_graph_create(const void *rowptr, int rowptr_is_64, const int32_t *col,
                                 const float *weights, int64_t n_vertices, int64_t n_edges, int flags,
                                 csaw_graph *out) {
    if (!out) return fail(CSAW_ERR_INVALID, "out is NULL");
    *out = nullptr;
    if (!rowptr || n_vertices < 1 || n_edges < 0 || (n_edges > 0 && !col))
        return fail(CSAW_ERR_INVALID, "bad CSR arguments");
    if (n_vertices >= (1ll << 31)) return fail(CSAW_ERR_INVALID, "vertex ids must fit int32");
    auto rp = [&](int64_t v) -> int64_t {
        return rowptr_is_64 ? ((const int64_t *)rowptr)[v] : (int64_t)((const int32_t *)rowptr)[v];
    };
    if (rp(0) != 0 || rp(n_vertices) != n_edges) return fail(CSAW_ERR_INVALID, "rowptr[0] != 0 or rowptr[V] != E");
    if (!rowptr_is_64 && n_edges >= (1ll << 31)) return fail(CSAW_ERR_INVALID, "E >= 2^31 needs int64 rowptr");
    int64_t maxdeg = 0, n_non = 0;
    std::vector<int32_t> non;
    non.reserve((size_t)n_vertices);
    for (int64_t v = 0; v < n_vertices; ++v) {
        int64_t d = rp(v + 1) - rp(v);
        if (d < 0) return fail(CSAW_ERR_INVALID, "rowptr is not monotone");
        if (d > maxdeg) maxdeg = d;
        if (d > 0) non.push_back((int32_t)v);
    }
    n_non = (int64_t)non.size();
    for (int64_t e = 0; e < n_edges; ++e)
        if (col[e] < 0 || col[e] >= n_vertices) return fail(CSAW_ERR_INVALID, "col entry out of range");
    if (weights)
        for (int64_t e = 0; e < n_edges; ++e)
            if (!(weights[e] >= 0.f) || std::isinf(weights[e]))
                return fail(CSAW_ERR_INVALID, "weights must be finite and >= 0");
    auto *g = new csaw_graph_s();
    cudaGetDevice(&g->device);
    cudaDeviceGetAttribute(&g->sm_count, cudaDevAttrMultiProcessorCount, g->device);
    g->V = n_vertices;
    g->E = n_edges;
    g->maxdeg = maxdeg;
    g->n_non = n_non;
    g->idx64 = rowptr_is_64 ? 1 : 0;
    const size_t rsz = (size_t)(n_vertices + 1) * (rowptr_is_64 ? 8 : 4);
    auto bail = [&](int rc) {
        csaw_graph_destroy(g);
        return rc;
    };
#define CKG(x)                                                                             \
    do {                                                                                   \
        cudaError_t e_ = (x);                                                              \
        if (e_ != cudaSuccess) {                                                           \
            cudaGetLastError();                                                            \
            return bail(fail(e_ == cudaErrorMemoryAllocation ? CSAW_ERR_NOMEM : CSAW_ERR_CUDA, \
                             std::string(#x) + ": " + cudaGetErrorString(e_)));            \
        }                                                                                  \
    } while (0)
    CKG(cudaMalloc(&g->rowptr, rsz));
    CKG(cudaMemcpy(g->rowptr, rowptr, rsz, cudaMemcpyHostToDevice));
    CKG(cudaMalloc((void **)&g->col, sizeof(int32_t) * (size_t)(n_edges > 0 ? n_edges : 1)));
    if (n_edges > 0) CKG(cudaMemcpy(g->col, col, sizeof(int32_t) * (size_t)n_edges, cudaMemcpyHostToDevice));
    g->dev_bytes = (int64_t)rsz + 4 * n_edges;
    if (weights) {
        CKG(cudaMalloc((void **)&g->weight, sizeof(float) * (size_t)(n_edges > 0 ? n_edges : 1)));
        if (n_edges > 0)
            CKG(cudaMemcpy(g->weight, weights, sizeof(float) * (size_t)n_edges, cudaMemcpyHostToDevice));
        g->dev_bytes += 4 * n_edges;
    }
    CKG(cudaMalloc((void **)&g->nonisolated, sizeof(int32_t) * (size_t)(n_non > 0 ? n_non : 1)));
    if (n_non > 0)
        CKG(cudaMemcpy(g->nonisolated, non.data(), sizeof(int32_t) * (size_t)n_non, cudaMemcpyHostToDevice));
    g->dev_bytes += 4 * n_non;
    CKG(cudaMalloc((void **)&g->ctr, sizeof(Counters)));
    CKG(cudaMallocHost((void **)&g->hctr, sizeof(Counters)));
    if ((flags & CSAW_GRAPH_DEGREE_BIAS) && n_edges > 0) {
        CKG(cudaMalloc((void **)&g->ebias, sizeof(float) * (size_t)n_edges));
        g->dev_bytes += 4 * n_edges;
        DevGraph dg = dev_view(g);
        int grid = g->sm_count * 8;
        if (g->idx64) k_edge_degree<int64_t><<<grid, 256>>>(dg, g->ebias);
        else k_edge_degree<int32_t><<<grid, 256>>>(dg, g->ebias);
        g->launches++;
        CKG(cudaGetLastError());
        CKG(cudaDeviceSynchronize());
    }
#undef CKG
    *out = g;
    return 0;
}

extern "C" int csaw_graph_destroy(csaw_graph g) {
    if (!g) return 0;
    cudaSetDevice(g->device);
    cudaFree(g->rowptr);
    cudaFree(g->col);
    cudaFree(g->weight);
    cudaFree(g->ebias);
    cudaFree(g->cdf);
    cudaFree(g->nonisolated);
    for (auto &qq : g->q)
        for (auto &b : qq) cudaFree(b.p);
    cudaFree(g->heavy.p);
    cudaFree(g->hscratch.p);
    cudaFree(g->wscratch.p);
    cudaFree(g->seeds_in.p);
    cudaFree(g->out_dev.p);
    cudaFree(g->ctr);
    if (g->hctr) cudaFreeHost(g->hctr);
    for (auto &pe : g->pending) {
        cudaEventDestroy(pe.second.first);
        cudaEventDestroy(pe.second.second);
    }
    for (auto e : g->event_pool) cudaEventDestroy(e);
    delete g;
    return 0;
}

extern "C" int csaw_graph_stats(csaw_graph g, csaw_stats *out) {
    if (!g || !out) return fail(CSAW_ERR_INVALID, "NULL argument");
    *out = g->last;
    out->n_vertices = g->V;
    out->n_edges = g->E;
    out->max_degree = g->maxdeg;
    out->device_bytes = g->dev_bytes;
    int64_t ws = 0;
    for (auto &qq : g->q)
        for (auto &b : qq) ws += (int64_t)b.n;
    ws += (int64_t)(g->heavy.n + g->hscratch.n + g->wscratch.n + g->seeds_in.n + g->out_dev.n);
    out->workspace_bytes = ws;
    out->kernel_launches = g->launches;
    return 0;
}

extern "C" int csaw_graph_profile(csaw_graph g, int enable) {
    if (!g) return fail(CSAW_ERR_INVALID, "graph is NULL");
    g->prof = enable != 0;
    for (int k = 0; k < KK_COUNT; ++k) {
        g->kms[k] = 0;
        g->klaunch[k] = 0;
        g->kbytes[k] = 0;
        g->kitems[k] = 0;
    }
    return 0;
}

extern "C" int csaw_graph_kernel_stats(csaw_graph g, int kind, double *ms, int64_t *launches,
                                       int64_t *bytes, int64_t *items) {
    if (!g || kind < 0 || kind >= KK_COUNT) return fail(CSAW_ERR_INVALID, "bad kernel kind");
    if (ms) *ms = g->kms[kind];
    if (launches) *launches = g->klaunch[kind];
    if (bytes) *bytes = (int64_t)g->kbytes[kind];
    if (items) *items = (int64_t)g->kitems[kind];
    return 0;
}

extern "C" int csaw_make_seeds(csaw_graph g, int64_t n, uint64_t seed, int32_t *out, void *stream) {
    if (!g || n < 0 || (n > 0 && !out)) return fail(CSAW_ERR_INVALID, "bad arguments");
    if (g->n_non == 0) return fail(CSAW_ERR_INVALID, "graph has no non-isolated vertex");
    if (n == 0) return 0;
    cudaStream_t st = (cudaStream_t)stream;
    int grid = (int)((n + 255) / 256);
    if (grid > g->sm_count * 16) grid = g->sm_count * 16;
    {
        LaunchScope ls(g, KK_INIT, st);
        k_make_seeds<<<grid, 256, 0, st>>>(g->nonisolated, (uint32_t)g->n_non, n, (uint32_t)seed,
                                            (uint32_t)(seed >> 32), out);
    }
    CK(cudaGetLastError());
    return 0;
}

extern "C" int csaw_sample(csaw_graph g, const csaw_params *p, const int32_t *seeds, int32_t *out_src,
                           int32_t *out_dst, int32_t *out_sample, int32_t *out_depth, int64_t capacity,
                           int64_t *n_out, void *stream) {
    return sample_impl(g, p, seeds, out_src, out_dst, out_sample, out_depth, capacity, n_out,
                       (cudaStream_t)stream);
}

extern "C" int csaw_sample_host(csaw_graph g, const csaw_params *p, const int32_t *seeds,
                                int32_t *out_src, int32_t *out_dst, int32_t *out_sample,
                                int32_t *out_depth, int64_t capacity, int64_t *n_out, void *stream) {
    if (!g || !p || !n_out) return fail(CSAW_ERR_INVALID, "NULL argument");
    if (capacity < 0) return fail(CSAW_ERR_INVALID, "capacity < 0");
    cudaStream_t st = (cudaStream_t)stream;
    CK(cudaSetDevice(g->device));
    const int64_t nseeds = (int64_t)p->n_samples * (p->mode == CSAW_MODE_WALK ? 1 : p->frontier_size);
    TRY(ensure(g->seeds_in, sizeof(int32_t) * (size_t)(nseeds > 0 ? nseeds : 1)));
    const int narr = 2 + (out_sample != nullptr) + (out_depth != nullptr);
    TRY(ensure(g->out_dev, sizeof(int32_t) * (size_t)(capacity > 0 ? capacity : 1) * narr));
    if (nseeds > 0)
        CK(cudaMemcpyAsync(g->seeds_in.p, seeds, sizeof(int32_t) * nseeds, cudaMemcpyHostToDevice, st));
    int32_t *d_src = (int32_t *)g->out_dev.p, *d_dst = d_src + capacity;
    int32_t *d_smp = out_sample ? d_dst + capacity : nullptr;
    int32_t *d_dep = out_depth ? (d_smp ? d_smp : d_dst) + capacity : nullptr;
    int rc = sample_impl(g, p, (const int32_t *)g->seeds_in.p, d_src, d_dst, d_smp, d_dep, capacity, n_out, st);
    if (rc) return rc;
    const size_t nb = sizeof(int32_t) * (size_t)*n_out;
    if (nb) {
        CK(cudaMemcpyAsync(out_src, d_src, nb, cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(out_dst, d_dst, nb, cudaMemcpyDeviceToHost, st));
        if (out_sample) CK(cudaMemcpyAsync(out_sample, d_smp, nb, cudaMemcpyDeviceToHost, st));
        if (out_depth) CK(cudaMemcpyAsync(out_depth, d_dep, nb, cudaMemcpyDeviceToHost, st));
    }
    CK(cudaStreamSynchronize(st));
    return 0;
}

// Reference file format: beg.bin = int64[V+1], csr.bin = int64[E]
// (graph.hpp:18-34).
static int read_i64_file(const char *path, std::vector<int64_t> &v) {
    FILE *f = fopen(path, "rb");
    if (!f) return fail(CSAW_ERR_INVALID, std::string("cannot open ") + path);
    fseek(f, 0, SEEK_END);
    long sz = ftell(f);
    fseek(f, 0, SEEK_SET);
    if (sz < 0 || sz % 8) {
        fclose(f);
        return fail(CSAW_ERR_INVALID, std::string("bad int64 file ") + path);
    }
    v.resize((size_t)sz / 8);
    size_t got = fread(v.data(), 8, v.size(), f);
    fclose(f);
    if (got != v.size()) return fail(CSAW_ERR_INVALID, std::string("short read ") + path);
    return 0;
}

extern "C" int csaw_sampler_compat(const char *beg_file, const char *csr_file, int n_blocks, int n_threads,
                                   int n_subgraph, int frontier_size, int neighbor_size, int depth,
                                   int *sampled_edges, double *seconds) {
    (void)n_blocks;
    (void)n_threads;
    if (!beg_file || !csr_file) return fail(CSAW_ERR_INVALID, "NULL file name");
    std::vector<int64_t> beg, adj;
    TRY(read_i64_file(beg_file, beg));
    TRY(read_i64_file(csr_file, adj));
    if (beg.size() < 2) return fail(CSAW_ERR_INVALID, "beg file too small");
    const int64_t V = (int64_t)beg.size() - 1, E = beg.back();
    if (E > (int64_t)adj.size() || E < 0) return fail(CSAW_ERR_INVALID, "csr file shorter than beg[V]");
    std::vector<int32_t> col((size_t)E);
    for (int64_t e = 0; e < E; ++e) {
        if (adj[e] < 0 || adj[e] >= V) return fail(CSAW_ERR_INVALID, "csr entry out of range");
        col[e] = (int32_t)adj[e];
    }
    csaw_graph g = nullptr;
    TRY(csaw_graph_create(beg.data(), 1, col.data(), nullptr, V, E, CSAW_GRAPH_DEGREE_BIAS, &g));
    csaw_params p{};
    p.mode = frontier_size > 1 ? CSAW_MODE_MDRW : CSAW_MODE_NEIGHBOR;
    p.bias = CSAW_BIAS_HOOK;
    p.n_samples = n_subgraph;
    p.frontier_size = frontier_size;
    p.neighbor_size = neighbor_size;
    p.depth = depth;
    p.seed = 56;
    double cap = 0;
    if (p.mode == CSAW_MODE_MDRW) {
        cap = (double)n_subgraph * depth;
    } else {
        double lvl = frontier_size;
        for (int l = 0; l < depth; ++l) {
            lvl *= neighbor_size;
            cap += lvl;
        }
        cap *= n_subgraph;
    }
    if (cap > 2e9) {
        csaw_graph_destroy(g);
        return fail(CSAW_ERR_INVALID, "output bound too large for the compatibility entry");
    }
    int32_t *seeds = nullptr, *out = nullptr;
    const int64_t ns = (int64_t)n_subgraph * frontier_size, c = (int64_t)cap + 1;
    int rc = 0;
    cudaEvent_t e0, e1;
    if (cudaMalloc(&seeds, sizeof(int32_t) * (size_t)(ns > 0 ? ns : 1)) != cudaSuccess ||
        cudaMalloc(&out, sizeof(int32_t) * 2 * (size_t)c) != cudaSuccess) {
        cudaGetLastError();
        rc = fail(CSAW_ERR_NOMEM, "compat output allocation failed");
    }
    int64_t n = 0;
    if (!rc) rc = csaw_make_seeds(g, ns, p.seed, seeds, nullptr);
    if (!rc) {
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        cudaEventRecord(e0);
        rc = csaw_sample(g, &p, seeds, out, out + c, nullptr, nullptr, c, &n, nullptr);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        if (seconds) *seconds = ms * 1e-3;
        if (sampled_edges) *sampled_edges = (int)n;
    }
    cudaFree(seeds);
    cudaFree(out);
    csaw_graph_destroy(g);
    return rc;
}
