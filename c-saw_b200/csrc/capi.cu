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
#include <algorithm>
#include <array>
#include <map>
#include <set>
#include <thread>
#include <vector>

#include "csaw.h"
#include "csaw_internal.h"
#include "kernels_fast.cuh"
#include "kernels_persist.cuh"
#include "sched_mlp.cuh"

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

enum { KK_EXPAND = 0, KK_HEAVY = 1, KK_WALK = 2, KK_MDRW = 3, KK_INIT = 4, KK_SELECT = 5, KK_HUB = 6, KK_PAIR = 7,
       KK_WALK_THREAD = 8, KK_PERSIST = 9, KK_SELECT_THREAD = 10, KK_COUNT = 11 };

struct Counters {
    unsigned long long out_count;
    unsigned long long bytes[KK_COUNT];
    unsigned long long items[KK_COUNT];
    uint32_t nq[2];
    uint32_t n_heavy;
    uint32_t n_sel;
    uint32_t n_cta[4];
    uint32_t n_retry;
    uint32_t n_hub;
    uint32_t n_pair;
    uint32_t n_refill;
    uint32_t n_thread;
    int err;
};

struct DevBuf {
    void *p = nullptr;
    size_t n = 0;
};

// Bumped whenever a device buffer is (re)allocated: cached CUDA graphs that
// captured older addresses are dropped.
uint64_t g_alloc_epoch = 1;

// Grows b to at least `bytes`.  With a stream that is not capturing, the old
// buffer is released and the new one taken stream-ordered (after the work
// already queued on st, without synchronising the device), so a job context
// growing under load does not stall other streams.
int ensure(DevBuf &b, size_t bytes, cudaStream_t st = nullptr) {
    if (b.n >= bytes) return 0;
    ++g_alloc_epoch;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    const bool ordered = st && cudaStreamIsCapturing(st, &cs) == cudaSuccess && cs == cudaStreamCaptureStatusNone;
    if (b.p) {
        if (ordered) cudaFreeAsync(b.p, st);
        else cudaFree(b.p);
    }
    b.p = nullptr;
    b.n = 0;
    if (bytes == 0) return 0;
    cudaError_t e = ordered ? cudaMallocAsync(&b.p, bytes, st) : cudaMalloc(&b.p, bytes);
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
constexpr int64_t SCRATCH_BUDGET = 4ll << 30;        // bytes of high-degree scratch (CTA prefix rebuilds)
// CTA width of the retry pass of cached hubs.  128: one warp resolves an
// item's slots while the others wait for the short incremental rebuild
// passes, so narrow CTAs keep more items in flight (measured: scale-25 step
// 26.2 ms at 256 threads, 25.5 ms at 128, 25.6 ms at 64).
#ifndef CSAW_RETRY_THREADS
#define CSAW_RETRY_THREADS 128
#endif
constexpr int MDRW_MAX_F = 4096;
constexpr int MAX_HOST_PARTS = 8;                   // parts of a host-buffer job (copy-out pipelining)
constexpr int MAX_POSTS = 64;                       // edge-count posts of a host-buffer job
constexpr size_t MAX_GRAPHS = 64;                   // cached CUDA graphs per graph handle
constexpr size_t MAX_WARM = 1024;                   // batch keys remembered for capture

// Per-job device state: counters, frontier queues, work lists and scratch.
// Job 0 serves csaw_sample; csaw_sample_batch runs job i on context i, each
// on its own stream, so independent jobs overlap on the device.
struct JobCtx {
    DevBuf q[2][5], heavy, sel, hlist, hscratch, wscratch, seeds_in, out_dev, cta[4], retry, stab, hubsel, pairsel, dedup,
        pctr,   // per-level counters and barrier words of a persistent job
        tsel;   // thread-per-item list
    Counters *ctr = nullptr, *hctr = nullptr;
    cudaStream_t stream = nullptr;   // owned (batch jobs); job 0 uses the caller's
    cudaEvent_t done = nullptr;
    cudaStream_t side = nullptr;     // CTA-granularity pass, concurrent with the warp pass
    cudaEvent_t fork = nullptr, join = nullptr;
    cudaEvent_t t0 = nullptr, t1 = nullptr;   // timed learned-schedule trial runs
    int trial_arm = -1;                       // arm this job ran under, or -1
    // Host-buffer jobs run as n_parts consecutive sample ranges appended to
    // one output.  While `posting`, the running edge count is posted to the
    // next of the page-locked slots `posts` after every hop and every part
    // (edges below a posted count are final), and the host copies them back
    // on the copy stream while the job still samples.
    int n_parts = 1;
    bool posting = false;
    int n_posts = 0;
    cudaStream_t copy = nullptr;
    unsigned long long *posts = nullptr;
};

}  // namespace

struct csaw_graph_s {
    int device = 0, sm_count = 148;
    int64_t V = 0, E = 0, maxdeg = 0, n_non = 0;
    int idx64 = 0;
    void *rowptr = nullptr;
    int32_t *col = nullptr;
    float *weight = nullptr;
    float *ebias = nullptr;
    bool ebias_flag = false;   // materialised at creation (visible to every schedule)
    float *cdf[4] = {};           // per bias kind: canonical per-vertex prefix, or null
    float2 *tsc[4] = {};          // per bias kind, with cdf: tile summaries of the rows above TSC_MIN_DEG
    int32_t *tsc_verts = nullptr; // those rows
    int64_t n_tsc = 0;
    bool incr_rebuild = true;     // CSAW_OPT_INCR_REBUILD
    bool cdf_flag = false;        // CSAW_GRAPH_CDF_CACHE: visible to the plain schedule too
    bool cdf_off = false;         // CSAW_GRAPH_NO_CDF_CACHE
    int grid_pct = 100;           // CSAW_OPT_GRID_PCT
    bool pair = true;             // CSAW_OPT_PAIR
    int host_parts = 0;           // CSAW_OPT_HOST_PARTS (0: by output size; -1: copy after the job)
    int retry_smem = 0;           // CSAW_OPT_RETRY_SMEM (bytes)
    bool persistent = false;      // CSAW_OPT_PERSISTENT
    int thread_sel = 1;           // CSAW_OPT_THREAD_SELECT: 0 off, 1 degree rule, 2 every d <= 32 item
    uint32_t class_mask = 0x7f;   // classes the trained model picks (bit c)
    int32_t *big_verts = nullptr; // vertices above CDF_BIG (the cache builds them one CTA each)
    int64_t n_big = 0;
    NbrRec *nrec = nullptr;       // per-edge neighbor records (batched schedules)
    int32_t *nonisolated = nullptr;
    int64_t dev_bytes = 0;
    std::vector<JobCtx *> jobs;
    int64_t launches = 0;
    csaw_stats last{};
    bool prof = false;
    double kms[KK_COUNT] = {};
    int64_t klaunch[KK_COUNT] = {};
    unsigned long long kbytes[KK_COUNT] = {}, kitems[KK_COUNT] = {};
    std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> pending;
    std::vector<cudaEvent_t> event_pool;
    // CUDA-graph replay of repeated batches: a batch key seen once runs
    // eagerly (allocating what it needs), the second time it is captured,
    // afterwards it is replayed as one graph launch.
    bool use_graphs = true;
    uint64_t graph_epoch = 0;
    std::set<std::string> warm;
    std::map<std::string, cudaGraphExec_t> graphs;
    std::map<std::string, int64_t> graph_kernels;   // kernel launches per replay
    // learned scheduler
    float2 *vstats = nullptr;         // per-vertex bias statistics
    int vstats_bias = -1;
    float *mlp_w = nullptr, *mlp_m = nullptr, *mlp_v = nullptr, *mlp_norm = nullptr, *mlp_grad = nullptr,
          *mlp_loss = nullptr;
    __nv_bfloat16 *mlp_wq = nullptr;
    ProfRec *rec = nullptr;
    uint32_t *n_rec = nullptr;
    int64_t max_rec = 0;
    bool recording = false, trained = false;
    float last_loss = -1.f;
    // After training, learned jobs alternate between the model's routing
    // (arm 1) and the degree rule (arm 0), timed on the device, until each
    // arm has TRIAL_RUNS runs; the model is kept only if its mean is lower.
    bool trial = false, mlp_lost = false;
    int trial_arm = 1;
    int trial_n[2] = {};
    double trial_ms[2] = {};
    SchedArgs *d_sched = nullptr;     // device copy read by the kernels
    SchedArgs sched_host{};           // what d_sched holds
    bool sched_valid = false;
};

namespace {

// The plain schedule sees the per-edge degree array and the prefix cache only
// when the caller asked for them at creation; the batched schedules
// materialise them on first use.  `bias` selects the prefix cache (-1: none).
DevGraph dev_view(const csaw_graph_s *g, int schedule = CSAW_SCHED_BATCHED, int bias = -1) {
    DevGraph d;
    d.v.rowptr = g->rowptr;
    d.v.rowptr_is_64 = g->idx64;
    d.v.col = g->col;
    d.v.weight = g->weight;
    d.v.n_vertices = g->V;
    d.v.n_edges = g->E;
    d.ebias = (schedule != CSAW_SCHED_PLAIN || g->ebias_flag) ? g->ebias : nullptr;
    const bool fast = schedule != CSAW_SCHED_PLAIN;
    d.cdf = ((fast || g->cdf_flag) && bias > 0 && bias < 4) ? g->cdf[bias] : nullptr;
    d.cdf1 = d.cdf ? d.cdf + g->E : nullptr;
    d.cdf2 = d.cdf ? d.cdf + g->E + ((g->E + 31) >> 5) : nullptr;
    d.cdf_bias = bias;
    d.nrec = fast ? g->nrec : nullptr;
    d.tsc = (d.cdf && g->incr_rebuild) ? g->tsc[bias] : nullptr;
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

// Per-edge neighbor records, built once per graph on first batched use
// (16 E bytes of HBM).
int ensure_nbr(csaw_graph_s *g, cudaStream_t st) {
    if (g->nrec || g->E == 0) return 0;
    ++g_alloc_epoch;
    CK(cudaMalloc((void **)&g->nrec, sizeof(NbrRec) * (size_t)g->E));
    g->dev_bytes += (int64_t)sizeof(NbrRec) * g->E;
    DevGraph dg = dev_view(g);
    LaunchScope ls(g, KK_INIT, st);
    if (g->idx64) k_nbr_records<int64_t><<<g->sm_count * 8, 256, 0, st>>>(dg, g->nrec);
    else k_nbr_records<int32_t><<<g->sm_count * 8, 256, 0, st>>>(dg, g->nrec);
    CK(cudaGetLastError());
    return 0;
}

constexpr int64_t CDF_BIG = 4096;   // vertices above are built by one CTA each
constexpr int RETRY_SMEM_MAX = 96 << 10;   // CSAW_OPT_RETRY_SMEM upper bound (bytes)

// Per-vertex CDF cache: the canonical prefix of every vertex's biases for bias
// kind BIAS (4E bytes, plus its search index), built on first biased use by a
// batched schedule, or by any schedule when the graph was created with
// CSAW_GRAPH_CDF_CACHE; never with CSAW_GRAPH_NO_CDF_CACHE.
template <typename I, int BIAS>
int ensure_cdf(csaw_graph_s *g, cudaStream_t st) {
    if (g->cdf[BIAS]) return 0;
    if (g->E == 0 || g->cdf_off) return 0;
    float *cdf = nullptr;   // prefix [E], then its search index levels [n1] and [n2]
    const int64_t n1 = (g->E + 31) >> 5, n2 = (g->E + 1023) >> 10;
    ++g_alloc_epoch;
    // + 16 floats: a row's 16-byte-aligned bulk-copy window may end up to 12
    // bytes past the row (kernels_fast.cuh, k_select_pair)
    CK(cudaMalloc((void **)&cdf, sizeof(float) * (size_t)(g->E + n1 + n2 + 16)));
    const DevGraph dg = dev_view(g);
    {
        LaunchScope ls(g, KK_INIT, st);
        k_cdf_build<I, BIAS><<<g->sm_count * 8, 256, 0, st>>>(dg, cdf, CDF_BIG, 0, g->V);
    }
    if (g->n_big > 0) {
        const int64_t stride = ((g->maxdeg >> 5) + 1 + (g->maxdeg >> 10) + 1 + 8 + 63) & ~63ll;
        float *scratch = nullptr;
        const int blocks = (int)std::min<int64_t>(g->n_big, g->sm_count * 2);
        CK(cudaMallocAsync((void **)&scratch, sizeof(float) * stride * blocks, st));
        LaunchScope ls(g, KK_INIT, st);
        k_cdf_build_big<I, BIAS><<<blocks, 1024, 0, st>>>(dg, cdf, g->big_verts, (int)g->n_big, scratch, stride);
        CK(cudaFreeAsync(scratch, st));
    }
    {
        LaunchScope ls(g, KK_INIT, st);
        k_cdf_index<<<g->sm_count * 4, 256, 0, st>>>(cdf, g->E, cdf + g->E, n1, cdf + g->E + n1, n2);
    }
    float2 *tsc = nullptr;   // tile summaries of the hub rows (incremental rebuilds)
    if (g->n_tsc > 0) {
        const size_t n = (size_t)((g->E >> 5) + g->V + 1);
        CK(cudaMalloc((void **)&tsc, sizeof(float2) * n));
        LaunchScope ls(g, KK_INIT, st);
        k_tile_summary<I, BIAS><<<(int)std::min<int64_t>(g->n_tsc, g->sm_count * 8), 256, 0, st>>>(
            dg, tsc, g->tsc_verts, (int)g->n_tsc);
        g->dev_bytes += 8 * (int64_t)n;
    }
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(st));
    g->cdf[BIAS] = cdf;
    g->tsc[BIAS] = tsc;
    g->dev_bytes += 4 * (g->E + n1 + n2);
    ++g_alloc_epoch;
    return 0;
}

// Per-vertex bias statistics for the learned scheduler (built once per bias).
template <typename I, int BIAS>
int ensure_vstats(csaw_graph_s *g, cudaStream_t st) {
    if (g->vstats && g->vstats_bias == BIAS) return 0;
    if (!g->vstats) {
        ++g_alloc_epoch;
        CK(cudaMalloc((void **)&g->vstats, sizeof(float2) * (size_t)g->V));
        g->dev_bytes += 8 * g->V;
    }
    DevGraph dg = dev_view(g);
    LaunchScope ls(g, KK_INIT, st);
    k_vertex_stats<I, BIAS><<<g->sm_count * 8, 256, 0, st>>>(dg, g->vstats);
    CK(cudaGetLastError());
    g->vstats_bias = BIAS;
    return 0;
}

// Device SchedArgs for a run of schedule `schedule` with bias `bias`.
int sched_for(csaw_graph_s *g, int schedule, int bias, int warp_slots, cudaStream_t st, const SchedArgs **out) {
    *out = nullptr;
    if (schedule != CSAW_SCHED_LEARNED || bias == CSAW_BIAS_UNBIASED) return 0;
    SchedArgs h{};
    // a trained model that picks neither a CTA class nor the thread class
    // leaves the degree rule in place; one that lost its timed trial is not used
    bool routes = g->trained && (g->class_mask & 0x7cu) && !g->mlp_lost;
    if (routes && g->trial) routes = g->trial_arm == 1;
    h.mode = g->recording ? SCHED_RECORD : (routes ? SCHED_MLP : SCHED_THRESHOLD);
    h.wq = g->mlp_wq;
    h.norm = g->mlp_norm;
    h.vstats = g->vstats;
    h.rec = g->rec;
    h.n_rec = g->n_rec;
    h.max_rec = (uint32_t)g->max_rec;
    h.bias_kind = bias;
    h.warp_slots = warp_slots;
    h.class_mask = g->class_mask;
    if (!g->d_sched) {
        ++g_alloc_epoch;
        CK(cudaMalloc((void **)&g->d_sched, sizeof(SchedArgs)));
    }
    // upload only on change (a change also drops cached graphs, so this never
    // runs inside a stream capture)
    if (!g->sched_valid || memcmp(&h, &g->sched_host, sizeof(SchedArgs)) != 0) {
        CK(cudaStreamSynchronize(st));
        CK(cudaMemcpy(g->d_sched, &h, sizeof(SchedArgs), cudaMemcpyHostToDevice));
        g->sched_host = h;
        g->sched_valid = true;
        ++g_alloc_epoch;
    }
    *out = g->d_sched;
    return 0;
}

int check_params(const csaw_graph_s *g, const csaw_params *p, int fan[CSAW_MAX_DEPTH]) {
    if (!p) return fail(CSAW_ERR_INVALID, "params is NULL");
    if (p->mode < CSAW_MODE_NEIGHBOR || p->mode > CSAW_MODE_MDRW)
        return fail(CSAW_ERR_INVALID, "unknown mode");
    if (p->bias < CSAW_BIAS_UNBIASED || p->bias > CSAW_BIAS_HOOK)
        return fail(CSAW_ERR_INVALID, "unknown bias");
    if (p->schedule < CSAW_SCHED_PLAIN || p->schedule > CSAW_SCHED_LEARNED)
        return fail(CSAW_ERR_INVALID, "unknown schedule");
    if (p->n_samples < 0) return fail(CSAW_ERR_INVALID, "n_samples < 0");
    if (p->sample_base < 0 || p->sample_base + p->n_samples > INT32_MAX)
        return fail(CSAW_ERR_INVALID, "sample ids must fit int32 (sample_base + n_samples)");
    if (p->depth < 0 || p->depth > (p->mode == CSAW_MODE_NEIGHBOR ? CSAW_MAX_DEPTH : (1 << 24) - 64))
        return fail(CSAW_ERR_INVALID, "depth out of range");
    if (p->frontier_size < 1) return fail(CSAW_ERR_INVALID, "frontier_size < 1");
    if (p->bias == CSAW_BIAS_EDGE_WEIGHT && !g->weight)
        return fail(CSAW_ERR_INVALID, "edge-weight bias needs a graph with weights");
    if (p->mode == CSAW_MODE_MDRW && p->bias == CSAW_BIAS_EDGE_WEIGHT)
        return fail(CSAW_ERR_INVALID, "MDRW picks frontier vertices: use a vertex bias");
    if (p->mode == CSAW_MODE_MDRW && p->frontier_size > MDRW_MAX_F)
        return fail(CSAW_ERR_INVALID, "MDRW frontier_size above 4096");
    if (p->flags & ~(int32_t)CSAW_PARAM_DEDUP) return fail(CSAW_ERR_INVALID, "unknown params flags");
    if ((p->flags & CSAW_PARAM_DEDUP) && p->mode != CSAW_MODE_NEIGHBOR)
        return fail(CSAW_ERR_INVALID, "dedup applies to neighbor sampling only");
    if (p->mode == CSAW_MODE_NEIGHBOR) {
        for (int l = 0; l < p->depth; ++l) {
            fan[l] = p->fanout[l] ? p->fanout[l] : p->neighbor_size;
            if (fan[l] < 1 || fan[l] > MAX_FANOUT)
                return fail(CSAW_ERR_INVALID, "NeighborSize must be in [1, 32] for every hop");
        }
    }
    return 0;
}

constexpr unsigned long long POST_PENDING = ~0ull;

// Publishes the running edge count to page-locked host memory (the host
// polls it; written after the kernels before it in stream order, so the
// edges below it are complete).
__global__ void k_post_count(const unsigned long long *count, unsigned long long *host_slot) {
    *(volatile unsigned long long *)host_slot = *count;
    __threadfence_system();
}

// Posts c's running edge count to its next slot (host-buffer jobs only).
void post_count(csaw_graph_s *g, JobCtx *c, cudaStream_t st) {
    if (!c->posting || c->n_posts >= MAX_POSTS) return;
    LaunchScope ls(g, KK_INIT, st);
    k_post_count<<<1, 1, 0, st>>>(&c->ctr->out_count, &c->posts[c->n_posts++]);
}

template <typename I, int BIAS>
int run_neighbor_t(csaw_graph_s *g, JobCtx *c, const csaw_params *p, const int fan[], const int32_t *seeds,
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
    const bool plain = p->schedule == CSAW_SCHED_PLAIN;
    // per-sample dedup: a (sample, vertex) table for every item one chunk can
    // queue (all levels that push), at most half full
    const bool dedup = (p->flags & CSAW_PARAM_DEDUP) != 0 && D > 1;
    uint64_t dmask = 0;
    if (dedup) {
        double items = F, l2 = F;
        for (int l = 0; l + 1 < D; ++l) {
            l2 *= fan[l];
            items += l2;
        }
        const double want = 2.0 * items * (double)B;
        uint64_t slots = 1024;
        while ((double)slots < want) slots <<= 1;
        dmask = slots - 1;
        TRY(ensure(c->dedup, 16 * (size_t)slots, st));
    }
    unsigned long long *dkeys = dedup ? (unsigned long long *)c->dedup.p : nullptr;
    unsigned long long *dvals = dedup ? dkeys + dmask + 1 : nullptr;
    const int dgrid = g->sm_count * 8;
    auto dedup_level = [&](int q, int level) -> int {
        int32_t *qdeg = plain ? nullptr : (int32_t *)c->q[q][4].p;
        LaunchScope ls(g, KK_INIT, st);
        k_dedup_insert<<<dgrid, 256, 0, st>>>((const int32_t *)c->q[q][0].p, (const int32_t *)c->q[q][1].p,
                                              (const uint32_t *)c->q[q][2].p, &c->ctr->nq[q], level, dkeys, dvals,
                                              dmask, &c->ctr->err);
        k_dedup_filter<<<dgrid, 256, 0, st>>>((int32_t *)c->q[q][0].p, (const int32_t *)c->q[q][1].p,
                                              (const uint32_t *)c->q[q][2].p, qdeg, &c->ctr->nq[q], level, dkeys,
                                              dvals, dmask);
        g->launches += 1;   // the second of the pair
        return 0;
    };
    for (int k = 0; k < 2; ++k) {
        for (int a = 0; a < 3; ++a) TRY(ensure(c->q[k][a], sizeof(int32_t) * qcap, st));
        if (!plain) {
            TRY(ensure(c->q[k][3], sizeof(int64_t) * qcap, st));
            TRY(ensure(c->q[k][4], sizeof(int32_t) * qcap, st));
        }
    }
    const SchedArgs *sched = nullptr;
    const int hgrid = plain ? 0 : std::max(1, grid_for(k_select_hub<I, BIAS>, FAST_THREADS, 0, g->sm_count) *
                                                     g->grid_pct / 100);
    const int pgrid = plain ? 0 : std::max(1, grid_for(k_select_pair<I, BIAS>, FAST_THREADS, 0, g->sm_count) *
                                                     g->grid_pct / 100);
    if (BIASED && (!plain || g->cdf_flag)) TRY((ensure_cdf<I, BIAS>(g, st)));
    const bool cached = BIASED && g->cdf[BIAS] && (!plain || g->cdf_flag);
    auto shaped = [&](int gsz) { return std::max(1, (int)((int64_t)gsz * g->grid_pct / 100)); };
    const int sgrid = plain ? 0
                      : shaped(cached ? grid_for(k_select_fast<I, BIAS, true>, FAST_THREADS, 0, g->sm_count)
                                      : grid_for(k_select_fast<I, BIAS, false>, FAST_THREADS, 0, g->sm_count));
    const int tgrid = plain ? 0 : shaped(grid_for(k_select_thread<I, BIAS>, FAST_THREADS, 0, g->sm_count));
    if (!plain) {
        TRY(ensure_nbr(g, st));
        TRY(ensure(c->sel, sizeof(SelEntry) * qcap, st));
        if (cached && g->maxdeg > WF) {
            TRY(ensure(c->retry, sizeof(SelEntry) * qcap, st));
            TRY(ensure(c->hubsel, sizeof(SelEntry) * qcap, st));
            TRY(ensure(c->pairsel, sizeof(SelEntry) * qcap, st));
        }
        if (p->schedule == CSAW_SCHED_LEARNED && BIASED) TRY((ensure_vstats<I, BIAS>(g, st)));
        TRY(sched_for(g, p->schedule, BIAS, sgrid * (FAST_THREADS / 32), st, &sched));
        for (int k = 0; k < 4; ++k)
            if (sched || k == 1) TRY(ensure(c->cta[k], sizeof(SelEntry) * qcap, st));
        if (sched && g->sched_host.mode == SCHED_MLP) TRY(ensure(c->stab, 2 * TAB_N, st));
        if (BIASED && g->thread_sel) TRY(ensure(c->tsel, sizeof(SelEntry) * qcap, st));
    }
    const bool tabled = sched && g->sched_host.mode == SCHED_MLP;
    // CTA classes launched: those the model may pick, and CTA-256 wherever the
    // degree rule needs it (hubs above WF without a cached prefix)
    const bool need256 = g->maxdeg > WF && !cached;
    auto launch_class = [&](int k) {
        if (!sched || g->sched_host.mode == SCHED_THRESHOLD) return k == 1 && need256;
        if (g->sched_host.mode == SCHED_RECORD) return true;
        return ((g->sched_host.class_mask >> (k + 2)) & 1u) || (k == 1 && need256);
    };
    bool any_class = false;
    for (int k = 0; k < 4; ++k) any_class |= launch_class(k);
    const int64_t smem_cap = plain ? WBUF : WF;
    int hblocks = 0;
    int64_t hstride = 0;
    int cta_grid[4] = {0, 0, 0, 0};
    int rgrid = 0;   // the retry pass's grid (CSAW_RETRY_THREADS per CTA)
    if (BIASED && (g->maxdeg > smem_cap || sched)) {
        TRY(ensure(c->heavy, sizeof(uint32_t) * qcap, st));
        hstride = g->maxdeg + 2 * ((g->maxdeg >> 5) + 1) + (g->maxdeg >> 10) + 1 + 8;
        hstride = (hstride + 63) & ~63ll;
        hblocks = g->sm_count * 2;
        const int64_t cap_blocks = std::max<int64_t>(1, SCRATCH_BUDGET / (hstride * 4));
        for (int k = 0; k < 4; ++k) {   // fill the GPU at each CTA width, within the scratch budget
            cta_grid[k] = (int)std::min<int64_t>(grid_for(k_expand_heavy<I, BIAS>, 128 << k, 0, g->sm_count), cap_blocks);
            hblocks = std::max(hblocks, cta_grid[k]);
        }
        rgrid = (int)std::min<int64_t>(grid_for(k_expand_heavy<I, BIAS>, CSAW_RETRY_THREADS, 0, g->sm_count), cap_blocks);
        hblocks = std::max(hblocks, rgrid);
        hblocks = (int)std::min<int64_t>(hblocks, cap_blocks);
        TRY(ensure(c->hscratch, sizeof(float) * hstride * hblocks, st));
    }
    const DevGraph dg = dev_view(g, p->schedule, BIAS);
    const uint64_t seed = p->seed;
    if (!plain && cached && g->maxdeg > WF) {
        static uint64_t smem_set = 0;   // per instantiation: bit = device
        if (g->device < 64 && !((smem_set >> g->device) & 1u)) {
            CK(cudaFuncSetAttribute(k_expand_heavy<I, BIAS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    RETRY_SMEM_MAX));
            smem_set |= 1ull << g->device;
        }
    }
    const int grid = plain ? grid_for(k_expand_warp<I, BIAS>, EXPAND_THREADS, 0, g->sm_count)
                           : shaped(grid_for(k_coop_fast<I, BIAS>, FAST_THREADS, 0, g->sm_count));
    // Persistent job kernel: every level in one cooperative launch (batched
    // degree-rule jobs over a cached prefix, or unbiased; not with dedup,
    // learned routing or more than PERSIST_MAX_LEVELS levels).
    int jgrid = 0;
    bool persist = !plain && g->persistent && !dedup && D <= PERSIST_MAX_LEVELS &&
                   (!sched || g->sched_host.mode == SCHED_THRESHOLD) && (!BIASED || cached);
    if (persist) {
        static uint64_t attr_set = 0;   // per instantiation: bit = device
        if (g->device < 64 && !((attr_set >> g->device) & 1u)) {
            CK(cudaFuncSetAttribute(k_persist<I, BIAS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)PERSIST_SMEM));
            attr_set |= 1ull << g->device;
        }
        int per_sm = 0;
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_persist<I, BIAS>, FAST_THREADS, PERSIST_SMEM));
        jgrid = per_sm * g->sm_count;   // all CTAs resident (cooperative launch)
        const bool retries = cached && g->maxdeg > WF;
        if (jgrid < 1 || (retries && (int64_t)jgrid * hstride * 4 > SCRATCH_BUDGET)) persist = false;
        if (persist) {
            TRY(ensure(c->pctr, sizeof(PersistLevelCtr) * PERSIST_MAX_LEVELS + sizeof(unsigned) * 3 * PERSIST_MAX_LEVELS,
                       st));
            if (retries) TRY(ensure(c->hscratch, sizeof(float) * hstride * (size_t)std::max(hblocks, jgrid), st));
        }
    }
    // Launch arguments of level l (queues ping-pong by level parity).
    auto make_level = [&](int l) {
        const int cur = l & 1, nxt = cur ^ 1;
        LevelArgs a;
        a.in_dep = nullptr;   // every item of this level is at depth l
        a.out_dep = nullptr;
        a.D = D;
        a.in_v = (const int32_t *)c->q[cur][0].p;
        a.in_s = (const int32_t *)c->q[cur][1].p;
        a.in_p = (const uint32_t *)c->q[cur][2].p;
        a.n_in = &c->ctr->nq[cur];
        a.out_v = (int32_t *)c->q[nxt][0].p;
        a.out_s = (int32_t *)c->q[nxt][1].p;
        a.out_p = (uint32_t *)c->q[nxt][2].p;
        a.n_out = &c->ctr->nq[nxt];
        a.in_beg = plain ? nullptr : c->q[cur][3].p;
        a.in_deg = plain ? nullptr : (const int32_t *)c->q[cur][4].p;
        a.out_beg = plain ? nullptr : c->q[nxt][3].p;
        a.out_deg = plain ? nullptr : (int32_t *)c->q[nxt][4].p;
        a.heavy = (uint32_t *)c->heavy.p;
        a.n_heavy = &c->ctr->n_heavy;
        a.sel_list = plain ? nullptr : (SelEntry *)c->sel.p;
        a.n_sel = &c->ctr->n_sel;
        a.heavy_list = nullptr;
        for (int k = 0; k < 4; ++k) a.cta_list[k] = (SelEntry *)c->cta[k].p;
        a.n_cta = c->ctr->n_cta;
        a.sched = sched;
        a.sched_tab = tabled ? (const uint8_t *)c->stab.p : nullptr;
        a.hub_list = (SelEntry *)c->hubsel.p;
        a.n_hub = &c->ctr->n_hub;
        const bool paired = !plain && cached && g->maxdeg > WF && fan[l] <= 16 && g->pair;
        a.pair_list = paired ? (SelEntry *)c->pairsel.p : nullptr;
        a.n_pair = &c->ctr->n_pair;
        a.refill_list = (SelEntry *)c->sel.p;   // free once k_select_fast has run
        a.n_refill = &c->ctr->n_refill;
        a.retry_list = (SelEntry *)c->retry.p;
        a.n_retry = &c->ctr->n_retry;
        // a thread list where some item of the level may take the thread class
        // (the degree rule sends none when N > 16 or when the level cannot
        // reach THREAD_RULE_MIN_ITEMS items; a model that routes or records may)
        double level_items = (double)B * F;
        for (int i = 0; i < l; ++i) level_items *= fan[i];
        const bool model = sched && g->sched_host.mode != SCHED_THRESHOLD;
        const bool rule_thr = fan[l] <= THREAD_RULE_MAX_N && level_items >= (double)THREAD_RULE_MIN_ITEMS;
        const bool thr_level = !plain && BIASED && g->thread_sel && (g->thread_sel == 2 || model || rule_thr);
        a.thread_list = thr_level ? (SelEntry *)c->tsel.p : nullptr;
        a.n_thread = &c->ctr->n_thread;
        a.thread_force = g->thread_sel == 2;
        a.heavy_scratch = (float *)c->hscratch.p;
        a.heavy_stride = hstride;
        a.heavy_smem = 0;   // only the retry launch below has dynamic shared memory
        a.o_src = o.src;
        a.o_dst = o.dst;
        a.o_smp = o.smp;
        a.o_dep = o.dep;
        a.o_count = o.count;
        a.cap = o.cap;
        a.bytes = c->ctr->bytes;
        a.items = c->ctr->items;
        a.err = &c->ctr->err;
        a.k0 = (uint32_t)seed;
        a.k1 = (uint32_t)(seed >> 32);
        a.depth = l;
        a.N = fan[l];
        a.push = l + 1 < D;
        return a;
    };
    for (int64_t s0 = 0; s0 < S; s0 += B) {
        const int64_t nb = (S - s0 < B) ? S - s0 : B;
        const uint32_t n0 = (uint32_t)(nb * F);
        {
            LaunchScope ls(g, KK_INIT, st);
            if (plain)
                k_init_queue<<<(n0 + 255) / 256, 256, 0, st>>>(
                    seeds + s0 * F, n0, F, (int)(p->sample_base + s0), g->V, (int32_t *)c->q[0][0].p, (int32_t *)c->q[0][1].p,
                    (uint32_t *)c->q[0][2].p, &c->ctr->nq[0], &c->ctr->err);
            else
                k_init_queue_fast<I><<<(n0 + 255) / 256, 256, 0, st>>>(
                    dg, seeds + s0 * F, n0, F, (int)(p->sample_base + s0), (int32_t *)c->q[0][0].p, (int32_t *)c->q[0][1].p,
                    (uint32_t *)c->q[0][2].p, (I *)c->q[0][3].p, (int32_t *)c->q[0][4].p, &c->ctr->nq[0],
                    &c->ctr->err);
        }
        if (persist) {
            PersistArgs pa{};
            PersistLevelCtr *pc = (PersistLevelCtr *)c->pctr.p;
            CK(cudaMemsetAsync(c->pctr.p, 0, c->pctr.n, st));
            const bool retries = cached && g->maxdeg > WF;
            for (int l = 0; l < D; ++l) {
                LevelArgs a = make_level(l);
                a.n_in = l == 0 ? &c->ctr->nq[0] : &pc[l - 1].n_out;
                a.n_out = &pc[l].n_out;
                a.n_heavy = &pc[l].n_heavy;
                a.n_sel = &pc[l].n_sel;
                a.n_cta = pc[l].n_cta;
                a.n_retry = &pc[l].n_retry;
                a.n_hub = &pc[l].n_hub;
                a.n_pair = &pc[l].n_pair;
                a.n_refill = &pc[l].n_refill;
                a.thread_list = nullptr;   // the thread pass's registers do not fit the persistent kernel
                a.n_thread = &pc[l].n_thread;
                a.refill_list = (SelEntry *)c->cta[1].p;   // the warp list is still being read beside the pair pass
                pa.lv[l] = a;
                LevelArgs ar = a;
                ar.sel_list = a.refill_list;
                ar.n_sel = a.n_refill;
                pa.refill[l] = ar;
                LevelArgs at = a;
                at.heavy_list = (SelEntry *)c->retry.p;
                at.n_heavy = a.n_retry;
                at.cta_class = 1;
                at.heavy_smem = 0;
                pa.retry[l] = at;
                uint32_t f = 0;
                if (retries) f |= (a.pair_list ? PF_PAIR : PF_HUB) | PF_RETRY;
                pa.flags[l] = f;
                pa.posts[l] = (c->posting && l + 1 < D && c->n_posts < MAX_POSTS) ? &c->posts[c->n_posts++] : nullptr;
            }
            pa.D = D;
            pa.arrive = (unsigned *)(pc + PERSIST_MAX_LEVELS);
            pa.err = &c->ctr->err;
            cudaLaunchConfig_t cfg = {};
            cfg.gridDim = dim3((unsigned)jgrid);
            cfg.blockDim = dim3(FAST_THREADS);
            cfg.dynamicSmemBytes = PERSIST_SMEM;
            cfg.stream = st;
            cudaLaunchAttribute attr[1];
            attr[0].id = cudaLaunchAttributeCooperative;
            attr[0].val.cooperative = 1;
            cfg.attrs = attr;
            cfg.numAttrs = 1;
            LaunchScope ls(g, KK_PERSIST, st);
            CK(cudaLaunchKernelEx(&cfg, k_persist<I, BIAS>, dg, pa));
            continue;
        }
        if (dedup) {
            CK(cudaMemsetAsync(dkeys, 0xff, 16 * (size_t)(dmask + 1), st));
            TRY(dedup_level(0, 0));
        }
        for (int l = 0; l < D; ++l) {
            const int cur = l & 1, nxt = cur ^ 1;
            CK(cudaMemsetAsync(&c->ctr->nq[nxt], 0, sizeof(uint32_t), st));
            CK(cudaMemsetAsync(&c->ctr->n_heavy, 0, 11 * sizeof(uint32_t), st));  // n_heavy .. n_thread
            LevelArgs a = make_level(l);
            if (tabled) {
                LaunchScope ls(g, KK_INIT, st);
                k_sched_table<<<TAB_N * 32 / 256, 256, 0, st>>>(sched, a.n_in, a.N, l, a.thread_list != nullptr,
                                                                 (uint8_t *)c->stab.p);
            }
            {
                LaunchScope ls(g, KK_EXPAND, st);
                if (plain) k_expand_warp<I, BIAS><<<grid, EXPAND_THREADS, 0, st>>>(dg, a);
                else k_coop_fast<I, BIAS><<<grid, FAST_THREADS, 0, st>>>(dg, a);
            }
            const bool side = hblocks && !plain && any_class;
            if (side) {
                // CTA-granularity items on the side stream, concurrent with the
                // warp-granularity pass (disjoint lists, reserved output slots);
                // one launch per CTA width that can hold items (degree rule: 256)
                CK(cudaEventRecord(c->fork, st));
                CK(cudaStreamWaitEvent(c->side, c->fork, 0));
                for (int k = 0; k < 4; ++k) {
                    if (!launch_class(k)) continue;
                    LevelArgs ak = a;
                    ak.heavy_list = (SelEntry *)c->cta[k].p;
                    ak.n_heavy = &c->ctr->n_cta[k];
                    ak.cta_class = k;
                    LaunchScope ls(g, KK_HEAVY, c->side);
                    k_expand_heavy<I, BIAS><<<cta_grid[k], 128 << k, 0, c->side>>>(dg, ak);
                }
                CK(cudaEventRecord(c->join, c->side));
            }
            if (!plain) {
                LaunchScope ls(g, KK_SELECT, st);
                if (cached) k_select_fast<I, BIAS, true><<<sgrid, FAST_THREADS, 0, st>>>(dg, a);
                else k_select_fast<I, BIAS, false><<<sgrid, FAST_THREADS, 0, st>>>(dg, a);
            }
            if (a.thread_list) {
                LaunchScope ls(g, KK_SELECT_THREAD, st);
                k_select_thread<I, BIAS><<<tgrid, FAST_THREADS, 0, st>>>(dg, a);
            }
            // with the pair list, every cached hub (d > WF >= 3N) is paired:
            // the hub list stays empty
            if (!plain && cached && g->maxdeg > WF && !a.pair_list) {
                LaunchScope ls(g, KK_HUB, st);
                k_select_hub<I, BIAS><<<hgrid, FAST_THREADS, 0, st>>>(dg, a);
            }
            if (a.pair_list) {
                {
                    LaunchScope ls(g, KK_PAIR, st);
                    k_select_pair<I, BIAS><<<pgrid, FAST_THREADS, 0, st>>>(dg, a);
                }
                LevelArgs ar = a;   // paired items that need a rebuild, redone by whole warps
                ar.sel_list = a.refill_list;
                ar.n_sel = a.n_refill;
                LaunchScope ls(g, KK_SELECT, st);
                k_select_fast<I, BIAS, true><<<sgrid, FAST_THREADS, 0, st>>>(dg, ar);
            }
            if (hblocks && plain) {
                LaunchScope ls(g, KK_HEAVY, st);
                k_expand_heavy<I, BIAS><<<hblocks, HEAVY_THREADS, 0, st>>>(dg, a);
            }
            if (!plain && cached && g->maxdeg > WF) {
                // cached hubs the warp pass could not rebuild in shared memory
                LevelArgs ar = a;
                ar.heavy_list = (SelEntry *)c->retry.p;
                ar.n_heavy = &c->ctr->n_retry;
                ar.cta_class = 0;   // recorded as the narrowest CTA class
                ar.heavy_smem = g->retry_smem / 4;   // rows whose rebuild fits use shared memory
                LaunchScope ls(g, KK_HEAVY, st);
                k_expand_heavy<I, BIAS><<<rgrid, CSAW_RETRY_THREADS, g->retry_smem, st>>>(dg, ar);
            }
            if (side) CK(cudaStreamWaitEvent(st, c->join, 0));
            if (dedup && l + 1 < D) TRY(dedup_level(nxt, l + 1));
            if (l + 1 < D) post_count(g, c, st);   // this hop's edges are final
        }
    }
    CK(cudaGetLastError());
    return 0;
}

template <typename I, int BIAS>
int run_walk_t(csaw_graph_s *g, JobCtx *c, const csaw_params *p, const int32_t *seeds, const OutArgs &o,
               cudaStream_t st) {
    const bool plain = p->schedule == CSAW_SCHED_PLAIN;
    if (!plain) TRY(ensure_nbr(g, st));
    if (BIAS != CSAW_BIAS_UNBIASED && (!plain || g->cdf_flag)) TRY((ensure_cdf<I, BIAS>(g, st)));
    const DevGraph dg = dev_view(g, p->schedule, BIAS);
    WalkArgs a{};
    a.seeds = seeds;
    a.n = p->n_samples;
    a.len = p->depth;
    a.F = 1;
    a.base = (int)p->sample_base;
    a.o_src = o.src;
    a.o_dst = o.dst;
    a.o_smp = o.smp;
    a.o_dep = o.dep;
    a.o_count = o.count;
    a.cap = o.cap;
    a.bytes = c->ctr->bytes;
    a.items = c->ctr->items;
    a.err = &c->ctr->err;
    a.k0 = (uint32_t)p->seed;
    a.k1 = (uint32_t)(p->seed >> 32);
    if (BIAS == CSAW_BIAS_UNBIASED) {
        int grid = (p->n_samples + WALK_THREADS - 1) / WALK_THREADS;
        int gmax = plain ? grid_for(k_walk_thread<I>, WALK_THREADS, 0, g->sm_count)
                         : grid_for(k_walk_thread_fast<I, CSAW_BIAS_UNBIASED>, WALK_THREADS, 0, g->sm_count);
        if (grid > gmax) grid = gmax;
        LaunchScope ls(g, KK_WALK_THREAD, st);
        if (plain) k_walk_thread<I><<<grid, WALK_THREADS, 0, st>>>(dg, a);
        else k_walk_thread_fast<I, CSAW_BIAS_UNBIASED><<<grid, WALK_THREADS, 0, st>>>(dg, a);
    } else if (!plain && dg.cdf && (int64_t)p->n_samples >= 16ll * grid_for(k_walk_fast<I, BIAS>, FAST_THREADS, 0,
                                                                               g->sm_count) * (FAST_THREADS / 32)) {
        // many biased walks over a cached prefix: one thread per walk
        int grid = (p->n_samples + WALK_THREADS - 1) / WALK_THREADS;
        const int gmax = grid_for(k_walk_thread_fast<I, BIAS>, WALK_THREADS, 0, g->sm_count);
        if (grid > gmax) grid = gmax;
        LaunchScope ls(g, KK_WALK_THREAD, st);
        k_walk_thread_fast<I, BIAS><<<grid, WALK_THREADS, 0, st>>>(dg, a);
    } else {
        int gmax = plain ? grid_for(k_walk_warp<I, BIAS>, WALK_THREADS, 0, g->sm_count)
                         : grid_for(k_walk_fast<I, BIAS>, FAST_THREADS, 0, g->sm_count);
        int grid = (p->n_samples + (WALK_THREADS / 32) - 1) / (WALK_THREADS / 32);
        if (grid > gmax) grid = gmax;
        if (g->maxdeg > (plain ? WBUF : WF) && !dg.cdf) {
            int64_t stride = (g->maxdeg + 63) & ~63ll;
            while (grid > 1 && (int64_t)grid * (WALK_THREADS / 32) * stride * 4 > SCRATCH_BUDGET) grid /= 2;
            TRY(ensure(c->wscratch, sizeof(float) * stride * grid * (WALK_THREADS / 32), st));
            a.scratch = (float *)c->wscratch.p;
            a.scratch_stride = stride;
        }
        LaunchScope ls(g, KK_WALK, st);
        if (plain) k_walk_warp<I, BIAS><<<grid, WALK_THREADS, 0, st>>>(dg, a);
        else k_walk_fast<I, BIAS><<<grid, FAST_THREADS, 0, st>>>(dg, a);
    }
    CK(cudaGetLastError());
    return 0;
}

template <typename I, int BIAS>
int run_mdrw_t(csaw_graph_s *g, JobCtx *c, const csaw_params *p, const int32_t *seeds, const OutArgs &o,
               cudaStream_t st) {
    const DevGraph dg = dev_view(g, p->schedule, BIAS);
    WalkArgs a{};
    a.seeds = seeds;
    a.n = p->n_samples;
    a.len = p->depth;
    a.F = p->frontier_size;
    a.base = (int)p->sample_base;
    a.o_src = o.src;
    a.o_dst = o.dst;
    a.o_smp = o.smp;
    a.o_dep = o.dep;
    a.o_count = o.count;
    a.cap = o.cap;
    a.bytes = c->ctr->bytes;
    a.items = c->ctr->items;
    a.err = &c->ctr->err;
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
int dispatch_bias(csaw_graph_s *g, JobCtx *c, const csaw_params *p, const int fan[], const int32_t *seeds,
                  const OutArgs &o, cudaStream_t st) {
#define CSAW_MODES(BIAS)                                                        \
    switch (p->mode) {                                                          \
        case CSAW_MODE_NEIGHBOR: return run_neighbor_t<I, BIAS>(g, c, p, fan, seeds, o, st); \
        case CSAW_MODE_WALK: return run_walk_t<I, BIAS>(g, c, p, seeds, o, st);    \
        default: return run_mdrw_t<I, BIAS>(g, c, p, seeds, o, st);                \
    }
    switch (p->bias) {
        case CSAW_BIAS_UNBIASED: CSAW_MODES(CSAW_BIAS_UNBIASED)
        case CSAW_BIAS_DEGREE: CSAW_MODES(CSAW_BIAS_DEGREE)
        case CSAW_BIAS_EDGE_WEIGHT:
            if (p->mode == CSAW_MODE_MDRW) return fail(CSAW_ERR_INVALID, "MDRW edge-weight bias");
            if (p->mode == CSAW_MODE_NEIGHBOR)
                return run_neighbor_t<I, CSAW_BIAS_EDGE_WEIGHT>(g, c, p, fan, seeds, o, st);
            return run_walk_t<I, CSAW_BIAS_EDGE_WEIGHT>(g, c, p, seeds, o, st);
        default: CSAW_MODES(CSAW_BIAS_HOOK)
    }
#undef CSAW_MODES
}

void free_job(JobCtx *c);

int new_job(JobCtx **out, bool own_stream) {
    auto *c = new JobCtx();
    cudaError_t e = cudaMalloc((void **)&c->ctr, sizeof(Counters));
    if (e == cudaSuccess) e = cudaMallocHost((void **)&c->hctr, sizeof(Counters));
    if (e == cudaSuccess && own_stream) e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->done, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->side, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->fork, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->join, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->copy, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMallocHost((void **)&c->posts, sizeof(unsigned long long) * MAX_POSTS);
    if (e != cudaSuccess) {
        cudaGetLastError();
        free_job(c);
        return fail(CSAW_ERR_NOMEM, std::string("job context: ") + cudaGetErrorString(e));
    }
    *out = c;
    return 0;
}

void free_job(JobCtx *c) {
    if (!c) return;
    if (c->copy) cudaStreamDestroy(c->copy);
    if (c->posts) cudaFreeHost(c->posts);
    for (auto &qq : c->q)
        for (auto &b : qq) cudaFree(b.p);
    for (DevBuf *b : {&c->heavy, &c->sel, &c->hlist, &c->hscratch, &c->wscratch, &c->seeds_in, &c->out_dev, &c->cta[0],
                      &c->cta[1], &c->cta[2], &c->cta[3], &c->retry, &c->stab, &c->hubsel, &c->pairsel, &c->dedup})
        cudaFree(b->p);
    cudaFree(c->ctr);
    if (c->hctr) cudaFreeHost(c->hctr);
    if (c->stream) cudaStreamDestroy(c->stream);
    if (c->done) cudaEventDestroy(c->done);
    if (c->side) cudaStreamDestroy(c->side);
    if (c->fork) cudaEventDestroy(c->fork);
    if (c->join) cudaEventDestroy(c->join);
    if (c->t0) cudaEventDestroy(c->t0);
    if (c->t1) cudaEventDestroy(c->t1);
    delete c;
}

int64_t job_workspace(const JobCtx *c) {
    int64_t ws = 0;
    for (auto &qq : c->q)
        for (auto &b : qq) ws += (int64_t)b.n;
    for (const DevBuf *b : {&c->heavy, &c->sel, &c->hlist, &c->hscratch, &c->wscratch, &c->seeds_in, &c->out_dev,
                            &c->cta[0], &c->cta[1], &c->cta[2], &c->cta[3], &c->retry, &c->stab, &c->hubsel, &c->pairsel, &c->dedup})
        ws += (int64_t)b->n;
    return ws;
}

int get_job(csaw_graph_s *g, size_t i, JobCtx **out) {
    while (g->jobs.size() <= i) {
        JobCtx *c = nullptr;
        TRY(new_job(&c, true));
        g->jobs.push_back(c);
    }
    *out = g->jobs[i];
    return 0;
}

// Enqueues one job on `st` (no host synchronisation): counter reset, the
// mode's kernels, and the asynchronous read-back of the counter block.
// reset = false appends to the previous job's output and counters (the
// later parts of a host-buffer job).
int enqueue_job(csaw_graph_s *g, JobCtx *c, const csaw_params *p, const int32_t *seeds, int32_t *src,
                int32_t *dst, int32_t *smp, int32_t *dep, int64_t cap, cudaStream_t st, bool reset = true) {
    int fan[CSAW_MAX_DEPTH];
    TRY(check_params(g, p, fan));
    if (cap < 0) return fail(CSAW_ERR_INVALID, "capacity < 0");
    if (cap > 0 && (!src || !dst)) return fail(CSAW_ERR_INVALID, "out_src/out_dst are NULL");
    if (p->n_samples > 0 && !seeds) return fail(CSAW_ERR_INVALID, "seeds is NULL");
    if (reset) CK(cudaMemsetAsync(c->ctr, 0, sizeof(Counters), st));
    OutArgs o{src, dst, smp, dep, &c->ctr->out_count, cap};
    c->trial_arm = -1;
    const bool timed = g->trial && p->schedule == CSAW_SCHED_LEARNED && p->mode == CSAW_MODE_NEIGHBOR &&
                       p->bias != CSAW_BIAS_UNBIASED && p->n_samples > 0 && p->depth > 0;
    if (timed) {
        if (!c->t0) CK(cudaEventCreate(&c->t0));
        if (!c->t1) CK(cudaEventCreate(&c->t1));
        CK(cudaEventRecord(c->t0, st));
    }
    if (p->n_samples > 0 && p->depth > 0) {
        int rc = g->idx64 ? dispatch_bias<int64_t>(g, c, p, fan, seeds, o, st)
                          : dispatch_bias<int32_t>(g, c, p, fan, seeds, o, st);
        if (rc) return rc;
    }
    if (timed) {
        CK(cudaEventRecord(c->t1, st));
        c->trial_arm = g->trial_arm;
    }
    CK(cudaMemcpyAsync(c->hctr, c->ctr, sizeof(Counters), cudaMemcpyDeviceToHost, st));
    return 0;
}

constexpr int TRIAL_RUNS = 3;

// Starts the timed trial of a freshly trained or loaded model (only when it
// picks some CTA class or the thread class; otherwise the degree rule stays).
void start_trial(csaw_graph_s *g) {
    g->mlp_lost = false;
    g->trial = g->trained && (g->class_mask & 0x7cu);
    g->trial_arm = 1;
    g->trial_n[0] = g->trial_n[1] = 0;
    g->trial_ms[0] = g->trial_ms[1] = 0.0;
}

// Folds a finished trial run in; picks the next arm or ends the trial.
void trial_account(csaw_graph_s *g, JobCtx *c) {
    if (c->trial_arm < 0) return;
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, c->t0, c->t1) == cudaSuccess && g->trial) {
        g->trial_ms[c->trial_arm] += ms;
        g->trial_n[c->trial_arm] += 1;
    }
    cudaGetLastError();
    c->trial_arm = -1;
    if (!g->trial) return;
    if (g->trial_n[0] >= TRIAL_RUNS && g->trial_n[1] >= TRIAL_RUNS) {
        g->mlp_lost = g->trial_ms[1] / g->trial_n[1] >= g->trial_ms[0] / g->trial_n[0];
        g->trial = false;
        ++g_alloc_epoch;   // cached graphs hold the trial's routing
    } else {
        g->trial_arm = g->trial_n[1] <= g->trial_n[0] ? 1 : 0;
    }
}

// After the job's stream has been synchronised: edge count, errors, stats.
int finish_job(csaw_graph_s *g, JobCtx *c, int64_t cap, int64_t *n_out) {
    trial_account(g, c);
    const Counters &k = *c->hctr;
    g->last.last_edges += (int64_t)k.out_count;
    for (int i = 0; i < KK_COUNT; ++i) {
        g->last.last_items += (int64_t)k.items[i];
        g->last.last_bytes += (int64_t)k.bytes[i];
        g->kbytes[i] += k.bytes[i];
        g->kitems[i] += k.items[i];
    }
    *n_out = (int64_t)k.out_count;
    if (k.err & ERR_SEED_RANGE) return fail(CSAW_ERR_INVALID, "a seed vertex is out of range");
    if (k.err & ERR_UPDATE_RANGE) return fail(CSAW_ERR_DEVICE, "Update() returned a vertex out of range");
    if (k.err & ERR_BARRIER)
        return fail(CSAW_ERR_DEVICE, "a grid barrier of the persistent job kernel expired (bounded wait)");
    if (k.err & ERR_COPY_WAIT)
        return fail(CSAW_ERR_DEVICE, "an asynchronous row copy did not complete within its bounded wait");
    if (k.err) return fail(CSAW_ERR_DEVICE, "kernel error flag " + std::to_string(k.err));
    if ((int64_t)k.out_count > cap)
        return fail(CSAW_ERR_CAPACITY, "output capacity " + std::to_string(cap) + " < " +
                                           std::to_string(k.out_count) + " edges");
    return 0;
}

void reset_last(csaw_graph_s *g) {
    g->last.last_edges = g->last.last_items = g->last.last_bytes = 0;
}

int64_t seed_count(const csaw_params *p) {
    return (int64_t)p->n_samples * (p->mode == CSAW_MODE_WALK ? 1 : p->frontier_size);
}

}  // namespace

// Accessors for other translation units of this library (declared in
// csaw_host.h); they touch no existing code path.
int csaw_host_fail(int code, const char *msg) { return fail(code, msg); }

int csaw_host_plain_view(csaw_graph g, const csaw_params *p, int fan[CSAW_MAX_DEPTH], DevGraph *view,
                         int64_t *maxdeg, int *device, int *idx64) {
    if (!g) return fail(CSAW_ERR_INVALID, "graph is NULL");
    TRY(check_params(g, p, fan));
    *view = dev_view(g, CSAW_SCHED_PLAIN, p->bias);
    *maxdeg = g->maxdeg;
    *device = g->device;
    *idx64 = g->idx64;
    return 0;
}

int csaw_host_graph_device(csaw_graph g) { return g ? g->device : -1; }

int csaw_host_edge_bound(csaw_graph g, const csaw_params *p, int64_t *bound, int64_t *n_seeds) {
    if (!g) return fail(CSAW_ERR_INVALID, "graph is NULL");
    int fan[CSAW_MAX_DEPTH];
    TRY(check_params(g, p, fan));
    double b = 0;   // saturates instead of overflowing (32^64 for deep fanouts)
    if (p->mode == CSAW_MODE_NEIGHBOR) {
        double lvl = p->frontier_size;
        for (int l = 0; l < p->depth; ++l) {
            lvl *= fan[l];
            b += lvl;
        }
        b *= p->n_samples;
    } else {
        b = (double)p->n_samples * p->depth;
    }
    *bound = b >= 4e18 ? (int64_t)4e18 : (int64_t)b;
    *n_seeds = seed_count(p);
    return 0;
}

int csaw_host_job_create(csaw_graph g, void **job, cudaStream_t *stream) {
    if (!g || !job || !stream) return fail(CSAW_ERR_INVALID, "NULL argument");
    JobCtx *c = nullptr;
    TRY(new_job(&c, true));
    *job = c;
    *stream = c->stream;
    return 0;
}

void csaw_host_job_destroy(void *job) { free_job((JobCtx *)job); }

int64_t csaw_host_job_workspace(const void *job) { return job ? job_workspace((const JobCtx *)job) : 0; }

int csaw_host_job_enqueue(csaw_graph g, void *job, const csaw_params *p, const int32_t *seeds, int32_t *src,
                          int32_t *dst, int32_t *smp, int32_t *dep, int64_t cap) {
    if (!g || !job || !p) return fail(CSAW_ERR_INVALID, "NULL argument");
    JobCtx *c = (JobCtx *)job;
    return enqueue_job(g, c, p, seeds, src, dst, smp, dep, cap, c->stream);
}

int csaw_host_job_finish(csaw_graph g, void *job, int64_t cap, int64_t *n_out) {
    if (!g || !job || !n_out) return fail(CSAW_ERR_INVALID, "NULL argument");
    return finish_job(g, (JobCtx *)job, cap, n_out);
}

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
    std::vector<int32_t> big, hubs;
    for (int64_t v = 0; v < n_vertices; ++v) {
        if (rp(v + 1) - rp(v) > CDF_BIG) big.push_back((int32_t)v);
        if (rp(v + 1) - rp(v) > TSC_MIN_DEG) hubs.push_back((int32_t)v);
    }
    for (int64_t e = 0; e < n_edges; ++e)
        if (col[e] < 0 || col[e] >= n_vertices) return fail(CSAW_ERR_INVALID, "col entry out of range");
    if (weights)
        for (int64_t e = 0; e < n_edges; ++e)
            if (!(weights[e] >= 0.f) || std::isinf(weights[e]))
                return fail(CSAW_ERR_INVALID, "weights must be finite and >= 0");
    auto *g = new csaw_graph_s();
    cudaGetDevice(&g->device);
    cudaDeviceGetAttribute(&g->sm_count, cudaDevAttrMultiProcessorCount, g->device);
    {   // keep up to 2 GiB of freed stream-ordered workspace cached in the
        // device's default pool (process-local), so regrowth maps no memory
        cudaMemPool_t pool;
        if (cudaDeviceGetDefaultMemPool(&pool, g->device) == cudaSuccess) {
            uint64_t thr = 2ull << 30;
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
        }
        cudaGetLastError();
    }
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
    g->cdf_off = (flags & CSAW_GRAPH_NO_CDF_CACHE) != 0;
    g->cdf_flag = !g->cdf_off && (flags & CSAW_GRAPH_CDF_CACHE) != 0;
    g->n_big = (int64_t)big.size();
    if (!big.empty()) {
        CKG(cudaMalloc((void **)&g->big_verts, sizeof(int32_t) * big.size()));
        CKG(cudaMemcpy(g->big_verts, big.data(), sizeof(int32_t) * big.size(), cudaMemcpyHostToDevice));
    }
    g->n_tsc = (int64_t)hubs.size();
    if (!hubs.empty()) {
        CKG(cudaMalloc((void **)&g->tsc_verts, sizeof(int32_t) * hubs.size()));
        CKG(cudaMemcpy(g->tsc_verts, hubs.data(), sizeof(int32_t) * hubs.size(), cudaMemcpyHostToDevice));
    }
    CKG(cudaMalloc((void **)&g->nonisolated, sizeof(int32_t) * (size_t)(n_non > 0 ? n_non : 1)));
    if (n_non > 0)
        CKG(cudaMemcpy(g->nonisolated, non.data(), sizeof(int32_t) * (size_t)n_non, cudaMemcpyHostToDevice));
    g->dev_bytes += 4 * n_non;
    {
        JobCtx *c0 = nullptr;
        int rc = new_job(&c0, false);
        if (rc) return bail(rc);
        g->jobs.push_back(c0);
    }
    if ((flags & CSAW_GRAPH_DEGREE_BIAS) && n_edges > 0) {
        g->ebias_flag = true;
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
    for (float *c : g->cdf) cudaFree(c);
    for (float2 *c : g->tsc) cudaFree(c);
    cudaFree(g->big_verts);
    cudaFree(g->tsc_verts);
    cudaFree(g->nrec);
    cudaFree(g->nonisolated);
    for (auto &kv : g->graphs) cudaGraphExecDestroy(kv.second);
    for (JobCtx *c : g->jobs) free_job(c);
    for (void *q : {(void *)g->vstats, (void *)g->mlp_w, (void *)g->mlp_m, (void *)g->mlp_v, (void *)g->mlp_norm,
                    (void *)g->mlp_grad, (void *)g->mlp_loss, (void *)g->mlp_wq, (void *)g->rec, (void *)g->n_rec,
                    (void *)g->d_sched})
        cudaFree(q);
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
    for (const JobCtx *c : g->jobs) ws += job_workspace(c);
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
    if (!g) return fail(CSAW_ERR_INVALID, "graph is NULL");
    if (!n_out) return fail(CSAW_ERR_INVALID, "n_out is NULL");
    CK(cudaSetDevice(g->device));
    cudaStream_t st = (cudaStream_t)stream;
    JobCtx *c = g->jobs[0];
    reset_last(g);
    int rc = enqueue_job(g, c, p, seeds, out_src, out_dst, out_sample, out_depth, capacity, st);
    cudaError_t e = cudaStreamSynchronize(st);
    drain_profile(g);
    if (rc) return rc;
    if (e != cudaSuccess) return fail(CSAW_ERR_CUDA, std::string("stream sync: ") + cudaGetErrorString(e));
    return finish_job(g, c, capacity, n_out);
}

// Parts a host-buffer job runs in: with P > 1 the output copy of part k
// overlaps the sampling of parts k+1.. (hop posts already overlap the copy
// of a hop's edges with the later hops; parts add overlap for single-kernel
// walks and for the last hop, whose copy of the final part is the tail).  A
// part costs the job's fixed per-kernel latency again, so by default 8 parts
// when the job can emit at least 4 M edges, 4 from 512 K, else 1, and only
// as many as keep each part throughput-bound (8192 samples; walks: 256 per
// SM).  Measured on the scale-25 batch through host buffers: 57.0 ms per
// step with 4 parts, 55.7 ms with 8 (the 3.05 GB copy-back then runs at the
// link's rate).  Never during a timed scheduler trial.
static int host_parts(const csaw_graph_s *g, const csaw_params *p, int64_t cap) {
    const int64_t S = p->n_samples;
    if (g->trial || S < 2 || p->depth < 1) return 1;
    int P = g->host_parts;
    if (P < 0) return 1;
    if (P == 0) {
        int64_t bound = 0, ns = 0;
        if (csaw_host_edge_bound((csaw_graph)g, p, &bound, &ns)) return 1;
        const int64_t min_part = p->mode == CSAW_MODE_WALK ? 256ll * g->sm_count : 8192;
        const int64_t out = std::min(bound, cap);
        P = out >= (4ll << 20) ? 8 : (out >= (512ll << 10) ? 4 : 1);
        while (P > 1 && S / P < min_part) --P;
    }
    return (int)std::max<int64_t>(1, std::min<int64_t>(P, S));
}

// Host-buffer job, before its kernels (never inside a graph capture): the
// device seeds and output buffers, the seeds copied in on `st`, the part
// count and the pending markers the parts overwrite.
static int prepare_host_job(csaw_graph_s *g, JobCtx *c, csaw_job *j, cudaStream_t st, int32_t **dev_out) {
    const csaw_params *p = j->params;
    const int64_t cap = j->capacity;
    if (cap < 0) return fail(CSAW_ERR_INVALID, "capacity < 0");
    const int64_t ns = seed_count(p);
    if (ns < 0) return fail(CSAW_ERR_INVALID, "n_samples < 0");
    if (ns > 0 && !j->seeds) return fail(CSAW_ERR_INVALID, "seeds is NULL");
    if (cap > 0 && (!j->out_src || !j->out_dst)) return fail(CSAW_ERR_INVALID, "out_src/out_dst are NULL");
    TRY(ensure(c->seeds_in, sizeof(int32_t) * (size_t)(ns > 0 ? ns : 1), st));
    const int narr = 2 + (j->out_sample != nullptr) + (j->out_depth != nullptr);
    TRY(ensure(c->out_dev, sizeof(int32_t) * (size_t)(cap > 0 ? cap : 1) * narr, st));
    if (ns > 0) CK(cudaMemcpyAsync(c->seeds_in.p, j->seeds, sizeof(int32_t) * ns, cudaMemcpyHostToDevice, st));
    int32_t *d_src = (int32_t *)c->out_dev.p, *d_dst = d_src + cap;
    int32_t *d_smp = j->out_sample ? d_dst + cap : nullptr;
    int32_t *d_dep = j->out_depth ? (d_smp ? d_smp : d_dst) + cap : nullptr;
    dev_out[0] = d_src;
    dev_out[1] = d_dst;
    dev_out[2] = d_smp;
    dev_out[3] = d_dep;
    c->n_parts = host_parts(g, p, cap);
    for (int k = 0; k < MAX_POSTS; ++k) c->posts[k] = POST_PENDING;
    return 0;
}

// The prepared host-buffer job's kernels on `st` (capturable): its parts,
// consecutive sample ranges appended to one output (sample ids, and so
// every draw, as in one run), posting the edge count after every hop and
// every part.
static int enqueue_host_parts(csaw_graph_s *g, JobCtx *c, const csaw_job *j, cudaStream_t st,
                              int32_t *const *dev_out) {
    const csaw_params *p = j->params;
    const int P = c->n_parts;
    const int64_t S = p->n_samples, per_sample = p->mode == CSAW_MODE_WALK ? 1 : p->frontier_size;
    const int32_t *seeds = (const int32_t *)c->seeds_in.p;
    c->posting = g->host_parts >= 0;
    c->n_posts = 0;
    int rc = 0;
    for (int k = 0; k < P && !rc; ++k) {
        csaw_params q = *p;
        const int64_t s0 = S * k / P, s1 = S * (k + 1) / P;
        if (P > 1) {
            q.n_samples = (int32_t)(s1 - s0);
            q.sample_base = p->sample_base + s0;
        }
        rc = enqueue_job(g, c, &q, seeds + s0 * per_sample, dev_out[0], dev_out[1], dev_out[2], dev_out[3],
                         j->capacity, st, k == 0);
        if (!rc) post_count(g, c, st);
    }
    c->posting = false;
    if (rc) return rc;
    CK(cudaGetLastError());
    return 0;
}

// Copies edges [lo, hi) of a host-buffer job's output back.
static int copy_range(csaw_job *j, int32_t *const *dev_out, int64_t lo, int64_t hi, cudaStream_t st) {
    if (hi <= lo) return 0;
    const size_t nb = sizeof(int32_t) * (size_t)(hi - lo);
    CK(cudaMemcpyAsync(j->out_src + lo, dev_out[0] + lo, nb, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(j->out_dst + lo, dev_out[1] + lo, nb, cudaMemcpyDeviceToHost, st));
    if (j->out_sample) CK(cudaMemcpyAsync(j->out_sample + lo, dev_out[2] + lo, nb, cudaMemcpyDeviceToHost, st));
    if (j->out_depth) CK(cudaMemcpyAsync(j->out_depth + lo, dev_out[3] + lo, nb, cudaMemcpyDeviceToHost, st));
    return 0;
}

// While the batch runs: as a host-buffer job posts edge counts (in slot
// order), copies the edges up to each (clipped to the capacity) back on the
// job's copy stream, so the copy overlaps the sampling still running.
// Returns once `st` (which joins all jobs) has finished or failed and the
// posts made by then are taken.  copied[i]: edges of job i on their way.
static void pipe_copies(csaw_job *jobs, int n_jobs, const std::vector<JobCtx *> &ctx,
                        const std::vector<std::array<int32_t *, 4>> &dev_out, cudaStream_t st,
                        std::vector<int64_t> &copied) {
    std::vector<int> next((size_t)n_jobs, 0);
    bool st_done = false;
    for (;;) {
        bool waiting = false;
        for (int i = 0; i < n_jobs; ++i) {
            JobCtx *c = ctx[i];
            csaw_job &j = jobs[i];
            if (!c || j.status || !j.host_buffers) continue;
            while (next[i] < MAX_POSTS) {
                const unsigned long long v = *(volatile unsigned long long *)&c->posts[next[i]];
                if (v == POST_PENDING) {
                    waiting = true;
                    break;
                }
                const int64_t hi = std::min<int64_t>((int64_t)v, j.capacity);
                if (hi > copied[i] && copy_range(&j, dev_out[i].data(), copied[i], hi, c->copy) == 0) copied[i] = hi;
                ++next[i];
            }
        }
        if (!waiting || st_done) return;
        // all posted counts are in host memory once st has finished
        st_done = cudaStreamQuery(st) != cudaErrorNotReady;
        if (!st_done) std::this_thread::yield();
    }
}

// Forks the jobs from `st` onto their context streams, enqueues them and
// joins them back into `st`.  Host-buffer jobs are already prepared.
static int enqueue_batch(csaw_graph_s *g, csaw_job *jobs, int n_jobs, cudaStream_t st, std::vector<JobCtx *> &ctx,
                         std::vector<std::array<int32_t *, 4>> &dev_out) {
    JobCtx *c0 = g->jobs[0];
    CK(cudaEventRecord(c0->done, st));
    int first_rc = 0;
    for (int i = 0; i < n_jobs; ++i) {
        csaw_job &j = jobs[i];
        if (j.status) continue;   // preparation failed
        int rc = get_job(g, (size_t)i + 1, &ctx[i]);
        if (!rc) rc = cudaStreamWaitEvent(ctx[i]->stream, c0->done, 0) == cudaSuccess ? 0 :
                      fail(CSAW_ERR_CUDA, "cudaStreamWaitEvent failed");
        if (!rc) {
            if (j.host_buffers) rc = enqueue_host_parts(g, ctx[i], &j, ctx[i]->stream, dev_out[i].data());
            else rc = enqueue_job(g, ctx[i], j.params, j.seeds, j.out_src, j.out_dst, j.out_sample, j.out_depth,
                                  j.capacity, ctx[i]->stream);
        }
        j.status = rc;
        if (rc && !first_rc) first_rc = rc;
    }
    for (int i = 0; i < n_jobs; ++i) {
        if (!ctx[i]) continue;
        cudaEventRecord(ctx[i]->done, ctx[i]->stream);
        cudaStreamWaitEvent(st, ctx[i]->done, 0);
    }
    return first_rc;
}

static std::string batch_key(const csaw_graph_s *g, const csaw_job *jobs, int n_jobs) {
    std::string k;
    for (int i = 0; i < n_jobs; ++i) {
        const csaw_job &j = jobs[i];
        k.append((const char *)j.params, sizeof(csaw_params));
        const void *ptrs[7] = {j.seeds, j.out_src, j.out_dst, j.out_sample, j.out_depth,
                               (const void *)(intptr_t)j.capacity, (const void *)(intptr_t)j.host_buffers};
        k.append((const char *)ptrs, sizeof(ptrs));
        if (j.host_buffers) {   // the parts' layout is part of the graph
            const int P = g->host_parts < 0 ? -1 : g->jobs.size() > (size_t)i + 1 ? g->jobs[(size_t)i + 1]->n_parts : 0;
            k.append((const char *)&P, sizeof(P));
        }
    }
    return k;
}

extern "C" int csaw_sample_batch(csaw_graph g, csaw_job *jobs, int n_jobs, void *stream) {
    if (!g) return fail(CSAW_ERR_INVALID, "graph is NULL");
    if (n_jobs < 0 || (n_jobs > 0 && !jobs)) return fail(CSAW_ERR_INVALID, "bad job array");
    if (n_jobs == 0) return 0;
    for (int i = 0; i < n_jobs; ++i)
        if (!jobs[i].params) return fail(CSAW_ERR_INVALID, "job params is NULL");
    CK(cudaSetDevice(g->device));
    cudaStream_t st = (cudaStream_t)stream;
    reset_last(g);
    std::vector<JobCtx *> ctx((size_t)n_jobs);
    std::vector<std::array<int32_t *, 4>> dev_out((size_t)n_jobs);
    for (int i = 0; i < n_jobs; ++i) {
        jobs[i].n_out = 0;
        jobs[i].status = 0;
    }
    int first_rc = 0;
    std::string first_msg;
    bool graphable = g->use_graphs && !g->prof && !g->trial;   // trial runs are timed one by one
    // host-buffer jobs: seeds in and buffers sized before anything is launched
    // or captured (the copies in and out stay outside any graph)
    for (int i = 0; i < n_jobs; ++i) {
        csaw_job &j = jobs[i];
        if (!j.host_buffers) continue;
        int rc = get_job(g, (size_t)i + 1, &ctx[i]);
        if (!rc) rc = prepare_host_job(g, ctx[i], &j, st, dev_out[i].data());
        if (rc) {
            j.status = rc;
            graphable = false;
            if (!first_rc) {
                first_rc = rc;
                first_msg = g_err;
            }
        }
    }
    if (g->graph_epoch != g_alloc_epoch) {   // workspace moved: cached graphs are stale
        for (auto &kv : g->graphs) cudaGraphExecDestroy(kv.second);
        g->graphs.clear();
        g->graph_kernels.clear();
        g->warm.clear();
        g->graph_epoch = g_alloc_epoch;
    }
    std::string key = graphable ? batch_key(g, jobs, n_jobs) : std::string();
    bool launched = false;
    if (graphable) {
        auto it = g->graphs.find(key);
        if (it == g->graphs.end() && g->warm.count(key)) {
            if (g->graphs.size() >= MAX_GRAPHS) {   // callers cycling through many buffers: start over
                for (auto &kv : g->graphs) cudaGraphExecDestroy(kv.second);
                g->graphs.clear();
                g->graph_kernels.clear();
                it = g->graphs.end();
            }
            cudaGraph_t graph = nullptr;
            cudaGraphExec_t exec = nullptr;
            if (cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
                const int64_t l0 = g->launches;
                int rc = enqueue_batch(g, jobs, n_jobs, st, ctx, dev_out);
                cudaError_t e = cudaStreamEndCapture(st, &graph);
                const int64_t nk = g->launches - l0;
                g->launches = l0;   // captured, not run: counted at each replay
                if (!rc && e == cudaSuccess && graph && cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess) {
                    it = g->graphs.emplace(key, exec).first;
                    g->graph_kernels[key] = nk;
                }
                if (graph) cudaGraphDestroy(graph);
            }
            cudaGetLastError();
            if (g->graph_epoch != g_alloc_epoch) {   // something allocated during capture: do not keep it
                if (it != g->graphs.end()) {
                    cudaGraphExecDestroy(it->second);
                    g->graph_kernels.erase(it->first);
                    g->graphs.erase(it);
                }
                it = g->graphs.end();
                g->graph_epoch = g_alloc_epoch;
            }
        }
        if (it != g->graphs.end()) {
            for (int i = 0; i < n_jobs; ++i) {
                ctx[i] = g->jobs[(size_t)i + 1];
                jobs[i].status = 0;
            }
            CK(cudaGraphLaunch(it->second, st));
            g->launches += g->graph_kernels[key];
            launched = true;
        }
    }
    if (!launched) {
        // a capture that was not kept left nothing queued: run eagerly
        if (graphable)
            for (int i = 0; i < n_jobs; ++i) jobs[i].status = 0;   // no preparation failed
        int rc = enqueue_batch(g, jobs, n_jobs, st, ctx, dev_out);
        if (rc && !first_rc) {
            first_rc = rc;
            first_msg = g_err;
        }
    }
    std::vector<int64_t> copied((size_t)n_jobs, 0);
    pipe_copies(jobs, n_jobs, ctx, dev_out, st, copied);
    cudaError_t e = cudaStreamSynchronize(st);
    drain_profile(g);
    if (e != cudaSuccess) {
        for (int i = 0; i < n_jobs; ++i)   // no copy into the caller's buffers outlives the call
            if (jobs[i].host_buffers && ctx[i]) cudaStreamSynchronize(ctx[i]->copy);
        return fail(CSAW_ERR_CUDA, std::string("stream sync: ") + cudaGetErrorString(e));
    }
    for (int i = 0; i < n_jobs; ++i) {
        csaw_job &j = jobs[i];
        if (j.status) continue;
        int rc = finish_job(g, ctx[i], j.capacity, &j.n_out);
        if (!rc && j.host_buffers) rc = copy_range(&j, dev_out[i].data(), copied[i], j.n_out, ctx[i]->copy);
        j.status = rc;
        if (rc && !first_rc) {
            first_rc = rc;
            first_msg = g_err;
        }
    }
    for (int i = 0; i < n_jobs; ++i)
        if (jobs[i].host_buffers && ctx[i]) CK(cudaStreamSynchronize(ctx[i]->copy));
    if (first_rc) {
        g_err = first_msg;
    } else if (graphable && !launched) {
        if (g->warm.size() >= MAX_WARM) g->warm.clear();   // keys of batches seen once
        g->warm.insert(key);
    }
    return first_rc;
}

extern "C" int csaw_sample_host(csaw_graph g, const csaw_params *p, const int32_t *seeds,
                                int32_t *out_src, int32_t *out_dst, int32_t *out_sample,
                                int32_t *out_depth, int64_t capacity, int64_t *n_out, void *stream) {
    if (!g || !p || !n_out) return fail(CSAW_ERR_INVALID, "NULL argument");
    csaw_job j{p, seeds, out_src, out_dst, out_sample, out_depth, capacity, 0, 0, 1};
    int rc = csaw_sample_batch(g, &j, 1, stream);
    *n_out = j.n_out;
    return rc;
}

static int ensure_mlp(csaw_graph_s *g) {
    if (g->mlp_w) return 0;
    ++g_alloc_epoch;
    CK(cudaMalloc((void **)&g->mlp_w, sizeof(float) * MLP_NPARAM));
    CK(cudaMalloc((void **)&g->mlp_m, sizeof(float) * MLP_NPARAM));
    CK(cudaMalloc((void **)&g->mlp_v, sizeof(float) * MLP_NPARAM));
    CK(cudaMalloc((void **)&g->mlp_grad, sizeof(float) * MLP_NPARAM));
    CK(cudaMalloc((void **)&g->mlp_norm, sizeof(float) * MLP_NORM));
    CK(cudaMalloc((void **)&g->mlp_loss, sizeof(float)));
    CK(cudaMalloc((void **)&g->mlp_wq, sizeof(__nv_bfloat16) * MLP_NPARAM));
    CK(cudaMalloc((void **)&g->n_rec, sizeof(uint32_t)));
    CK(cudaMemset(g->n_rec, 0, sizeof(uint32_t)));
    return 0;
}

extern "C" int csaw_graph_set_option(csaw_graph g, int option, int64_t value) {
    if (!g) return fail(CSAW_ERR_INVALID, "graph is NULL");
    CK(cudaSetDevice(g->device));
    switch (option) {
        case CSAW_OPT_CUDA_GRAPHS:
            g->use_graphs = value != 0;
            return 0;
        case CSAW_OPT_SCHED_RECORD:
            if (value < 0) return fail(CSAW_ERR_INVALID, "record capacity < 0");
            TRY(ensure_mlp(g));
            if (value > g->max_rec) {
                ++g_alloc_epoch;
                cudaFree(g->rec);
                g->rec = nullptr;
                CK(cudaMalloc((void **)&g->rec, sizeof(ProfRec) * (size_t)value));
                g->max_rec = value;
            }
            if (value > 0) CK(cudaMemset(g->n_rec, 0, sizeof(uint32_t)));
            g->recording = value > 0;
            ++g_alloc_epoch;   // launch sets differ by mode: drop cached graphs
            return 0;
        case CSAW_OPT_GRID_PCT:
            if (value < 25 || value > 400) return fail(CSAW_ERR_INVALID, "grid percent must be in [25, 400]");
            g->grid_pct = (int)value;
            ++g_alloc_epoch;   // launch shapes are baked into cached graphs
            return 0;
        case CSAW_OPT_PAIR:
            g->pair = value != 0;
            ++g_alloc_epoch;
            return 0;
        case CSAW_OPT_HOST_PARTS:
            if (value < -1 || value > MAX_HOST_PARTS) return fail(CSAW_ERR_INVALID, "host parts must be in [-1, 8]");
            g->host_parts = (int)value;
            return 0;
        case CSAW_OPT_INCR_REBUILD:
            g->incr_rebuild = value != 0;
            ++g_alloc_epoch;   // the device view is baked into cached graphs
            return 0;
        case CSAW_OPT_THREAD_SELECT:
            if (value < 0 || value > 2) return fail(CSAW_ERR_INVALID, "thread select: 0, 1 or 2");
            g->thread_sel = (int)value;
            ++g_alloc_epoch;   // launch structure is baked into cached graphs
            return 0;
        case CSAW_OPT_PERSISTENT:
            g->persistent = value != 0;
            ++g_alloc_epoch;   // launch structure is baked into cached graphs
            return 0;
        case CSAW_OPT_RETRY_SMEM:
            if (value < 0 || value > RETRY_SMEM_MAX) return fail(CSAW_ERR_INVALID, "retry shared memory must be in [0, 98304]");
            g->retry_smem = (int)(value & ~15ll);
            ++g_alloc_epoch;   // launch shapes are baked into cached graphs
            return 0;
        default:
            return fail(CSAW_ERR_INVALID, "unknown option");
    }
}

extern "C" int csaw_graph_autotune(csaw_graph g, csaw_job *jobs, int n_jobs, void *stream, csaw_tune_result *out) {
    if (!g || !out) return fail(CSAW_ERR_INVALID, "NULL argument");
    CK(cudaSetDevice(g->device));
    cudaStream_t st = (cudaStream_t)stream;
    const int pcts[3] = {100, 50, 200};
    const int old_pct = g->grid_pct;
    const bool old_pair = g->pair, old_graphs = g->use_graphs, old_persist = g->persistent;
    g->use_graphs = false;   // each candidate timed launch by launch
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    double best = 1e300, dflt = 0.0;
    int best_pct = old_pct, n = 0;
    bool best_pair = old_pair, best_persist = old_persist;
    int rc = 0;
    // candidates: per-level launches (grid % x pairing), then the persistent
    // job kernel (its grid is the occupancy-filled one) with pairing
    for (int cand = 0; cand < 7 && !rc; ++cand) {
        const int pair = cand < 3 || cand == 6 ? 1 : 0, k = cand % 3;
        g->persistent = cand == 6;
        g->grid_pct = cand == 6 ? 100 : pcts[k];
        g->pair = pair != 0;
        rc = csaw_sample_batch(g, jobs, n_jobs, stream);   // untimed: workspace, caches
        if (rc) break;
        cudaEventRecord(e0, st);
        rc = csaw_sample_batch(g, jobs, n_jobs, stream);
        cudaEventRecord(e1, st);
        if (rc) break;
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        ++n;
        if (cand == 0) dflt = ms;
        if (ms < best) {
            best = ms;
            best_pct = g->grid_pct;
            best_pair = pair != 0;
            best_persist = g->persistent;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    g->use_graphs = old_graphs;
    if (rc) {
        g->grid_pct = old_pct;
        g->pair = old_pair;
        g->persistent = old_persist;
        return rc;
    }
    g->grid_pct = best_pct;
    g->pair = best_pair;
    g->persistent = best_persist;
    ++g_alloc_epoch;
    out->grid_pct = best_pct;
    out->pair = best_pair ? 1 : 0;
    out->best_ms = best;
    out->default_ms = dflt;
    out->candidates = n;
    out->persistent = best_persist ? 1 : 0;
    return 0;
}

extern "C" int csaw_sched_info(csaw_graph g, int64_t *n_records, int *trained, float *last_loss) {
    if (!g) return fail(CSAW_ERR_INVALID, "graph is NULL");
    uint32_t n = 0;
    if (g->n_rec) CK(cudaMemcpy(&n, g->n_rec, sizeof(n), cudaMemcpyDeviceToHost));
    if (n_records) *n_records = std::min<int64_t>(n, g->max_rec);
    if (trained) *trained = g->trained ? 1 : 0;
    if (last_loss) *last_loss = g->last_loss;
    return 0;
}

// Class mask of a trained model: classes 0 and 1 always (the warp pass),
// CTA classes and the thread class only where the model picks them on its
// training records.
static int pick_classes(csaw_graph_s *g, int n) {
    g->class_mask = 0x7f;
    if (n <= 0) return 0;
    uint32_t *m = nullptr;
    CK(cudaMalloc((void **)&m, sizeof(uint32_t)));
    CK(cudaMemset(m, 0, sizeof(uint32_t)));
    const int slots = grid_for(k_select_fast<int32_t, CSAW_BIAS_EDGE_WEIGHT, false>, FAST_THREADS, 0, g->sm_count) *
                      (FAST_THREADS / 32);
    k_sched_pick<<<g->sm_count * 4, 256>>>(g->rec, n, g->mlp_wq, g->mlp_norm, slots, WF, m);
    uint32_t h = 0;
    cudaError_t e = cudaMemcpy(&h, m, sizeof(uint32_t), cudaMemcpyDeviceToHost);
    cudaFree(m);
    CK(e);
    g->class_mask = h | 0x3u;
    g->launches += 1;
    return 0;
}

extern "C" int csaw_sched_classes(csaw_graph g, uint32_t *mask) {
    if (!g || !mask) return fail(CSAW_ERR_INVALID, "NULL argument");
    *mask = !g->trained ? 0x7fu : (g->mlp_lost ? 0x3u : g->class_mask);
    return 0;
}

// Full-batch Adam on the recorded profiles; initial weights are He-scaled
// uniform from a 64-bit LCG keyed by `seed`.
extern "C" int csaw_sched_train(csaw_graph g, int epochs, float lr, uint64_t seed, float *final_loss) {
    if (!g) return fail(CSAW_ERR_INVALID, "graph is NULL");
    if (epochs < 1 || !(lr > 0.f)) return fail(CSAW_ERR_INVALID, "epochs >= 1 and lr > 0 required");
    CK(cudaSetDevice(g->device));
    TRY(ensure_mlp(g));
    int64_t n = 0;
    TRY(csaw_sched_info(g, &n, nullptr, nullptr));
    if (n < 16) return fail(CSAW_ERR_INVALID, "fewer than 16 recorded profiles: run the learned schedule with "
                                              "CSAW_OPT_SCHED_RECORD first");
    std::vector<float> w(MLP_NPARAM, 0.f);
    uint64_t st = seed * 6364136223846793005ull + 1442695040888963407ull;
    auto uni = [&]() {
        st = st * 6364136223846793005ull + 1442695040888963407ull;
        return (float)((st >> 40) * (1.0 / 16777216.0)) * 2.f - 1.f;
    };
    for (int i = 0; i < MLP_H * MLP_IN; ++i) w[MLP_W1 + i] = uni() * sqrtf(6.f / MLP_IN);
    for (int i = 0; i < MLP_H * MLP_H; ++i) w[MLP_W2 + i] = uni() * sqrtf(6.f / MLP_H);
    for (int i = 0; i < MLP_OUT * MLP_H; ++i) w[MLP_W3 + i] = uni() * sqrtf(3.f / MLP_H);
    CK(cudaMemcpy(g->mlp_w, w.data(), sizeof(float) * MLP_NPARAM, cudaMemcpyHostToDevice));
    CK(cudaMemset(g->mlp_m, 0, sizeof(float) * MLP_NPARAM));
    CK(cudaMemset(g->mlp_v, 0, sizeof(float) * MLP_NPARAM));
    k_mlp_norm<<<1, 1024>>>(g->rec, (int)n, g->mlp_norm);
    const int gb = (int)std::min<int64_t>(g->sm_count * 2, (n + MLP_GRAD_THREADS - 1) / MLP_GRAD_THREADS);
    for (int e = 1; e <= epochs; ++e) {
        cudaMemsetAsync(g->mlp_grad, 0, sizeof(float) * MLP_NPARAM);
        k_mlp_grad<<<gb, MLP_GRAD_THREADS>>>(g->mlp_w, g->mlp_norm, g->rec, (int)n, g->mlp_grad, g->mlp_loss);
        k_mlp_adam<<<(MLP_NPARAM + 255) / 256, 256>>>(g->mlp_w, g->mlp_grad, g->mlp_m, g->mlp_v, lr, e, (int)n);
    }
    cudaMemsetAsync(g->mlp_grad, 0, sizeof(float) * MLP_NPARAM);
    cudaMemsetAsync(g->mlp_loss, 0, sizeof(float));
    k_mlp_grad<<<gb, MLP_GRAD_THREADS>>>(g->mlp_w, g->mlp_norm, g->rec, (int)n, g->mlp_grad, g->mlp_loss);
    k_mlp_to_bf16<<<(MLP_NPARAM + 255) / 256, 256>>>(g->mlp_w, g->mlp_wq);
    g->launches += 2 * epochs + 3;
    CK(cudaGetLastError());
    TRY(pick_classes(g, (int)n));
    float loss = 0.f;
    CK(cudaMemcpy(&loss, g->mlp_loss, sizeof(float), cudaMemcpyDeviceToHost));
    loss /= (float)n;
    g->last_loss = loss;
    g->trained = true;
    start_trial(g);
    g->recording = false;
    ++g_alloc_epoch;
    if (final_loss) *final_loss = loss;
    return 0;
}

extern "C" int csaw_sched_get_records(csaw_graph g, void *out, int64_t max_n, int64_t *n) {
    if (!g || !n || (max_n > 0 && !out)) return fail(CSAW_ERR_INVALID, "bad arguments");
    int64_t have = 0;
    TRY(csaw_sched_info(g, &have, nullptr, nullptr));
    *n = std::min(have, max_n);
    if (*n > 0) CK(cudaMemcpy(out, g->rec, sizeof(ProfRec) * (size_t)*n, cudaMemcpyDeviceToHost));
    return 0;
}

extern "C" int csaw_sched_get_model(csaw_graph g, float *params, float *norm) {
    if (!g || !g->trained) return fail(CSAW_ERR_INVALID, "no trained model");
    if (params) CK(cudaMemcpy(params, g->mlp_w, sizeof(float) * MLP_NPARAM, cudaMemcpyDeviceToHost));
    if (norm) CK(cudaMemcpy(norm, g->mlp_norm, sizeof(float) * MLP_NORM, cudaMemcpyDeviceToHost));
    return 0;
}

extern "C" int csaw_sched_set_model(csaw_graph g, const float *params, const float *norm) {
    if (!g || !params || !norm) return fail(CSAW_ERR_INVALID, "NULL argument");
    CK(cudaSetDevice(g->device));
    TRY(ensure_mlp(g));
    CK(cudaMemcpy(g->mlp_w, params, sizeof(float) * MLP_NPARAM, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(g->mlp_norm, norm, sizeof(float) * MLP_NORM, cudaMemcpyHostToDevice));
    k_mlp_to_bf16<<<(MLP_NPARAM + 255) / 256, 256>>>(g->mlp_w, g->mlp_wq);
    CK(cudaGetLastError());
    CK(cudaDeviceSynchronize());
    g->class_mask = 0x7f;   // no training records to prune by
    g->trained = true;
    start_trial(g);
    g->recording = false;
    ++g_alloc_epoch;
    return 0;
}

extern "C" int csaw_mlp_grad_host(const float *params, const float *norm, const void *records, int n, float *grad,
                                  float *loss) {
    if (!params || !norm || !records || n < 1 || !grad) return fail(CSAW_ERR_INVALID, "bad arguments");
    float *dw = nullptr, *dn = nullptr, *dg = nullptr, *dl = nullptr;
    ProfRec *dr = nullptr;
    int rc = 0;
    if (cudaMalloc((void **)&dw, sizeof(float) * MLP_NPARAM) != cudaSuccess ||
        cudaMalloc((void **)&dn, sizeof(float) * MLP_NORM) != cudaSuccess ||
        cudaMalloc((void **)&dg, sizeof(float) * MLP_NPARAM) != cudaSuccess ||
        cudaMalloc((void **)&dl, sizeof(float)) != cudaSuccess ||
        cudaMalloc((void **)&dr, sizeof(ProfRec) * (size_t)n) != cudaSuccess) {
        cudaGetLastError();
        rc = fail(CSAW_ERR_NOMEM, "allocation failed");
    }
    if (!rc) {
        cudaMemcpy(dw, params, sizeof(float) * MLP_NPARAM, cudaMemcpyHostToDevice);
        cudaMemcpy(dn, norm, sizeof(float) * MLP_NORM, cudaMemcpyHostToDevice);
        cudaMemcpy(dr, records, sizeof(ProfRec) * (size_t)n, cudaMemcpyHostToDevice);
        cudaMemset(dg, 0, sizeof(float) * MLP_NPARAM);
        cudaMemset(dl, 0, sizeof(float));
        k_mlp_grad<<<std::min(64, (n + MLP_GRAD_THREADS - 1) / MLP_GRAD_THREADS), MLP_GRAD_THREADS>>>(dw, dn, dr, n,
                                                                                                   dg, dl);
        cudaMemcpy(grad, dg, sizeof(float) * MLP_NPARAM, cudaMemcpyDeviceToHost);
        for (int i = 0; i < MLP_NPARAM; ++i) grad[i] /= (float)n;
        if (loss) {
            cudaMemcpy(loss, dl, sizeof(float), cudaMemcpyDeviceToHost);
            *loss /= (float)n;
        }
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) rc = fail(CSAW_ERR_CUDA, cudaGetErrorString(e));
    }
    cudaFree(dw);
    cudaFree(dn);
    cudaFree(dg);
    cudaFree(dl);
    cudaFree(dr);
    return rc;
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
