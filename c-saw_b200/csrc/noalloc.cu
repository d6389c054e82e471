// noalloc.cu -- neighbor sampling that allocates no device memory.
//
// Some callers cannot call cudaMalloc while they sample: a serving loop that
// reserved its whole memory budget at start-up and must not grow or fragment
// it, a host thread that must not stall on the implicit device
// synchronisation cudaMalloc/cudaFree can cause, or code that runs inside
// another framework's memory pool and may not allocate behind its back.  For
// them csaw_sample_noalloc runs the plain neighbor-sampling level loop with
// its frontier queues and counters in one file-scope device array of fixed
// size instead of the graph's grow-only workspace.  The graph must already be
// resident (csaw_graph_create, called at set-up) and the caller passes seeds
// and output buffers, as for csaw_sample.
//
// Limits and sharing:
//   - the array is NOALLOC_BYTES (32 MiB) and every GPU that loads the
//     library holds it until the process exits;
//   - a job must fit: two levels of frontier queues of 12 bytes per item, so
//     at most (32 MiB - 256 B) / 24 items in the largest level (about 1.4 M),
//     and biased sampling needs max degree <= 1024 (no high-degree scratch);
//     anything larger is rejected with CSAW_ERR_INVALID before any GPU work;
//   - every call on a device shares the one array and the array keeps the last
//     call's contents; the counters are cleared at the start of each call, but
//     two calls whose work overlaps on the GPU (different streams, or host
//     threads) race on the same queues -- serialise them;
//   - the first call on a device looks up the array's device address
//     (cudaGetSymbolAddress, with that device current); with CUDA's lazy
//     module loading that call may also load this library's device code and
//     reserve the array, so make the first call during set-up, before any
//     stream capture;
//   - p->schedule is ignored: the plain level loop always runs (every
//     schedule gives the same output).
#include <cuda_runtime.h>

#include <mutex>

#include "csaw.h"
#include "csaw_host.h"
#include "csaw_internal.h"
#include "kernels_sample.cuh"

using namespace csaw;

namespace {

constexpr size_t NOALLOC_BYTES = 32u << 20;
constexpr size_t COUNTER_BYTES = 256;

static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_BYTES];

struct NoAllocCounters {
    unsigned long long out_count;
    unsigned long long bytes[8];
    unsigned long long items[8];
    uint32_t nq[2];
    uint32_t n_heavy;
    int err;
};
static_assert(sizeof(NoAllocCounters) <= COUNTER_BYTES, "counter block");

constexpr int MAX_DEVICES = 64;
std::mutex g_mu;
void *g_addr[MAX_DEVICES] = {};

// Device address of the array on `device` (which must be current).
int scratch_address(int device, unsigned char **out) {
    if (device < 0 || device >= MAX_DEVICES) return csaw_host_fail(CSAW_ERR_INVALID, "device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_addr[device]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            cudaGetLastError();
            return csaw_host_fail(CSAW_ERR_CUDA, "cudaGetSymbolAddress of the no-alloc scratch failed");
        }
        g_addr[device] = p;
    }
    *out = (unsigned char *)g_addr[device];
    return 0;
}

template <typename I, int BIAS>
void launch_levels(const DevGraph &dg, const csaw_params *p, const int fan[], const int32_t *seeds,
                   unsigned char *base, int64_t qcap, int32_t *src, int32_t *dst, int32_t *smp, int32_t *dep,
                   int64_t cap, int grid, cudaStream_t st) {
    NoAllocCounters *c = (NoAllocCounters *)base;
    int32_t *q[2][3];
    unsigned char *cur = base + COUNTER_BYTES;
    for (int k = 0; k < 2; ++k)
        for (int a = 0; a < 3; ++a) {
            q[k][a] = (int32_t *)cur;
            cur += sizeof(int32_t) * (size_t)qcap;
        }
    const int S = p->n_samples, F = p->frontier_size, D = p->depth;
    const uint32_t n0 = (uint32_t)((int64_t)S * F);
    k_init_queue<<<(n0 + 255) / 256, 256, 0, st>>>(seeds, n0, F, (int)p->sample_base, dg.v.n_vertices, q[0][0], q[0][1],
                                                   (uint32_t *)q[0][2], &c->nq[0], &c->err);
    for (int l = 0; l < D; ++l) {
        const int s = l & 1, t = s ^ 1;
        cudaMemsetAsync(&c->nq[t], 0, sizeof(uint32_t), st);
        LevelArgs a{};
        a.in_v = q[s][0];
        a.in_s = q[s][1];
        a.in_p = (const uint32_t *)q[s][2];
        a.n_in = &c->nq[s];
        a.out_v = q[t][0];
        a.out_s = q[t][1];
        a.out_p = (uint32_t *)q[t][2];
        a.n_out = &c->nq[t];
        a.n_heavy = &c->n_heavy;
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
        k_expand_warp<I, BIAS><<<grid, EXPAND_THREADS, 0, st>>>(dg, a);
    }
}

template <typename I>
int dispatch(const DevGraph &dg, const csaw_params *p, const int fan[], const int32_t *seeds, unsigned char *base,
             int64_t qcap, int32_t *src, int32_t *dst, int32_t *smp, int32_t *dep, int64_t cap, int sm, cudaStream_t st) {
    int per_sm = 1;
    switch (p->bias) {
#define CSAW_NOALLOC_BIAS(B)                                                                          \
    case B:                                                                                           \
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_expand_warp<I, B>, EXPAND_THREADS, 0); \
        launch_levels<I, B>(dg, p, fan, seeds, base, qcap, src, dst, smp, dep, cap, sm * (per_sm > 0 ? per_sm : 1), st); \
        break;
        CSAW_NOALLOC_BIAS(CSAW_BIAS_UNBIASED)
        CSAW_NOALLOC_BIAS(CSAW_BIAS_DEGREE)
        CSAW_NOALLOC_BIAS(CSAW_BIAS_EDGE_WEIGHT)
        CSAW_NOALLOC_BIAS(CSAW_BIAS_HOOK)
#undef CSAW_NOALLOC_BIAS
        default: return csaw_host_fail(CSAW_ERR_INVALID, "unknown bias");
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return csaw_host_fail(CSAW_ERR_CUDA, cudaGetErrorString(e));
    return 0;
}

}  // namespace

extern "C" int csaw_sample_noalloc(csaw_graph g, const csaw_params *p, const int32_t *seeds, int32_t *out_src,
                                   int32_t *out_dst, int32_t *out_sample, int32_t *out_depth, int64_t capacity,
                                   int64_t *n_out, void *stream) {
    int fan[CSAW_MAX_DEPTH];
    DevGraph dg;
    int64_t maxdeg = 0;
    int device = 0, idx64 = 0;
    if (!n_out) return csaw_host_fail(CSAW_ERR_INVALID, "n_out is NULL");
    *n_out = 0;
    if (!p) return csaw_host_fail(CSAW_ERR_INVALID, "params is NULL");
    int rc = csaw_host_plain_view(g, p, fan, &dg, &maxdeg, &device, &idx64);
    if (rc) return rc;
    if (p->mode != CSAW_MODE_NEIGHBOR)
        return csaw_host_fail(CSAW_ERR_INVALID, "csaw_sample_noalloc runs neighbor sampling only");
    if (p->flags) return csaw_host_fail(CSAW_ERR_INVALID, "csaw_sample_noalloc does not take params flags (dedup)");
    if (p->bias != CSAW_BIAS_UNBIASED && maxdeg > WBUF)
        return csaw_host_fail(CSAW_ERR_INVALID,
                              "csaw_sample_noalloc: biased sampling needs max degree <= 1024 (no high-degree scratch)");
    if (capacity < 0 || (capacity > 0 && (!out_src || !out_dst)))
        return csaw_host_fail(CSAW_ERR_INVALID, "bad output buffers");
    if (p->n_samples > 0 && !seeds) return csaw_host_fail(CSAW_ERR_INVALID, "seeds is NULL");
    // largest level, all samples at once (no chunking: the array is fixed)
    double level = (double)p->n_samples * p->frontier_size, largest = level;
    for (int l = 0; l + 1 < p->depth; ++l) {
        level *= fan[l];
        if (level > largest) largest = level;
    }
    const int64_t max_items = (int64_t)((NOALLOC_BYTES - COUNTER_BYTES) / (2 * 3 * sizeof(int32_t)));
    if (largest > (double)max_items)
        return csaw_host_fail(CSAW_ERR_INVALID,
                              "csaw_sample_noalloc: a frontier level may exceed the 32 MiB scratch "
                              "(at most 1398090 items per level: reduce samples or fanout)");
    if (p->n_samples == 0 || p->depth == 0) return 0;
    if (largest / p->n_samples > 4294967295.0)
        return csaw_host_fail(CSAW_ERR_INVALID, "lineage items exceed 2^32");
    if (cudaSetDevice(device) != cudaSuccess) return csaw_host_fail(CSAW_ERR_CUDA, "cudaSetDevice failed");
    unsigned char *base = nullptr;
    rc = scratch_address(device, &base);
    if (rc) return rc;
    int sm = 148;
    cudaDeviceGetAttribute(&sm, cudaDevAttrMultiProcessorCount, device);
    cudaStream_t st = (cudaStream_t)stream;
    if (cudaMemsetAsync(base, 0, COUNTER_BYTES, st) != cudaSuccess)
        return csaw_host_fail(CSAW_ERR_CUDA, "counter reset failed");
    rc = idx64 ? dispatch<int64_t>(dg, p, fan, seeds, base, max_items, out_src, out_dst, out_sample, out_depth,
                                   capacity, sm, st)
               : dispatch<int32_t>(dg, p, fan, seeds, base, max_items, out_src, out_dst, out_sample, out_depth,
                                   capacity, sm, st);
    if (rc) return rc;
    NoAllocCounters h;
    if (cudaMemcpyAsync(&h, base, sizeof(h), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess) {
        cudaGetLastError();
        return csaw_host_fail(CSAW_ERR_CUDA, "counter read-back failed");
    }
    *n_out = (int64_t)h.out_count;
    if (h.err & ERR_SEED_RANGE) return csaw_host_fail(CSAW_ERR_INVALID, "a seed vertex is out of range");
    if (h.err) return csaw_host_fail(CSAW_ERR_DEVICE, "kernel error flag set");
    if ((int64_t)h.out_count > capacity) return csaw_host_fail(CSAW_ERR_CAPACITY, "output capacity too small");
    return 0;
}
