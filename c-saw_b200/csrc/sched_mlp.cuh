// sched_mlp.cuh -- learned execution-granularity scheduler (sm_100a).
//
// For every frontier item that needs draws (d > N, biased), the batched
// expansion can run it at one of seven granularities:
//   0 warp, registers (d <= 32)      1 warp, shared memory (d <= WF)
//   2 CTA of 128 threads            3 CTA of 256     4 CTA of 512     5 CTA of 1024
//   6 one thread (d <= 32, the row's prefix in its registers; 32 items a warp)
// The choice never changes the output (every draw is keyed by the work item),
// only the time.  The degree rule picks 0 / 1 / 3, and 6 for d <= 32 when
// N <= 16 and the level is large (rule_class).  The learned rule runs a small
// MLP (8 -> 32 -> 32 -> 7, ReLU, 1575 parameters) on per-item features and
// predicts each class's latency (normalised log2 cycles); the class chosen
// minimises predicted latency x (1 + u (width - 1)), width in warps (1/32 for
// a thread), where u in [0, 1] grows with the level's size relative to the
// warp slots: a small frontier leaves warps idle, so wide CTAs cost little and
// narrow threads gain little; a large one is throughput-bound, so width is
// weighed in.
//
// Features (all cheap per item): log2 d, log2 N, log2(d/N), coefficient of
// variation of the neighbor biases, collision estimate N * sum p_i^2 (both
// from per-vertex statistics built once per graph), log2 of level items per
// warp slot, depth, bias kind.
//
// The network is trained on the GPU on profiles the sampler records: in
// recording mode every drawn item gets a uniformly random valid class, and
// the consumer kernel writes (features, class, clock64 cycles).  Training is
// full-batch Adam on the squared error of the recorded class's output,
// FP32 forward and backward kernels written here; inference uses BF16
// weights held in shared memory.
#pragma once

#include <cuda_bf16.h>

#include "csaw_device.cuh"

namespace csaw {

constexpr int MLP_IN = 8, MLP_H = 32, MLP_OUT = 7;
constexpr int MLP_W1 = 0;                              // [32][8]
constexpr int MLP_B1 = MLP_W1 + MLP_H * MLP_IN;        // [32]
constexpr int MLP_W2 = MLP_B1 + MLP_H;                 // [32][32]
constexpr int MLP_B2 = MLP_W2 + MLP_H * MLP_H;         // [32]
constexpr int MLP_W3 = MLP_B2 + MLP_H;                 // [7][32]
constexpr int MLP_B3 = MLP_W3 + MLP_OUT * MLP_H;       // [7]
constexpr int MLP_NPARAM = MLP_B3 + MLP_OUT;           // 1575
constexpr int MLP_NORM = 2 * MLP_IN + 2;               // x mean/std, y mean/std
constexpr int N_CLASSES = 7;
constexpr int CLS_THREAD = 6;
constexpr uint32_t CLS_CTA_MASK = 0x3cu;   // classes 2..5
// The degree rule's thread class: levels of at least this many items (fewer
// leave most warps idle when 32 items share one), at most this many draws
// per item (a thread runs its slots one after another).
constexpr uint32_t THREAD_RULE_MIN_ITEMS = 1u << 16;
constexpr int THREAD_RULE_MAX_N = 16;

enum : int { SCHED_THRESHOLD = 0, SCHED_MLP = 1, SCHED_RECORD = 2 };

struct ProfRec {
    float x[MLP_IN];
    int cls;
    float cycles;
};

struct SchedArgs {
    int mode;                      // SCHED_THRESHOLD / SCHED_MLP / SCHED_RECORD
    const __nv_bfloat16 *wq;       // MLP_NPARAM bf16 weights (SCHED_MLP)
    const float *norm;             // MLP_NORM floats
    const float2 *vstats;          // per vertex: (CoV of biases, sum p^2)
    ProfRec *rec;                  // SCHED_RECORD: profile records
    uint32_t *n_rec;
    uint32_t max_rec;
    int bias_kind;
    int warp_slots;                // resident warps of the selection kernel
    uint32_t class_mask;           // SCHED_MLP: classes the model may pick (bit c)
};

// Width of a class in warps.
__device__ __forceinline__ float class_width(int c) {
    return c == CLS_THREAD ? 1.f / 32.f : (c <= 1 ? 1.f : (float)(4 << (c - 2)));
}

// Item features (shared by the router and the profile recorders).
__device__ __forceinline__ void item_features(float x[MLP_IN], int64_t d, int N, float2 st, uint32_t n_level,
                                              int depth, int bias_kind, int warp_slots) {
    x[0] = __log2f((float)d);
    x[1] = __log2f((float)N);
    x[2] = __log2f((float)d / (float)N);
    x[3] = st.x;
    x[4] = fminf(8.f, (float)N * st.y);
    x[5] = __log2f(1.f + (float)n_level / (float)warp_slots);
    x[6] = (float)depth;
    x[7] = (float)bias_kind;
}

// Valid classes for degree d (bit c set if class c can run the item).
// One-tile rows (d <= 32) run in a warp's registers or in one thread (thr:
// the job has a thread list; batched, biased, not disabled): wider classes
// only idle more lanes on them.  Longer rows run at warp or CTA width; with
// the per-vertex prefix cache, class 1 (one warp) also takes items above wf:
// it searches the cached prefix instead of building one in shared memory.
__device__ __forceinline__ unsigned valid_classes(int64_t d, int wf, bool cached, bool thr) {
    if (d <= 32) return thr ? 0x41u : 0x1u;
    unsigned m = CLS_CTA_MASK;       // CTAs always
    if (d <= wf || cached) m |= 0x2u;
    return m;
}

__device__ __forceinline__ int threshold_class(int64_t d, int wf, bool cached) {
    return d <= 32 ? 0 : ((d <= wf || cached) ? 1 : 3);
}

// The degree rule with the thread class: one-tile rows with few draws, on
// large levels, run a thread each (every one-tile row when forced).
__device__ __forceinline__ int rule_class(int64_t d, int N, uint32_t n_level, int wf, bool cached, bool thr,
                                          bool force = false) {
    if (thr && d <= 32 && (force || (N <= THREAD_RULE_MAX_N && n_level >= THREAD_RULE_MIN_ITEMS))) return CLS_THREAD;
    return threshold_class(d, wf, cached);
}

// Warp-cooperative MLP inference for one item (warp-uniform x); returns the
// predicted normalised log2 latency of class `lane` on lanes 0..6.
// W: the bf16 weights (3 KB, read through the read-only cache).
__device__ __forceinline__ float mlp_infer(const __nv_bfloat16 *W, const float *norm, const float x[MLP_IN], int lane) {
    float h = __bfloat162float(__ldg(W + MLP_B1 + lane));
#pragma unroll
    for (int k = 0; k < MLP_IN; ++k) {
        const float xn = (x[k] - __ldg(norm + k)) * __frcp_rn(__ldg(norm + MLP_IN + k));
        h = fmaf(__bfloat162float(__ldg(W + MLP_W1 + lane * MLP_IN + k)), xn, h);
    }
    h = fmaxf(h, 0.f);
    float h2 = __bfloat162float(__ldg(W + MLP_B2 + lane));
#pragma unroll 8
    for (int i = 0; i < MLP_H; ++i)
        h2 = fmaf(__bfloat162float(__ldg(W + MLP_W2 + lane * MLP_H + i)), __shfl_sync(FULL, h, i), h2);
    h2 = fmaxf(h2, 0.f);
    const int o = lane < MLP_OUT ? lane : 0;
    float y = __bfloat162float(__ldg(W + MLP_B3 + o));
#pragma unroll 8
    for (int i = 0; i < MLP_H; ++i)
        y = fmaf(__bfloat162float(__ldg(W + MLP_W3 + o * MLP_H + i)), __shfl_sync(FULL, h2, i), y);
    return y;
}

// Cheapest class among `valid` from the predicted normalised log2 latency y
// of class `lane` (lanes 0..6), or -1 when `valid` is empty.
__device__ __forceinline__ int class_argmin(float y, const float *norm, uint32_t n_level, int warp_slots,
                                            unsigned valid, int lane) {
    const float u = fminf(1.f, (float)n_level / (16.f * (float)warp_slots));
    // predicted latency in cycles (up to the common scale), weighted by width
    float cost = exp2f(y * norm[2 * MLP_IN + 1] + norm[2 * MLP_IN]) *
                 (1.f + u * (class_width(lane < MLP_OUT ? lane : 0) - 1.f));
    if (lane >= MLP_OUT || !((valid >> lane) & 1u)) cost = __int_as_float(0x7f800000);   // +inf
    // argmin over lanes 0..7 (ties: lowest class)
    int best = lane;
#pragma unroll
    for (int off = 4; off; off >>= 1) {
        const float oc = __shfl_down_sync(FULL, cost, off);
        const int ob = __shfl_down_sync(FULL, best, off);
        if (oc < cost || (oc == cost && ob < best)) {
            cost = oc;
            best = ob;
        }
    }
    best = __shfl_sync(FULL, best, 0);
    return (valid >> best) & 1u ? best : -1;
}

// Class for one drawn biased item (warp-uniform inputs; all lanes call).
__device__ __forceinline__ int choose_class(const SchedArgs *sa, const __nv_bfloat16 *W, int64_t d, int N, float2 st,
                                            uint32_t n_level, int depth, uint32_t hash, int wf, bool cached,
                                            bool thr, int lane) {
    const unsigned valid = valid_classes(d, wf, cached, thr);
    if (!sa || sa->mode == SCHED_THRESHOLD) return rule_class(d, N, n_level, wf, cached, thr);
    if (sa->mode == SCHED_RECORD) {
        const int nv = __popc(valid);
        int pick = (int)(hash % (uint32_t)nv);
        unsigned m = valid;
        for (; pick > 0; --pick) m &= m - 1;
        return __ffs(m) - 1;
    }
    float x[MLP_IN];
    item_features(x, d, N, st, n_level, depth, sa->bias_kind, sa->warp_slots);
    const float y = mlp_infer(W, sa->norm, x, lane);
    const int best = class_argmin(y, sa->norm, n_level, sa->warp_slots, valid & sa->class_mask, lane);
    return best >= 0 ? best : rule_class(d, N, n_level, wf, cached, thr);
}

// ------------------------------------------------------- decision table
// Per level, the model is evaluated once per cell of a grid over the three
// per-item features that vary within a level (degree: steps of 4 up to 32,
// then log2 d in half steps from 5; CoV in half steps; N sum p^2 in unit
// steps; the level's N, size, depth and bias fixed), and the expansion kernel
// routes each item by one table load.  Each cell holds two picks: over the
// classes valid for an item a warp can run (0 and the thread for d <= 32; 1
// and the CTAs above) and over the CTA classes 2..5 (255: none allowed).
constexpr int TAB_SMALL = 8;   // degree bins of d <= 32
constexpr int TAB_D = 40, TAB_C = 8, TAB_P = 8, TAB_N = TAB_D * TAB_C * TAB_P;

__device__ __forceinline__ int tab_degree_bin(int64_t d) {
    if (d <= 32) return (int)((d - 1) >> 2);
    return min(TAB_D - 1, TAB_SMALL + max(0, (int)((__log2f((float)d) - 5.f) * 2.f)));
}

__device__ __forceinline__ int tab_index(int64_t d, float2 st, int N) {
    const int bd = tab_degree_bin(d);
    const int bc = min(TAB_C - 1, max(0, (int)(st.x * 2.f)));
    const int bp = min(TAB_P - 1, max(0, (int)fminf(8.f, (float)N * st.y)));
    return (bd * TAB_C + bc) * TAB_P + bp;
}

// Class of a drawn item from the level's table (built with the same thr).
__device__ __forceinline__ int table_class(const uint8_t *tab, int64_t d, float2 st, int N, int wf, bool cached) {
    const bool warp_ok = cached || d <= wf;
    const int c = tab[2 * tab_index(d, st, N) + (warp_ok ? 0 : 1)];
    return c < N_CLASSES ? c : threshold_class(d, wf, cached);
}

// One warp per cell; n_level read on the device (the level's item count).
// thr: the level has a thread list.
static __global__ void k_sched_table(const SchedArgs *sa, const uint32_t *n_in, int N, int depth, int thr,
                                     uint8_t *tab) {
    const int lane = threadIdx.x & 31;
    const int cell = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (cell >= TAB_N) return;
    const int bp = cell % TAB_P, bc = (cell / TAB_P) % TAB_C, bd = cell / (TAB_P * TAB_C);
    const uint32_t n_level = *n_in;
    const bool small = bd < TAB_SMALL;
    const float ld = small ? __log2f(4.f * (float)bd + 2.5f) : 5.f + ((float)(bd - TAB_SMALL) + 0.5f) * 0.5f;
    const float lN = __log2f((float)N);
    float x[MLP_IN];
    x[0] = ld;
    x[1] = lN;
    x[2] = ld - lN;
    x[3] = ((float)bc + 0.5f) * 0.5f;
    x[4] = (float)bp + 0.5f;
    x[5] = __log2f(1.f + (float)n_level / (float)sa->warp_slots);
    x[6] = (float)depth;
    x[7] = (float)sa->bias_kind;
    const float y = mlp_infer(sa->wq, sa->norm, x, lane);
    // a small cell's degree d may be below N: such items take all their
    // neighbors and are never routed, so the cell's pick does not matter
    const unsigned va = small ? (thr ? 0x41u : 0x1u) : 0x3eu;
    const int a = class_argmin(y, sa->norm, n_level, sa->warp_slots, sa->class_mask & va, lane);
    const int b = class_argmin(y, sa->norm, n_level, sa->warp_slots, sa->class_mask & CLS_CTA_MASK, lane);
    if (lane == 0) {
        tab[2 * cell] = (uint8_t)(a < 0 ? 255 : a);
        tab[2 * cell + 1] = (uint8_t)(b < 0 ? 255 : b);
    }
}

// Classes the trained model picks on its own training records (both with and
// without a prefix cache): classes it never picks are not launched.
static __global__ void k_sched_pick(const ProfRec *rec, int n, const __nv_bfloat16 *W, const float *norm, int warp_slots,
                                    int wf, uint32_t *mask) {
    const int lane = threadIdx.x & 31;
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
    for (int i = gw; i < n; i += nw) {
        const float *x = rec[i].x;
        const int64_t d = (int64_t)(exp2f(x[0]) + 0.5f);
        const uint32_t n_level = (uint32_t)((exp2f(x[5]) - 1.f) * (float)warp_slots + 0.5f);
        const float y = mlp_infer(W, norm, x, lane);
        const int a = class_argmin(y, norm, n_level, warp_slots, valid_classes(d, wf, false, true), lane);
        const int b = class_argmin(y, norm, n_level, warp_slots, valid_classes(d, wf, true, true), lane);
        if (lane == 0) {
            if (a >= 0) atomicOr(mask, 1u << a);
            if (b >= 0) atomicOr(mask, 1u << b);
        }
    }
}

// Appends one profile record (recording mode).
__device__ __forceinline__ void record_profile(const SchedArgs *sa, int64_t d, int N, float2 st, uint32_t n_level,
                                               int depth, int cls, long long cycles) {
    if (!sa || sa->mode != SCHED_RECORD) return;
    const uint32_t i = atomicAdd(sa->n_rec, 1u);
    if (i >= sa->max_rec) return;
    ProfRec r;
    item_features(r.x, d, N, st, n_level, depth, sa->bias_kind, sa->warp_slots);
    r.cls = cls;
    r.cycles = (float)cycles;
    sa->rec[i] = r;
}

// --------------------------------------------------------- vertex stats
// Per vertex: coefficient of variation of its neighbor biases and sum p_i^2
// (p_i = normalised bias), one warp per vertex.
template <typename I, int BIAS>
__global__ void k_vertex_stats(DevGraph g, float2 *out) {
    const int lane = threadIdx.x & 31;
    const int64_t gw = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t v = gw; v < g.v.n_vertices; v += nw) {
        const int64_t beg = row_begin<I>(g, v), d = row_begin<I>(g, v + 1) - beg;
        float s1 = 0.f, s2 = 0.f;
        for (int64_t i = lane; i < d; i += 32) {
            const float w = edge_bias<I, BIAS>(g, beg + i);
            s1 += w;
            s2 += w * w;
        }
#pragma unroll
        for (int off = 16; off; off >>= 1) {
            s1 += __shfl_xor_sync(FULL, s1, off);
            s2 += __shfl_xor_sync(FULL, s2, off);
        }
        if (lane == 0) {
            float cov = 0.f, p2 = d > 0 ? 1.f / (float)d : 0.f;
            if (d > 1 && s1 > 0.f) {
                const float r = (float)d * s2 / (s1 * s1) - 1.f;
                cov = sqrtf(fmaxf(r, 0.f));
                p2 = s2 / (s1 * s1);
            }
            out[v] = make_float2(cov, p2);
        }
    }
}

// ------------------------------------------------------------ training
// Forward and backward of one record (FP32); accumulates dL/dtheta into g.
// Loss: 0.5 * (y[cls] - t)^2 with normalised inputs and target.
__device__ __forceinline__ float mlp_fwd_bwd(const float *w, const float *norm, const ProfRec &r, float *grad) {
    float xn[MLP_IN], h1[MLP_H], h2[MLP_H];
#pragma unroll
    for (int k = 0; k < MLP_IN; ++k) xn[k] = (r.x[k] - norm[k]) / norm[MLP_IN + k];
    for (int j = 0; j < MLP_H; ++j) {
        float a = w[MLP_B1 + j];
#pragma unroll
        for (int k = 0; k < MLP_IN; ++k) a += w[MLP_W1 + j * MLP_IN + k] * xn[k];
        h1[j] = fmaxf(a, 0.f);
    }
    for (int j = 0; j < MLP_H; ++j) {
        float a = w[MLP_B2 + j];
        for (int i = 0; i < MLP_H; ++i) a += w[MLP_W2 + j * MLP_H + i] * h1[i];
        h2[j] = fmaxf(a, 0.f);
    }
    const int c = r.cls;
    float y = w[MLP_B3 + c];
    for (int i = 0; i < MLP_H; ++i) y += w[MLP_W3 + c * MLP_H + i] * h2[i];
    const float t = (__log2f(fmaxf(r.cycles, 1.f)) - norm[2 * MLP_IN]) / norm[2 * MLP_IN + 1];
    const float e = y - t;
    // backward
    atomicAdd(&grad[MLP_B3 + c], e);
    float dh2[MLP_H];
    for (int i = 0; i < MLP_H; ++i) {
        atomicAdd(&grad[MLP_W3 + c * MLP_H + i], e * h2[i]);
        dh2[i] = h2[i] > 0.f ? e * w[MLP_W3 + c * MLP_H + i] : 0.f;
    }
    float dh1[MLP_H];
    for (int i = 0; i < MLP_H; ++i) dh1[i] = 0.f;
    for (int j = 0; j < MLP_H; ++j) {
        if (dh2[j] == 0.f) continue;
        atomicAdd(&grad[MLP_B2 + j], dh2[j]);
        for (int i = 0; i < MLP_H; ++i) {
            atomicAdd(&grad[MLP_W2 + j * MLP_H + i], dh2[j] * h1[i]);
            dh1[i] += dh2[j] * w[MLP_W2 + j * MLP_H + i];
        }
    }
    for (int j = 0; j < MLP_H; ++j) {
        if (!(h1[j] > 0.f) || dh1[j] == 0.f) continue;
        atomicAdd(&grad[MLP_B1 + j], dh1[j]);
#pragma unroll
        for (int k = 0; k < MLP_IN; ++k) atomicAdd(&grad[MLP_W1 + j * MLP_IN + k], dh1[j] * xn[k]);
    }
    return 0.5f * e * e;
}

// Mean loss and gradient over n records (one CTA of MLP_GRAD_THREADS
// threads; gradients accumulate in shared memory).
constexpr int MLP_GRAD_THREADS = 256;

// Summed loss and gradient over n records, accumulated into grad_sum /
// loss_sum (zeroed by the caller): every CTA sums its records in shared
// memory, then adds its partial sums to the global buffers.
static __global__ void __launch_bounds__(MLP_GRAD_THREADS)
k_mlp_grad(const float *w, const float *norm, const ProfRec *rec, int n, float *grad_sum, float *loss_sum) {
    __shared__ float sw[MLP_NPARAM], sg[MLP_NPARAM], sloss;
    for (int i = threadIdx.x; i < MLP_NPARAM; i += blockDim.x) {
        sw[i] = w[i];
        sg[i] = 0.f;
    }
    if (threadIdx.x == 0) sloss = 0.f;
    __syncthreads();
    float l = 0.f;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        l += mlp_fwd_bwd(sw, norm, rec[i], sg);
    atomicAdd(&sloss, l);
    __syncthreads();
    for (int i = threadIdx.x; i < MLP_NPARAM; i += blockDim.x)
        if (sg[i] != 0.f) atomicAdd(&grad_sum[i], sg[i]);
    if (threadIdx.x == 0) atomicAdd(loss_sum, sloss);
}

// Adam step on the FP32 master weights (one thread per parameter).
static __global__ void k_mlp_adam(float *w, const float *grad_sum, float *m, float *v, float lr, int step, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= MLP_NPARAM) return;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    const float g = grad_sum[i] / (float)n;
    m[i] = b1 * m[i] + (1.f - b1) * g;
    v[i] = b2 * v[i] + (1.f - b2) * g * g;
    const float mh = m[i] / (1.f - powf(b1, (float)step));
    const float vh = v[i] / (1.f - powf(b2, (float)step));
    w[i] -= lr * mh / (sqrtf(vh) + eps);
}

static __global__ void k_mlp_to_bf16(const float *w, __nv_bfloat16 *wq) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < MLP_NPARAM) wq[i] = __float2bfloat16_rn(w[i]);
}

// Feature / target normalisation from the records (one CTA).
static __global__ void k_mlp_norm(const ProfRec *rec, int n, float *norm) {
    __shared__ float s1[MLP_IN + 1], s2[MLP_IN + 1];
    if (threadIdx.x <= MLP_IN) {
        s1[threadIdx.x] = 0.f;
        s2[threadIdx.x] = 0.f;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        for (int k = 0; k < MLP_IN; ++k) {
            atomicAdd(&s1[k], rec[i].x[k]);
            atomicAdd(&s2[k], rec[i].x[k] * rec[i].x[k]);
        }
        const float t = __log2f(fmaxf(rec[i].cycles, 1.f));
        atomicAdd(&s1[MLP_IN], t);
        atomicAdd(&s2[MLP_IN], t * t);
    }
    __syncthreads();
    if (threadIdx.x <= MLP_IN && n > 0) {
        const float mean = s1[threadIdx.x] / n;
        const float sd = sqrtf(fmaxf(s2[threadIdx.x] / n - mean * mean, 0.f));
        const float s = sd > 1e-3f ? sd : 1.f;
        if (threadIdx.x < MLP_IN) {
            norm[threadIdx.x] = mean;
            norm[MLP_IN + threadIdx.x] = s;
        } else {
            norm[2 * MLP_IN] = mean;
            norm[2 * MLP_IN + 1] = s;
        }
    }
}

}  // namespace csaw
