// csaw_internal.h -- constants and launch-argument structs shared by the
// csaw-b200 kernels and their host driver.
//
// Output semantics (the CPU oracle restates them in plain C):
//
// RNG.  Philox4x32-10 keyed by (seed lo, seed hi).  Neighbor selection of
// (sample s, depth l, lineage item p, slot j, draw A) uses word (A & 3) of the
// block at counter {p, s, (TAG_SAMPLE << 24) | l, (j << 16) | (A >> 2)}.  A
// walk is neighbor sampling with N = 1.  MDRW step t of sample s uses words 0
// and 1 of {0, s, (TAG_MDRW << 24) | t, 0}; seed i uses word 0 of
// {i lo, i hi, TAG_SEED << 24, 0}.  Because the counter names the work item and
// never the thread, the output does not depend on the schedule.
//
// Canonical prefix of d biases: Kogge-Stone scans over 32-element tiles,
// Kogge-Stone over the tile totals of each 32-tile group, serial carry across
// groups, P_i = C_g + (Qex_t + v_i), then a running max.  Inverse transform:
// t = unit24(x) * T (kept below T), index = first i with P_i > t.
//
// Selection without replacement (k = min(N, d)): d <= N takes every neighbor;
// otherwise slots 0..N-1 in order draw until the index is new; after
// REJECT_ATTEMPTS rejected draws in one phase the selected set is zeroed out of
// the prefix (unbiased: excluded from the index range) and a new phase starts;
// with no positive mass left, remaining slots take the smallest unselected
// indices, and a slot that has used MAX_SLOT_DRAWS draws takes the smallest
// unselected index (termination guard).
#pragma once

#include <cstdint>

namespace csaw {

constexpr uint32_t TAG_SAMPLE = 1u;
constexpr uint32_t TAG_MDRW = 2u;
constexpr uint32_t TAG_SEED = 3u;
constexpr int REJECT_ATTEMPTS = 4;
constexpr int MAX_SLOT_DRAWS = 16;     // termination guard per slot
// A pair item of up to RESUME_MAX_DEG edges whose first phase fails keeps
// that phase's end state (the failing slot j, then the accepted indices of
// slots < j, as 16-bit values) in its consumed 48-byte pair entry; larger
// ones replay the phase.  (32-bit indices for larger hubs, N <= 11, measured
// neutral on the scale-25 step: 22.998 vs 22.986 ms.)
constexpr int RESUME_MAX_DEG = 65535;

constexpr int MAX_FANOUT = 32;      // slots are lanes of one warp
constexpr int WBUF = 1024;          // prefix held in shared memory per warp
constexpr int EXPAND_THREADS = 256; // 8 warps per CTA
constexpr int HEAVY_THREADS = 256;
constexpr int WALK_THREADS = 256;

// A frontier item whose output and next-queue slots are already reserved
// (batched schedules): item index in the input queue, first queue slot,
// first output slot, and a copy of the item (vertex, sample, lineage, degree,
// row begin) so the consumer needs a single load.
struct SelEntry {
    uint32_t it;
    uint32_t q;
    unsigned long long ob;
    int32_t v;
    int32_t s;
    uint32_t p;
    int32_t d;
    long long beg;
    int32_t cls;      // execution granularity chosen for the item
    int32_t pad;
};

struct SchedArgs;

// One level of neighbor sampling: input queue -> output edges + next queue.
struct LevelArgs {
    const int32_t *in_v;
    const int32_t *in_s;
    const uint32_t *in_p;
    const uint32_t *n_in;     // device count of input items
    int32_t *out_v;
    int32_t *out_s;
    uint32_t *out_p;
    uint32_t *n_out;          // device count of next-level items
    const void *in_beg;       // batched queues: row begin (I) and degree of
    const int32_t *in_deg;    //   each item, or null (then read rowptr)
    void *out_beg;
    int32_t *out_deg;
    uint32_t *heavy;          // deferred item indices (biased, d > WBUF)
    uint32_t *n_heavy;
    SelEntry *sel_list;       // batched: warp-granularity items (d > N)
    uint32_t *n_sel;
    SelEntry *heavy_list;     // batched: CTA-granularity items (count n_heavy)
    SelEntry *cta_list[4];    // batched: items per CTA class (128/256/512/1024)
    uint32_t *n_cta;          //   and their counts
    int cta_class;            // class of the CTA launch (0..3), for profiles
    const uint8_t *sched_tab; // learned (trained): the level's decision table
    SelEntry *hub_list;       // batched: items above WF searching a cached prefix
    uint32_t *n_hub;
    SelEntry *pair_list;      // batched: cached items run two per warp (N <= 16, d >= 3N)
    uint32_t *n_pair;
    SelEntry *refill_list;    // batched: paired items redone by a whole warp (the warp list's buffer)
    uint32_t *n_refill;
    SelEntry *retry_list;     // batched: cached hubs the warp pass handed back
    uint32_t *n_retry;
    SelEntry *thread_list;    // batched: thread-class items (N < d <= 32), a thread each, or null
    uint32_t *n_thread;
    int thread_force;         // the degree rule sends every N < d <= 32 item to the thread list
    const SchedArgs *sched;   // learned scheduler, or null (degree rule)
    float *heavy_scratch;     // per-CTA scratch for the heavy kernel
    int64_t heavy_stride;     // floats per CTA
    int64_t heavy_smem;       // floats of dynamic shared memory the heavy launch has (0: none)
    int32_t *o_src, *o_dst, *o_smp, *o_dep;
    unsigned long long *o_count;
    int64_t cap;
    unsigned long long *bytes; // algorithmic bytes accumulator
    unsigned long long *items; // expanded-items accumulator
    int *err;
    uint32_t k0, k1;
    int depth, N, push;
    // Mixed-depth input (streaming): each item's depth in in_dep, its fanout
    // fan[depth], children pushed while depth + 1 < D with their depth in
    // out_dep.  Null in_dep: every item is at `depth` with N and push.
    const int32_t *in_dep;
    int32_t *out_dep;
    int D;
    uint8_t fan[CSAW_MAX_DEPTH];
    // Streaming, one launch over all pending items: per partition (vertex >>
    // pbits) the column and weight bases re-based so that col[e] is edge e,
    // or a null column base when the partition is not sampled this round
    // (its items stay pending).
    const int32_t *const *part_col;
    const float *const *part_w;
    int pbits;
    // Streaming with a prefix cache: part_w holds each partition's canonical
    // prefix (re-based like part_col), the two index levels are resident for
    // the whole graph, and raw biases (a rebuild) are read from the
    // page-locked host weights.
    int part_cdf;
    const float *cdf1_all, *cdf2_all;
    const float *host_w;
};

// Level of input item `it`: depth, fanout, whether its children are pushed.
__host__ __device__ __forceinline__ void item_level(const LevelArgs &a, uint32_t it, int &l, int &N, bool &push) {
    if (a.in_dep) {
        l = a.in_dep[it];
        N = a.fan[l];
        push = l + 1 < a.D;
    } else {
        l = a.depth;
        N = a.N;
        push = a.push != 0;
    }
}

struct WalkArgs {
    const int32_t *seeds;
    int n;                    // walks (or samples for MDRW)
    int len;                  // steps
    int F;                    // MDRW frontier size
    int base;                 // id of the first walk / sample
    int32_t *o_src, *o_dst, *o_smp, *o_dep;
    unsigned long long *o_count;
    int64_t cap;
    float *scratch;           // per-warp prefix scratch for d > WBUF (walks)
    int64_t scratch_stride;
    unsigned long long *bytes;
    unsigned long long *items;
    int *err;
    uint32_t k0, k1;
};

enum : int { ERR_SEED_RANGE = 1, ERR_UPDATE_RANGE = 2, ERR_SCRATCH = 4, ERR_COPY_WAIT = 8, ERR_BARRIER = 16 };

}  // namespace csaw
