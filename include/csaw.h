/*
 * csaw.h -- C ABI of the csaw-b200 graph sampling / random-walk engine.
 *
 * Drop-in boundary for C-SAW's sampler.  C-SAW's own boundary is
 *   - the compile-time operator plugin api.cuh (non-stream/api.cuh:4-27):
 *     VertexBias / EdgeBias / Update, kept in include/csaw_api.cuh, and
 *   - the host entry Sampler(beg, csr, n_blocks, n_threads, n_subgraph,
 *     FrontierSize, NeighborSize, Depth, args, rank) (non-stream/sampler.cuh:3-8,
 *     non-stream/main.cu:196-308), kept as csaw_sampler_compat() below,
 * plus its CSR input (graph.hpp:9-111: int64 beg_pos/adj files) and its Si
 * edge-list output (sample_class.cuh:76-90).
 *
 * Everything here is plain C: opaque handles, plain pointers and sizes, int
 * status codes (no exit(), unlike HRR/H_ERR in herror.h:1-10 and util.h:4-14).
 * "stream" arguments are cudaStream_t passed as void* (NULL = legacy default
 * stream).  Device pointers are marked "device"; everything else is host.
 * One handle per host thread; calls on one handle are not thread-safe.
 */
#ifndef CSAW_H
#define CSAW_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------- status */
enum {
    CSAW_OK = 0,
    CSAW_ERR_INVALID = 1,   /* bad argument (see csaw_last_error) */
    CSAW_ERR_CUDA = 2,      /* a CUDA runtime call failed */
    CSAW_ERR_CAPACITY = 3,  /* output capacity too small; *n_out = needed */
    CSAW_ERR_NOMEM = 4,     /* device allocation failed */
    CSAW_ERR_DEVICE = 5,    /* a kernel reported an error flag */
    CSAW_PENDING = 6        /* csaw_server_wait: not finished within the timeout */
};

/* ------------------------------------------------------------- modes */
enum {
    CSAW_MODE_NEIGHBOR = 0, /* neighbor sampling, check (main.cu:21-93) */
    CSAW_MODE_WALK = 1,     /* random walk (README.md:30: NeighborSize 1) */
    CSAW_MODE_MDRW = 2      /* multi-dimensional RW, check_layer (main.cu:95-194) */
};

enum {
    CSAW_BIAS_UNBIASED = 0,    /* every neighbor equally likely */
    CSAW_BIAS_DEGREE = 1,      /* bias = out-degree of the neighbor (api.cuh:14-20) */
    CSAW_BIAS_EDGE_WEIGHT = 2, /* bias = weight of the edge */
    CSAW_BIAS_HOOK = 3         /* bias = EdgeBias()/VertexBias() of csaw_api.cuh */
};

enum {
    CSAW_SCHED_PLAIN = 0,    /* one launch per level, degree-threshold rule */
    CSAW_SCHED_BATCHED = 1,  /* per-level passes by item class, CUDA-graph
                                replayed; the one-launch persistent job
                                kernel is CSAW_OPT_PERSISTENT */
    CSAW_SCHED_LEARNED = 2   /* batched + learned granularity */
};

#define CSAW_MAX_DEPTH 64

typedef struct {
    int32_t mode;           /* CSAW_MODE_* */
    int32_t bias;           /* CSAW_BIAS_* */
    int32_t schedule;       /* CSAW_SCHED_* (never changes the output) */
    int32_t n_samples;      /* #samples (n_subgraph) or #walks */
    int32_t frontier_size;  /* FrontierSize: seeds per sample (walk: 1) */
    int32_t neighbor_size;  /* NeighborSize: used for hops whose fanout is 0 */
    int32_t depth;          /* Depth (hops), walk length, or MDRW steps */
    int32_t fanout[CSAW_MAX_DEPTH]; /* per-hop NeighborSize (0 = neighbor_size) */
    uint64_t seed;          /* Philox key: the whole output is a function of it */
    int64_t sample_base;    /* id of the first sample (keys and output ids are
                               sample_base + i), so shards of one job run on
                               several GPUs give exactly the single-GPU output */
    int32_t flags;          /* CSAW_PARAM_* (0: none) */
    int32_t reserved;
} csaw_params;

/* csaw_params.flags */
enum {
    /* Per-sample vertex dedup (neighbor mode; the reference's Ht hash,
     * functions.cuh:929-953, disabled there at :979-981): a vertex is
     * expanded at most once per sample.  Seeds and the children of each
     * level are taken in lineage order; one whose vertex was already taken
     * (a seed, an earlier level's child, or a lower-lineage child of the same
     * level) is not expanded.  Every selected edge is still emitted, so
     * sampled subgraphs keep their edges but each vertex's neighborhood is
     * drawn once (layer-sampling / induced-subgraph style).  Not available in
     * csaw_sample_noalloc or the streaming graph. */
    CSAW_PARAM_DEDUP = 1
};

typedef struct csaw_graph_s *csaw_graph;

/* graph creation flags */
enum {
    CSAW_GRAPH_DEGREE_BIAS = 1,  /* materialise per-edge neighbor degree (4E B) */
    CSAW_GRAPH_CDF_CACHE = 2,    /* per-vertex bias prefix (4E B) for every schedule,
                                    the plain one included */
    CSAW_GRAPH_NO_CDF_CACHE = 4  /* never build the prefix cache.  Without either
                                    flag the batched and learned schedules build it
                                    on first biased use (4.13 E bytes per bias
                                    kind) */
};

typedef struct {
    int64_t n_vertices, n_edges, max_degree;
    int64_t device_bytes;     /* graph residency bytes */
    int64_t workspace_bytes;  /* scratch currently held */
    int64_t kernel_launches;  /* launches since creation */
    int64_t last_edges;       /* edges emitted by the last run */
    int64_t last_items;       /* vertex expansions (or walk steps) of the last run */
    int64_t last_bytes;       /* algorithmic bytes of the last run */
} csaw_stats;

/* Last error message of this thread (never NULL). */
const char *csaw_last_error(void);
/* Library version string. */
const char *csaw_version(void);

/*
 * CSR residency (replaces gpu_graph, non-stream/gpu_graph.cuh:25-66, which
 * built a misindexed per-edge degree list and never loaded weights).
 * rowptr: n_vertices+1 entries, int32 or int64 (rowptr_is_64); col: n_edges
 * int32 in [0, n_vertices); weights: n_edges float >= 0, or NULL.
 * csaw_graph_create copies host arrays to the current device.
 */
int csaw_graph_create(const void *rowptr, int rowptr_is_64, const int32_t *col,
                      const float *weights, int64_t n_vertices, int64_t n_edges,
                      int flags, csaw_graph *out);
int csaw_graph_destroy(csaw_graph g);
int csaw_graph_stats(csaw_graph g, csaw_stats *out);

/*
 * Per-kernel timing (replaces the clock() stamps accumulated into
 * wvar->total_counter, functions.cuh:342-396).  With profiling on, every
 * launch is bracketed by CUDA events on its stream; csaw_graph_kernel_stats
 * returns, per kernel kind, the summed device time, launches, algorithmic
 * bytes and work items since profiling was (re)enabled.
 * Kinds: 0 level expansion (batched: take-all pass), 1 high-degree (CTA)
 * expansion, 2 walk, 3 MDRW, 4 queue/seed/residency setup, 5 batched
 * warp-granularity selection pass, 6 batched hub selection (cached prefix),
 * 7 batched two-items-per-warp selection (cached prefix, N <= 16), 8 walk
 * with one thread per walk (unbiased walks; many biased walks over a cached
 * prefix), 9 persistent job kernel (every level of a batched neighbor job in
 * one launch; its bytes and items are counted under the kinds of the passes
 * it runs), 10 batched thread-per-item selection (N < d <= 32).
 */
int csaw_graph_profile(csaw_graph g, int enable);
int csaw_graph_kernel_stats(csaw_graph g, int kind, double *ms, int64_t *launches,
                            int64_t *bytes, int64_t *items);

/* Seeds uniform over non-isolated vertices (Philox keyed by seed).
 * out: device, n entries. */
int csaw_make_seeds(csaw_graph g, int64_t n, uint64_t seed, int32_t *out, void *stream);

/*
 * Run one sampling job (all three modes).  seeds: device, n_samples *
 * frontier_size vertex ids (walk: n_samples).  Outputs: device arrays of
 * `capacity` entries; out_sample and out_depth may be NULL.  Edge (src, dst)
 * of sample s at hop/step l.  Order within the output is unspecified; the
 * multiset is a pure function of (graph, params, seeds).  Synchronises
 * `stream` and stores the edge count in *n_out.
 */
int csaw_sample(csaw_graph g, const csaw_params *p, const int32_t *seeds,
                int32_t *out_src, int32_t *out_dst, int32_t *out_sample,
                int32_t *out_depth, int64_t capacity, int64_t *n_out, void *stream);

/* Same, with HOST seeds and HOST outputs (copies inside the call; large
 * jobs copy edges back while they still sample, CSAW_OPT_HOST_PARTS).  On
 * an error the host arrays hold an unspecified part of the output. */
int csaw_sample_host(csaw_graph g, const csaw_params *p, const int32_t *seeds,
                     int32_t *out_src, int32_t *out_dst, int32_t *out_sample,
                     int32_t *out_depth, int64_t capacity, int64_t *n_out, void *stream);

/*
 * One job of a batch.  params/seeds/outputs as for csaw_sample (device
 * pointers), or host pointers when host_buffers != 0.  n_out and status are
 * written by the call.
 */
typedef struct {
    const csaw_params *params;
    const int32_t *seeds;
    int32_t *out_src, *out_dst, *out_sample, *out_depth;
    int64_t capacity;
    int64_t n_out;
    int32_t status;
    int32_t host_buffers;
} csaw_job;

/*
 * Runs n_jobs independent jobs together: each on its own stream and device
 * context, forked from and joined back into `stream`, so latency-bound jobs
 * (walks, small frontiers) overlap.  Every job's output equals what
 * csaw_sample would give for it alone.  Returns the first failing status;
 * per-job status in jobs[i].status.
 */
int csaw_sample_batch(csaw_graph g, csaw_job *jobs, int n_jobs, void *stream);

/* Graph options. */
enum {
    /* 1 (default): a batch seen before with the same parameters and buffers
     * is captured once into a CUDA graph and replayed as one launch
     * afterwards (host-buffer jobs too: their copies in and out stay outside
     * the graph, so new seed values in the same arrays are used); at most 64
     * graphs are kept per graph handle.  0: always launch kernel by kernel.
     * Off while profiling is on. */
    CSAW_OPT_CUDA_GRAPHS = 1,
    /* n > 0: the next CSAW_SCHED_LEARNED runs record up to n execution
     * profiles (features, granularity, cycles) with a random valid
     * granularity per item; 0: stop recording. */
    CSAW_OPT_SCHED_RECORD = 2,
    /* Launch shape of the batched kernels (never changes the output):
     * persistent grid size in percent of the occupancy-filled grid
     * (25..400, default 100) ... */
    CSAW_OPT_GRID_PCT = 3,
    /* ... and whether cached items with N <= 16 run two per warp (1, the
     * default) or one per warp (0). */
    CSAW_OPT_PAIR = 4,
    /* Host-buffer jobs (csaw_sample_host, host_buffers != 0) copy edges
     * back while they still sample: the edges of every finished hop, and of
     * every finished part when the job runs as P consecutive sample ranges
     * (1..8); 0 (default): 8 ranges when the job can emit at least 4 Mi
     * edges, 4 from 512 Ki, else 1, and no more than keep 8192 samples in
     * a range (walks: 256 per SM);
     * -1: one range, copied back after all of its sampling.  Never changes
     * the edge multiset. */
    CSAW_OPT_HOST_PARTS = 5,
    /* Bytes of shared memory (0..98304, default 0) the CTA pass that retries
     * cached hub items may use to rebuild a row's prefix: rows whose
     * rebuild fits are done in shared memory, larger ones in global scratch.
     * More shared memory means fewer resident CTAs; never changes the
     * output. */
    CSAW_OPT_RETRY_SMEM = 6,
    /* 1: batched neighbor jobs run all their levels in one persistent
     * cooperative kernel (items pushed for the next level are consumed in
     * the same launch; grid barriers with bounded waits between passes);
     * 0 (default): one launch per pass and level.  Applies to degree-rule
     * jobs over a cached prefix (or unbiased) without dedup, up to 4 levels;
     * others use the per-level launches.  Never changes the output. */
    CSAW_OPT_PERSISTENT = 7,
    /* Thread class of batched biased items with N < d <= 32 (one thread
     * each, the row's prefix in registers, 32 items per warp, instead of a
     * warp each).  1 (default): the degree rule uses it when N <= 16 on
     * levels of at least 65,536 items, and the learned scheduler may pick
     * it; 2: the degree rule uses it for every such item; 0: never.  Never
     * changes the output. */
    CSAW_OPT_THREAD_SELECT = 8,
    /* 1 (default): a CTA retry of a cached hub (more than 512 edges) rebuilds
     * its prefix incrementally from per-tile summaries built with the cache
     * (8 bytes per 32 edges of the hub rows, E/32 + V + 1 slots); 0: every
     * rebuild rescans the whole row.  Never changes the output. */
    CSAW_OPT_INCR_REBUILD = 9
};
int csaw_graph_set_option(csaw_graph g, int option, int64_t value);

/*
 * Autotuner of the launch shape for a recurring batch (the reference fixes
 * n_blocks x n_threads by hand, main.cu:219-224): times the batch under
 * each candidate
 * (per-level launches with grid 50/100/200 % x pairing on/off, and the
 * persistent job kernel with pairing), device-timed, after one untimed run
 * each, and keeps the fastest in the graph's options.  The jobs' outputs are
 * overwritten by the runs (identical under every candidate).
 */
typedef struct {
    int32_t grid_pct, pair;         /* chosen shape */
    double best_ms, default_ms;     /* its time, and the default shape's */
    int32_t candidates;
    int32_t persistent;             /* chosen: 1 = persistent job kernel */
} csaw_tune_result;
int csaw_graph_autotune(csaw_graph g, csaw_job *jobs, int n_jobs, void *stream, csaw_tune_result *out);

/*
 * Learned execution-granularity scheduler (CSAW_SCHED_LEARNED).  Replaces
 * the reference's fixed warp-per-vertex schedule (main.cu:60-91); it never
 * changes the output.  An MLP 8 -> 32 -> 32 -> 7 predicts, per item that
 * needs draws, the latency of seven granularities (class 0 warp in
 * registers, 1 warp in shared memory, 2-5 CTA of 128/256/512/1024 threads,
 * 6 one thread, for d <= 32 in batched jobs with CSAW_OPT_THREAD_SELECT on);
 * without a trained model the degree rule is used (0 / 1 / CTA-256 by degree,
 * 6 for d <= 32 with N <= 16 on levels of at least 65,536 items).
 * csaw_sched_train fits it on the GPU (FP32 forward and backward kernels,
 * full-batch Adam) to the recorded profiles; csaw_mlp_grad_host exposes the
 * mean loss and gradient for checking.
 * Parameter layout: W1[32][8] b1[32] W2[32][32] b2[32] W3[7][32] b3[7]
 * (1575 floats); norm: x mean[8], x std[8], y mean, y std (18 floats).
 * Profile record: float x[8], int32 class, float cycles (40 bytes).
 */
int csaw_sched_info(csaw_graph g, int64_t *n_records, int *trained, float *last_loss);
int csaw_sched_get_records(csaw_graph g, void *out, int64_t max_n, int64_t *n);
int csaw_sched_train(csaw_graph g, int epochs, float lr, uint64_t seed, float *final_loss);
/* Classes a trained model may pick (bit c for class c).  Training keeps the
 * warp classes 0 and 1 and the CTA classes and thread class the model picks
 * on its own training records; only those CTA widths are launched (plus
 * CTA-256 for hubs above 512 edges without a cached prefix).  0x7f when
 * untrained.  A trained (or loaded) model that routes items to CTA classes or
 * the thread class is then on trial: the
 * next learned biased neighbor jobs alternate between its routing and the
 * degree rule, timed on the device, three runs each; if its mean time is not
 * lower it is not used and the mask reads 0x3 (the degree rule).  Output is
 * the same under either arm. */
int csaw_sched_classes(csaw_graph g, uint32_t *mask);
int csaw_sched_get_model(csaw_graph g, float *params, float *norm);
int csaw_sched_set_model(csaw_graph g, const float *params, const float *norm);
int csaw_mlp_grad_host(const float *params, const float *norm, const void *records, int n,
                       float *grad, float *loss);

/*
 * Neighbor sampling that allocates no device memory.  No counterpart in the
 * reference.  For callers that must not call cudaMalloc while sampling: a
 * serving loop whose memory budget was reserved at start-up, a host thread
 * that must not stall on the device synchronisation cudaMalloc/cudaFree can
 * cause, code running inside another framework's memory pool.  Same
 * arguments and output as csaw_sample (device seeds and outputs, plain
 * schedule, mode CSAW_MODE_NEIGHBOR only); the frontier queues and counters
 * live in one fixed 32 MiB device array per GPU, held until process exit.
 * Rejects, with CSAW_ERR_INVALID and before any GPU work, jobs whose largest
 * frontier level exceeds 1398090 items, and biased jobs on graphs with a
 * vertex of degree above 1024.  All calls on a device share the array:
 * calls whose GPU work overlaps race -- serialise them.  The first call on
 * a device looks up the array's address and, with CUDA's lazy module
 * loading, may be the point where the library's device code is loaded and
 * the 32 MiB array reserved: make that first call during set-up, before any
 * stream capture.  The schedule field of p is ignored (the plain level loop
 * always runs; its output equals every schedule's).
 */
int csaw_sample_noalloc(csaw_graph g, const csaw_params *p, const int32_t *seeds,
                        int32_t *out_src, int32_t *out_dst, int32_t *out_sample,
                        int32_t *out_depth, int64_t capacity, int64_t *n_out, void *stream);

/*
 * Streaming (partitioned) sampling for graphs whose adjacency exceeds the
 * device budget (replaces streaming/streaming_sampling.cu:427-728).  The row
 * offsets are copied to the device; col (and weights) stay in the caller's
 * host arrays, page-locked in place, and are paged in as partitions of
 * 2^partition_bits vertices into as many device slots as slot_budget_bytes
 * allows (at least 2).  The host arrays must outlive the handle.
 * csaw_stream_sample runs neighbor sampling or walks (MDRW is not offered;
 * walk Depth <= 64) and gives exactly the csaw_sample output.
 */
typedef struct csaw_stream_graph_s *csaw_stream_graph;
typedef struct {
    int64_t n_partitions, n_slots;
    int64_t partition_loads;   /* partitions copied to the device */
    int64_t partition_hits;    /* partition uses served by a resident slot */
    int64_t bytes_h2d;         /* adjacency bytes copied */
    int64_t kernel_launches;
    int64_t host_pinned_in_place; /* bit 0: col, bit 1: weights registered */
    int64_t items_read_in_place;  /* pending items served from host memory (CSAW_STREAM_OPT_READ_IN_PLACE) */
} csaw_stream_info;
int csaw_stream_graph_create(const void *rowptr, int rowptr_is_64, const int32_t *col,
                             const float *weights, int64_t n_vertices, int64_t n_edges,
                             int partition_bits, int64_t slot_budget_bytes,
                             csaw_stream_graph *out);
int csaw_stream_graph_destroy(csaw_stream_graph g);
int csaw_stream_sample(csaw_stream_graph g, const csaw_params *p, const int32_t *seeds,
                       int32_t *out_src, int32_t *out_dst, int32_t *out_sample,
                       int32_t *out_depth, int64_t capacity, int64_t *n_out, void *stream);
int csaw_stream_stats(csaw_stream_graph g, csaw_stream_info *out);
/* Options of a streaming graph.  CSAW_STREAM_OPT_READ_IN_PLACE, 1 (default):
 * when the host arrays a job reads are page-locked and mapped, partitions
 * that are not in the device arena are read in place from host memory by
 * the kernels (only the prefix lines and columns a hop touches cross the
 * link), every round processes every pending item, and free arena space
 * takes the partitions with the most pending items per byte without
 * evicting any; 0: partitions are copied in before use and evicted when
 * the budget is full (sweeps).  Output unchanged.  No counterpart in the
 * reference, which copies fixed partitions (streaming_sampling.cu:597-714). */
enum { CSAW_STREAM_OPT_READ_IN_PLACE = 1 };
int csaw_stream_graph_set_option(csaw_stream_graph g, int option, int64_t value);
/* Builds the per-vertex prefix cache of a bias kind (DEGREE, EDGE_WEIGHT or
 * HOOK) for a streaming graph: every row's canonical prefix in page-locked
 * host memory (4 E bytes) and its two index levels on the device (4.13 E/32
 * bytes); later jobs with that bias stream each partition's prefix in place
 * of its weights and search it instead of recomputing a row's prefix per
 * expansion (raw weights, for the rare rebuild after repeated collisions,
 * are read from the page-locked host array).  The in-memory cache's
 * streamed-partition counterpart (SURVEY's Cp, functions.cuh:329-341);
 * output unchanged.  Edge-weight and hook biases need the weights
 * page-locked in place (csaw_stream_info.host_pinned_in_place bit 1). */
int csaw_stream_graph_cache(csaw_stream_graph g, int bias);

/*
 * Request loop (continuous batching).  The reference runs one synchronous
 * Sampler() call per process (non-stream/main.cu:196-308, caller
 * mpi_main.cpp:40); a server instead keeps the graph resident and serves a
 * stream of independent requests.  A worker thread admits queued requests
 * while a slot (a job context with its own stream) is free and the request's
 * device bytes (seeds + outputs sized by its edge bound) fit the device
 * budget; admitted requests run concurrently on
 * the device, and each result is copied into the caller's host buffers (a
 * direct asynchronous copy when they are page-locked).  Queued requests are
 * admitted first-fit in arrival order; one waiting longer than
 * max_wait_us (0: 2000 us) blocks later ones until it fits.  A request's
 * output depends only on its params and seeds, never on what else runs.
 * Latency = submit to result in host memory.  While a server exists, its
 * graph must not be used by other calls; submit/wait/stats are thread-safe.
 */
typedef struct csaw_server_s *csaw_server;
typedef struct {
    int32_t n_slots;        /* concurrent requests on the device (1..64) */
    int32_t max_wait_us;    /* head-of-line bound for first-fit admission */
    int64_t device_budget;  /* bytes for in-flight request seeds and outputs */
} csaw_server_config;
typedef struct {
    int64_t submitted, completed, failed;
    int64_t queued, in_flight;
    int64_t edges;                 /* edges returned by completed requests */
    int64_t peak_device_bytes;     /* of the budget, at most */
    int64_t workspace_bytes;       /* job contexts' scratch */
    double p50_ms, p90_ms, p99_ms, max_ms, mean_ms;   /* completed since reset */
    double p99_queue_ms;           /* submit -> admitted */
    double p99_launch_ms;          /* admitted -> kernels enqueued (host) */
    double p99_gpu_ms;             /* enqueued -> edge count read back */
    double first_submit_s, last_done_s;               /* steady clock, seconds */
    double max_worker_call_ms;     /* longest single launch or completion step of the
                                      worker thread since reset: a host-side stall
                                      (a blocking CUDA call) shows here */
    int64_t worker_calls_over_1ms; /* such steps longer than 1 ms since reset */
} csaw_server_stats;
int csaw_server_create(csaw_graph g, const csaw_server_config *cfg, csaw_server *out);
/* Waits for every submitted request, then frees the server. */
int csaw_server_destroy(csaw_server s);
/* Copies params and seeds (host; seed count as csaw_sample: n_samples x
 * frontier_size, or n_samples walks); outputs are host buffers of `capacity`
 * edges each (out_sample / out_depth may be NULL) that must stay valid until
 * the request is waited for.  Fails at once (CSAW_ERR_CAPACITY) if the
 * request alone exceeds the device budget. */
int csaw_server_submit(csaw_server s, const csaw_params *p, const int32_t *seeds, int32_t *out_src,
                       int32_t *out_dst, int32_t *out_sample, int32_t *out_depth, int64_t capacity,
                       uint64_t *ticket);
/* Waits up to timeout_us (< 0: forever) for the request; returns its status
 * (CSAW_PENDING if still running, the ticket stays valid), its edge count
 * and latency.  A finished ticket is released by the call that reports it. */
int csaw_server_wait(csaw_server s, uint64_t ticket, int64_t timeout_us, int64_t *n_out, double *latency_ms);
/* Counters and latency percentiles; reset != 0 clears the latency record. */
int csaw_server_get_stats(csaw_server s, int reset, csaw_server_stats *out);

/*
 * Reference-compatible entry (Sampler, non-stream/main.cu:196-308): loads
 * int64 beg.bin / csr.bin (graph.hpp:18-34 format), draws FrontierSize seeds
 * per sample, runs neighbor sampling (FrontierSize == 1) or MDRW
 * (FrontierSize > 1) exactly as the reference dispatches (main.cu:281-288),
 * and returns the number of sampled edges and the sampling time in seconds.
 * n_blocks and n_threads are accepted and ignored (the engine sizes its own
 * grids).  The edge list stays inside the call, as in the reference.
 */
int csaw_sampler_compat(const char *beg_file, const char *csr_file, int n_blocks,
                        int n_threads, int n_subgraph, int frontier_size,
                        int neighbor_size, int depth, int *sampled_edges,
                        double *seconds);

#ifdef __cplusplus
}
#endif
#endif
