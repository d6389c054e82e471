// csaw_host.h -- host-side helpers shared between the library's translation
// units (not part of the C ABI).
#pragma once

#include "csaw.h"
#include "csaw_device.cuh"

// Sets the thread's error message and returns code.
int csaw_host_fail(int code, const char *msg);

// Validates p for g, fills the per-hop fanouts and the plain-schedule device
// view of g (no lazily built per-edge arrays), its max degree, device ordinal
// and rowptr width.
int csaw_host_plain_view(csaw_graph g, const csaw_params *p, int fan[CSAW_MAX_DEPTH], csaw::DevGraph *view,
                         int64_t *maxdeg, int *device, int *idx64);

// Device ordinal of g (-1 for NULL).
int csaw_host_graph_device(csaw_graph g);

// Validates p for g; the largest number of edges it can emit and its seed count.
int csaw_host_edge_bound(csaw_graph g, const csaw_params *p, int64_t *bound, int64_t *n_seeds);

// A job context of its own (counters, queues, scratch, a non-blocking stream):
// jobs on different contexts run concurrently.  Workspace grows on demand.
int csaw_host_job_create(csaw_graph g, void **job, cudaStream_t *stream);
void csaw_host_job_destroy(void *job);
int64_t csaw_host_job_workspace(const void *job);

// Enqueues a run on the context's stream (no host synchronisation), device
// seeds and outputs; the counter block is read back asynchronously.  After
// the stream has passed that point, finish gives the edge count and status.
int csaw_host_job_enqueue(csaw_graph g, void *job, const csaw_params *p, const int32_t *seeds, int32_t *src,
                          int32_t *dst, int32_t *smp, int32_t *dep, int64_t cap);
int csaw_host_job_finish(csaw_graph g, void *job, int64_t cap, int64_t *n_out);
