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
