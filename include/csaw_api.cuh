/*
 * csaw_api.cuh -- user operator hooks (compile-time plugin).
 *
 * Same three hooks, same names and same roles as C-SAW's api.cuh
 * (non-stream/api.cuh:4-27):
 *   VertexBias(v)            bias of frontier vertex v (MDRW slot choice)
 *   EdgeBias(u)              bias of neighbor u (neighbor sampling, walks)
 *   Update(G, selected, src) vertex recorded and expanded for a selection
 * They are used when csaw_params.bias == CSAW_BIAS_HOOK; Update is always
 * applied.  Edit this file and rebuild the library, as with the reference
 * (README.md:26 "Define the required API in API.cuh").
 *
 * Differences from the reference, on purpose:
 *   - biases return float (the reference returns int, a subset);
 *   - EdgeBias also receives the edge index, so edge-weight biased hooks can
 *     read g->weight[edge] (the reference never loads weights,
 *     graph.hpp:76-108);
 *   - degree() is the real out-degree (the reference's degree_list is indexed
 *     by edge, gpu_graph.cuh:44-60, but read by vertex).
 * Biases must be finite and >= 0.  Update must return a vertex in
 * [0, n_vertices).
 */
#ifndef CSAW_API_CUH
#define CSAW_API_CUH

#include <stdint.h>

struct csaw_graph_view {
    const void *rowptr;
    int rowptr_is_64;
    const int32_t *col;
    const float *weight;
    int64_t n_vertices, n_edges;

    __device__ __forceinline__ int64_t begin(int v) const {
        return rowptr_is_64 ? ((const int64_t *)rowptr)[v] : (int64_t)((const int32_t *)rowptr)[v];
    }
    __device__ __forceinline__ int64_t degree(int v) const { return begin(v + 1) - begin(v); }
};

/* MDRW: pick frontier vertices in proportion to their degree. */
__device__ __forceinline__ float VertexBias(int vertex, const csaw_graph_view *g) {
    return (float)g->degree(vertex);
}

/* Biased neighbor sampling (BNS) / layer sampling: neighbor degree. */
__device__ __forceinline__ float EdgeBias(int vertex, int64_t edge, const csaw_graph_view *g) {
    (void)edge;
    return (float)g->degree(vertex);
}

/* Identity: record and expand the selected vertex itself. */
__device__ __forceinline__ int Update(const csaw_graph_view *g, int selected, int source) {
    (void)g;
    (void)source;
    return selected;
}

#endif
