/*
 * csaw_oracle.h -- CPU oracle for the csaw-b200 sampler.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product library links, loads or
 * calls this code.  Only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg use it, to check or to time against.
 *
 * PARITY UNPINNED against the reference: C-SAW ships no tests, no golden
 * vectors and no known-answer data (its only example graph, web-Google, is not
 * in the repository), and its sampling path is __device__ code driven by
 * cuRAND XORWOW, so it cannot run on a CPU.  What IS pinned:
 *   - philox4x32_10() against cuRAND's host Philox4_32_10 generator (an
 *     independent implementation), see tests/golden/make_philox_golden.py;
 *   - the sampling semantics against committed golden edge lists produced by
 *     this oracle (regression), and distributionally (chi-square) against the
 *     ideal normalised bias.
 *
 * The semantics restated here follow C-SAW's operator surface:
 *   neighbor sampling  non-stream/main.cu:21-93 (check), functions.cuh:743-868
 *                      (heur_normalize), :971-1011 (frontier)
 *   random walk        README.md:30 (NeighborSize=1, Depth=walk length)
 *   MDRW               non-stream/main.cu:95-194 (check_layer),
 *                      functions.cuh:1014-1060 (ITS_MDRW), :210-216
 * with the build's own deterministic RNG keying (Philox counters keyed by
 * sample, depth, lineage item, slot and attempt) in place of per-thread
 * cuRAND state, and the reference bugs (misindexed degree_list, int scan
 * temporaries, copy-first-N past the list) not reproduced.
 */
#ifndef CSAW_ORACLE_H
#define CSAW_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORACLE_MAX_DEPTH 128

enum { ORACLE_NEIGHBOR = 0, ORACLE_WALK = 1, ORACLE_MDRW = 2 };
enum { ORACLE_UNBIASED = 0, ORACLE_DEGREE = 1, ORACLE_EDGE_WEIGHT = 2 };

typedef struct {
    int32_t mode;           /* ORACLE_NEIGHBOR / WALK / MDRW */
    int32_t bias;           /* ORACLE_UNBIASED / DEGREE / EDGE_WEIGHT */
    int32_t n_samples;      /* samples (or walks) */
    int32_t frontier_size;  /* seeds per sample (F) */
    int32_t depth;          /* hops (neighbor), walk length, MDRW steps */
    int32_t fanout[ORACLE_MAX_DEPTH]; /* N per hop (neighbor mode) */
    uint64_t seed;          /* Philox key */
    int64_t sample_base;    /* id of the first sample (keys and output ids) */
    int32_t flags;          /* ORACLE_DEDUP: per-sample vertex dedup */
} oracle_params;

/* Per-sample vertex dedup (neighbor mode): a vertex is expanded at most once
 * per sample.  Seeds and pushed children are taken in lineage order; one whose
 * vertex was already taken (an earlier seed, an earlier level's child, or a
 * lower-lineage child of the same level) is not expanded.  Every selected
 * edge is still emitted. */
#define ORACLE_DEDUP 1

/* Philox4x32-10 (Salmon et al., SC11). */
void oracle_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);

/* Canonical inclusive prefix of w[0..d) (see csaw_oracle.c for the order). */
void oracle_canon_prefix(const float *w, int64_t d, float *P);

/* Seeds: n draws uniform over the non-isolated vertices. */
int oracle_make_seeds(const int64_t *rowptr, int64_t V, int64_t n, uint64_t seed, int32_t *out);

/* Run one sampling job.  Output is sample-major, then level by level, items
 * in lineage order, slots in selection order.  Any output pointer except src
 * and dst may be NULL.  Returns 0, or 3 if cap is too small (n_out then holds
 * the needed count), or 1 on invalid arguments. */
int oracle_run(const int64_t *rowptr, const int32_t *col, const float *weight,
               int64_t V, int64_t E, const oracle_params *p, const int32_t *seeds,
               int32_t *src, int32_t *dst, int32_t *sample, int32_t *depth,
               int64_t cap, int64_t *n_out, int n_threads);

#ifdef __cplusplus
}
#endif
#endif
