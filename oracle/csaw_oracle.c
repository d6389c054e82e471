/*
 * csaw_oracle.c -- CPU oracle (test infrastructure only; see csaw_oracle.h).
 *
 * Build with -ffp-contract=off and without -ffast-math: every float result
 * below is one IEEE-754 round-to-nearest add, multiply or max, in a fixed
 * order that the CUDA kernels reproduce.
 *
 * Specification restated here (the CUDA kernels implement the same thing):
 *
 * RNG.  Philox4x32-10 keyed by (seed lo, seed hi).  The word for neighbor
 * selection of (sample s, depth l, lineage item p, slot j, attempt a) is
 * word (a & 3) of the block at counter
 *     { p, s, (1 << 24) | l, (j << 16) | (a >> 2) }.
 * Walk step t of walk w is neighbor sampling with N = 1, so it uses
 * (s = w, l = t, p = 0, j = 0, a = 0).  MDRW step t of sample s uses words 0
 * and 1 of the block at { 0, s, (2 << 24) | t, 0 }.  Seed i uses word 0 of
 * { i, 0, 3 << 24, 0 }.
 *   unit(x)   = (x >> 8) * 2^-24                     (exact, in [0, 1))
 *   mulhi(x,n)= (x * n) >> 32 in 64-bit integers     (uniform in [0, n))
 *
 * Canonical prefix of w[0..d) (replaces the reference's in-place Blelloch
 * scan, functions.cuh:112-176, whose int temporaries truncate FP32 biases):
 *   tile t = elements [32t, 32t+32), zero padded; Kogge-Stone inclusive scan
 *   inside the tile (offsets 1,2,4,8,16; v[l] = v[l] + v_prev[l-off]);
 *   tile totals S_t; group g = tiles [32g, 32g+32): Kogge-Stone scan of the
 *   group's tile totals gives Q, exclusive Qex_t (0 for the group's first
 *   tile); group carry C_0 = 0, C_{g+1} = C_g + Q_last(g) (serial);
 *   P_i = C_g + (Qex_t + v_i); finally a running max (P_i = max(P_{i-1},P_i))
 *   makes P monotone.  T = P_{d-1}.
 *
 * Inverse-transform search (replaces binary_search, functions.cuh:11-43):
 *   t = unit(x) * T; if !(t < T) t = the float just below T;
 *   result = first i with P_i > t.  That index always has positive weight.
 *
 * Selection of k = min(N, d) distinct neighbors of one item (replaces
 * heur_normalize, functions.cuh:743-868, and the bitmap collision test,
 * :45-70).  If d <= N every neighbor is taken in adjacency order.  Otherwise
 * slots j = 0..N-1 are filled in order.  State: the selected list S, an
 * excluded set Z (initially empty) and the prefix P of the weights with the
 * members of Z set to 0.  Slot j loops:
 *     biased and T == 0, or 16 draws used by this slot: take the smallest
 *         index not in S (zero-mass fill / draw cap; the cap only guards
 *         termination against 1-ulp intervals a zeroed neighbor can keep at a
 *         tile boundary);
 *     after R = 4 rejected draws in the current phase: Z = S, rebuild P
 *         (a new phase; its first draw cannot collide);
 *     draw word (s, l, p, j, A_j++); biased: index = search(P, unit*T);
 *         unbiased: index = the mulhi(x, d - |Z|)-th index not in Z;
 *     accept if the index is not in S.
 * This is successive sampling without replacement (rejection against the
 * renormalised remainder is exact), bounded at R + 1 draws per slot, and the
 * result depends only on the keys, never on the GPU schedule.
 *
 * Neighbor sampling (check, main.cu:21-93; frontier, functions.cuh:971-1011):
 * depth-0 items are the F seeds of a sample with lineage f; an item (v, p) at
 * depth l < D emits (v, col[beg+idx]) for each selected idx in slot order
 * (Update() is the identity), and if l + 1 < D pushes the child with lineage
 * p * N_l + j.
 *
 * MDRW (check_layer, main.cu:95-194): per step, pick a frontier slot by
 * inverse transform over VertexBias (degree, or 1 when unbiased) of the F
 * frontier vertices (slot 0 when F == 1 or all biases are 0); if the picked
 * vertex has degree 0 the step emits nothing; else a uniform neighbor
 * (mulhi) replaces it and one edge is emitted (rand_integer, functions.cuh:
 * 210-216).
 */
#include "csaw_oracle.h"

#include <pthread.h>
#include <stdlib.h>
#include <string.h>

#define TAG_SAMPLE 1u
#define TAG_MDRW 2u
#define TAG_SEED 3u
#define REJECT_ATTEMPTS 4
#define MAX_SLOT_DRAWS 16

/* ---------------------------------------------------------------- Philox */

void oracle_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
    uint32_t k0 = key[0], k1 = key[1];
    for (int r = 0; r < 10; ++r) {
        uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        c0 = hi1 ^ c1 ^ k0;
        c1 = lo1;
        c2 = hi0 ^ c3 ^ k1;
        c3 = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

static uint32_t sample_word(uint64_t seed, uint32_t s, uint32_t l, uint32_t p,
                            uint32_t j, uint32_t a) {
    uint32_t c[4] = {p, s, (TAG_SAMPLE << 24) | l, (j << 16) | (a >> 2)};
    uint32_t k[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    uint32_t o[4];
    oracle_philox4x32_10(c, k, o);
    return o[a & 3];
}

static float unit24(uint32_t x) { return (float)(x >> 8) * 0x1p-24f; }

static uint32_t mulhi(uint32_t x, uint32_t n) {
    return (uint32_t)(((uint64_t)x * (uint64_t)n) >> 32);
}

static float float_below(float T) {
    uint32_t b;
    memcpy(&b, &T, 4);
    b -= 1u;
    float r;
    memcpy(&r, &b, 4);
    return r;
}

/* ------------------------------------------------------ canonical prefix */

static void ks32(float *a) {
    for (int off = 1; off < 32; off <<= 1) {
        float prev[32];
        memcpy(prev, a, sizeof(prev));
        for (int l = off; l < 32; ++l) a[l] = prev[l] + prev[l - off];
    }
}

void oracle_canon_prefix(const float *w, int64_t d, float *P) {
    if (d <= 0) return;
    int64_t ntiles = (d + 31) / 32;
    float *tsum = (float *)malloc(sizeof(float) * (size_t)ntiles);
    for (int64_t t = 0; t < ntiles; ++t) {
        float a[32];
        for (int l = 0; l < 32; ++l) {
            int64_t i = 32 * t + l;
            a[l] = i < d ? w[i] : 0.0f;
        }
        ks32(a);
        for (int l = 0; l < 32; ++l) {
            int64_t i = 32 * t + l;
            if (i < d) P[i] = a[l];
        }
        tsum[t] = a[31];
    }
    int64_t ngroups = (ntiles + 31) / 32;
    float C = 0.0f;
    for (int64_t g = 0; g < ngroups; ++g) {
        float q[32];
        for (int l = 0; l < 32; ++l) {
            int64_t t = 32 * g + l;
            q[l] = t < ntiles ? tsum[t] : 0.0f;
        }
        ks32(q);
        for (int l = 0; l < 32; ++l) {
            int64_t t = 32 * g + l;
            if (t >= ntiles) break;
            float qex = l ? q[l - 1] : 0.0f;
            for (int m = 0; m < 32; ++m) {
                int64_t i = 32 * t + m;
                if (i >= d) break;
                P[i] = C + (qex + P[i]);
            }
        }
        C = C + q[31];
    }
    float mx = P[0];
    for (int64_t i = 1; i < d; ++i) {
        if (P[i] < mx) P[i] = mx;
        mx = P[i];
    }
    free(tsum);
}

static int64_t search_upper(const float *P, int64_t d, float t) {
    int64_t lo = 0, hi = d - 1;
    while (lo < hi) {
        int64_t mid = (lo + hi) >> 1;
        if (P[mid] > t) hi = mid; else lo = mid + 1;
    }
    return lo;
}

static float its_target(uint32_t x, float T) {
    float t = unit24(x) * T;
    if (!(t < T)) t = float_below(T);
    return t;
}

/* ----------------------------------------------------------- selection */

typedef struct {
    const int64_t *rowptr;
    const int32_t *col;
    const float *weight;
    int64_t V;
    int bias;
    uint64_t seed;
    float *wbuf;      /* scratch, max degree */
    float *pbuf;      /* scratch, max degree */
} ctx_t;

static float edge_bias(const ctx_t *c, int64_t e) {
    if (c->bias == ORACLE_EDGE_WEIGHT) return c->weight[e];
    int32_t u = c->col[e];
    return (float)(c->rowptr[u + 1] - c->rowptr[u]);
}

static int in_list(const int64_t *a, int n, int64_t x) {
    for (int i = 0; i < n; ++i)
        if (a[i] == x) return 1;
    return 0;
}

static int cmp_i64(const void *a, const void *b) {
    int64_t x = *(const int64_t *)a, y = *(const int64_t *)b;
    return (x > y) - (x < y);
}

/* prefix of the biases of [beg, beg+d) with the sorted indices Z zeroed */
static float build_prefix(ctx_t *c, int64_t beg, int64_t d, const int64_t *Z, int nZ) {
    int zi = 0;
    for (int64_t i = 0; i < d; ++i) {
        float w = edge_bias(c, beg + i);
        if (zi < nZ && Z[zi] == i) { w = 0.0f; ++zi; }
        c->wbuf[i] = w;
    }
    oracle_canon_prefix(c->wbuf, d, c->pbuf);
    return c->pbuf[d - 1];
}

/* returns k, fills sel[0..k) with neighbor offsets in slot order */
static int select_item(ctx_t *c, int64_t beg, int64_t d, int N, uint32_t s,
                       uint32_t l, uint32_t p, int64_t *sel) {
    if (d <= N) {
        for (int64_t j = 0; j < d; ++j) sel[j] = j;
        return (int)d;
    }
    const int biased = c->bias != ORACLE_UNBIASED;
    int64_t Z[1024];
    int nZ = 0, nS = 0;
    float T = 0.0f;
    if (biased) T = build_prefix(c, beg, d, NULL, 0);
    for (int j = 0; j < N; ++j) {
        uint32_t A = 0;
        int a = 0;
        int64_t idx;
        for (;;) {
            if ((biased && !(T > 0.0f)) || A == MAX_SLOT_DRAWS) {
                idx = 0;
                while (in_list(sel, nS, idx)) ++idx;
                break;
            }
            if (a == REJECT_ATTEMPTS) {
                memcpy(Z, sel, sizeof(int64_t) * (size_t)nS);
                nZ = nS;
                qsort(Z, (size_t)nZ, sizeof(int64_t), cmp_i64);
                if (biased) T = build_prefix(c, beg, d, Z, nZ);
                a = 0;
                continue;
            }
            uint32_t x = sample_word(c->seed, s, l, p, (uint32_t)j, A);
            ++A;
            ++a;
            if (biased) {
                idx = search_upper(c->pbuf, d, its_target(x, T));
            } else {
                int64_t t = mulhi(x, (uint32_t)(d - nZ));
                for (int z = 0; z < nZ; ++z)
                    if (Z[z] <= t) ++t;
                idx = t;
            }
            if (!in_list(sel, nS, idx)) break;
        }
        sel[nS++] = idx;
    }
    return nS;
}

/* ------------------------------------------------------------- output */

typedef struct {
    int32_t *src, *dst, *smp, *dep;
    int64_t n, cap;
} ebuf_t;

static void emit(ebuf_t *b, int32_t u, int32_t v, int32_t s, int32_t l) {
    if (b->n == b->cap) {
        int64_t nc = b->cap ? 2 * b->cap : 1024;
        b->src = (int32_t *)realloc(b->src, sizeof(int32_t) * (size_t)nc);
        b->dst = (int32_t *)realloc(b->dst, sizeof(int32_t) * (size_t)nc);
        b->smp = (int32_t *)realloc(b->smp, sizeof(int32_t) * (size_t)nc);
        b->dep = (int32_t *)realloc(b->dep, sizeof(int32_t) * (size_t)nc);
        b->cap = nc;
    }
    b->src[b->n] = u; b->dst[b->n] = v; b->smp[b->n] = s; b->dep[b->n] = l;
    b->n++;
}

/* ------------------------------------------------------------- modes */

typedef struct {
    const oracle_params *p;
    const int32_t *seeds;
    ctx_t c;
    int s0, s1;
    ebuf_t out;
    int status;
} job_t;

/* Set of vertex ids (open addressing, linear probing, grows at 1/2 load). */
typedef struct {
    int32_t *slot;
    int64_t cap, n;
} vset_t;

static int vset_insert(vset_t *h, int32_t v) {   /* 1 if newly inserted */
    if (2 * (h->n + 1) > h->cap) {
        int64_t oc = h->cap, nc = oc ? 2 * oc : 64;
        int32_t *old = h->slot;
        h->slot = (int32_t *)malloc(sizeof(int32_t) * (size_t)nc);
        for (int64_t i = 0; i < nc; ++i) h->slot[i] = -1;
        h->cap = nc;
        h->n = 0;
        for (int64_t i = 0; i < oc; ++i)
            if (old[i] >= 0) vset_insert(h, old[i]);
        free(old);
    }
    uint64_t i = ((uint64_t)(uint32_t)v * 0x9E3779B97F4A7C15ull) & (uint64_t)(h->cap - 1);
    while (h->slot[i] >= 0) {
        if (h->slot[i] == v) return 0;
        i = (i + 1) & (uint64_t)(h->cap - 1);
    }
    h->slot[i] = v;
    h->n++;
    return 1;
}

/* Keeps the items of (v, p) whose vertex is new to the set, in order. */
static int64_t dedup_items(vset_t *h, int32_t *v, uint32_t *p, int64_t n) {
    int64_t k = 0;
    for (int64_t i = 0; i < n; ++i)
        if (vset_insert(h, v[i])) {
            v[k] = v[i];
            p[k] = p[i];
            ++k;
        }
    return k;
}

static void run_neighbor(job_t *jb, int sl) {
    const oracle_params *p = jb->p;
    const int s = (int)(p->sample_base + sl);
    ctx_t *c = &jb->c;
    int64_t cap = 64, n = 0;
    int32_t *cv = (int32_t *)malloc(sizeof(int32_t) * (size_t)cap);
    uint32_t *cp = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)cap);
    for (int f = 0; f < p->frontier_size; ++f) {
        if (n == cap) {
            cap *= 2;
            cv = (int32_t *)realloc(cv, sizeof(int32_t) * (size_t)cap);
            cp = (uint32_t *)realloc(cp, sizeof(uint32_t) * (size_t)cap);
        }
        cv[n] = jb->seeds[(int64_t)sl * p->frontier_size + f];
        cp[n] = (uint32_t)f;
        ++n;
    }
    const int dedup = (p->flags & ORACLE_DEDUP) != 0;
    vset_t seen = {NULL, 0, 0};
    if (dedup) n = dedup_items(&seen, cv, cp, n);
    int64_t sel[1024];
    for (int l = 0; l < p->depth; ++l) {
        int N = p->fanout[l];
        int push = l + 1 < p->depth;
        int64_t ncap = 64, nn = 0;
        int32_t *nv = (int32_t *)malloc(sizeof(int32_t) * (size_t)ncap);
        uint32_t *np = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)ncap);
        for (int64_t it = 0; it < n; ++it) {
            int32_t v = cv[it];
            int64_t beg = c->rowptr[v], d = c->rowptr[v + 1] - beg;
            if (d <= 0) continue;
            int k = select_item(c, beg, d, N, (uint32_t)s, (uint32_t)l, cp[it], sel);
            for (int j = 0; j < k; ++j) {
                int32_t u = c->col[beg + sel[j]];
                emit(&jb->out, v, u, s, l);
                if (push) {
                    if (nn == ncap) {
                        ncap *= 2;
                        nv = (int32_t *)realloc(nv, sizeof(int32_t) * (size_t)ncap);
                        np = (uint32_t *)realloc(np, sizeof(uint32_t) * (size_t)ncap);
                    }
                    nv[nn] = u;
                    np[nn] = cp[it] * (uint32_t)N + (uint32_t)j;
                    ++nn;
                }
            }
        }
        free(cv); free(cp);
        if (dedup) nn = dedup_items(&seen, nv, np, nn);
        cv = nv; cp = np; n = nn; cap = ncap;
    }
    free(cv); free(cp);
    free(seen.slot);
}

static void run_walk(job_t *jb, int sl) {
    const oracle_params *p = jb->p;
    ctx_t *c = &jb->c;
    const int s = (int)(p->sample_base + sl);
    int32_t v = jb->seeds[sl];
    int64_t sel[1];
    for (int t = 0; t < p->depth; ++t) {
        int64_t beg = c->rowptr[v], d = c->rowptr[v + 1] - beg;
        if (d <= 0) break;
        select_item(c, beg, d, 1, (uint32_t)s, (uint32_t)t, 0u, sel);
        int32_t u = c->col[beg + sel[0]];
        emit(&jb->out, v, u, s, t);
        v = u;
    }
}

static void run_mdrw(job_t *jb, int sl) {
    const oracle_params *p = jb->p;
    const int s = (int)(p->sample_base + sl);
    ctx_t *c = &jb->c;
    int F = p->frontier_size;
    int32_t *f = (int32_t *)malloc(sizeof(int32_t) * (size_t)F);
    float *b = (float *)malloc(sizeof(float) * (size_t)F);
    float *P = (float *)malloc(sizeof(float) * (size_t)F);
    memcpy(f, jb->seeds + (int64_t)sl * F, sizeof(int32_t) * (size_t)F);
    uint32_t key[2] = {(uint32_t)c->seed, (uint32_t)(c->seed >> 32)};
    for (int t = 0; t < p->depth; ++t) {
        for (int i = 0; i < F; ++i)
            b[i] = c->bias == ORACLE_UNBIASED
                       ? 1.0f
                       : (float)(c->rowptr[f[i] + 1] - c->rowptr[f[i]]);
        uint32_t ctr[4] = {0u, (uint32_t)s, (TAG_MDRW << 24) | (uint32_t)t, 0u}, o[4];
        oracle_philox4x32_10(ctr, key, o);
        int slot = 0;
        if (F > 1) {
            oracle_canon_prefix(b, F, P);
            float T = P[F - 1];
            if (T > 0.0f) slot = (int)search_upper(P, F, its_target(o[0], T));
        }
        int32_t v = f[slot];
        int64_t beg = c->rowptr[v], d = c->rowptr[v + 1] - beg;
        if (d <= 0) continue;
        int32_t u = c->col[beg + mulhi(o[1], (uint32_t)d)];
        emit(&jb->out, v, u, s, t);
        f[slot] = u;
    }
    free(f); free(b); free(P);
}

static void *job_main(void *arg) {
    job_t *jb = (job_t *)arg;
    for (int s = jb->s0; s < jb->s1; ++s) {
        switch (jb->p->mode) {
            case ORACLE_NEIGHBOR: run_neighbor(jb, s); break;
            case ORACLE_WALK: run_walk(jb, s); break;
            default: run_mdrw(jb, s); break;
        }
    }
    return NULL;
}

int oracle_make_seeds(const int64_t *rowptr, int64_t V, int64_t n, uint64_t seed, int32_t *out) {
    int64_t nl = 0;
    for (int64_t v = 0; v < V; ++v) nl += rowptr[v + 1] > rowptr[v];
    if (nl == 0 || nl > 0xFFFFFFFFll) return 1;
    int32_t *L = (int32_t *)malloc(sizeof(int32_t) * (size_t)nl);
    int64_t m = 0;
    for (int64_t v = 0; v < V; ++v)
        if (rowptr[v + 1] > rowptr[v]) L[m++] = (int32_t)v;
    uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    for (int64_t i = 0; i < n; ++i) {
        uint32_t ctr[4] = {(uint32_t)i, (uint32_t)(i >> 32), TAG_SEED << 24, 0u}, o[4];
        oracle_philox4x32_10(ctr, key, o);
        out[i] = L[mulhi(o[0], (uint32_t)nl)];
    }
    free(L);
    return 0;
}

int oracle_run(const int64_t *rowptr, const int32_t *col, const float *weight,
               int64_t V, int64_t E, const oracle_params *p, const int32_t *seeds,
               int32_t *src, int32_t *dst, int32_t *sample, int32_t *depth,
               int64_t cap, int64_t *n_out, int n_threads) {
    (void)E;
    if (!p || !rowptr || !col || !seeds || !n_out || p->n_samples < 0 || p->sample_base < 0 ||
        p->depth < 0 || p->depth > ORACLE_MAX_DEPTH || p->frontier_size < 1)
        return 1;
    if (p->bias == ORACLE_EDGE_WEIGHT && !weight) return 1;
    if (p->mode == ORACLE_MDRW && p->bias == ORACLE_EDGE_WEIGHT) return 1;
    int per = p->mode == ORACLE_WALK ? 1 : p->frontier_size;
    for (int64_t i = 0; i < (int64_t)p->n_samples * per; ++i)
        if (seeds[i] < 0 || seeds[i] >= V) return 1;
    if (p->mode == ORACLE_NEIGHBOR)
        for (int l = 0; l < p->depth; ++l)
            if (p->fanout[l] < 1 || p->fanout[l] > 1024) return 1;
    int64_t maxdeg = 1;
    for (int64_t v = 0; v < V; ++v)
        if (rowptr[v + 1] - rowptr[v] > maxdeg) maxdeg = rowptr[v + 1] - rowptr[v];
    if (n_threads < 1) n_threads = 1;
    if (n_threads > p->n_samples) n_threads = p->n_samples > 0 ? p->n_samples : 1;
    job_t *jobs = (job_t *)calloc((size_t)n_threads, sizeof(job_t));
    pthread_t *th = (pthread_t *)calloc((size_t)n_threads, sizeof(pthread_t));
    for (int t = 0; t < n_threads; ++t) {
        job_t *jb = &jobs[t];
        jb->p = p;
        jb->seeds = seeds;
        jb->c.rowptr = rowptr; jb->c.col = col; jb->c.weight = weight;
        jb->c.V = V; jb->c.bias = p->bias; jb->c.seed = p->seed;
        jb->c.wbuf = (float *)malloc(sizeof(float) * (size_t)maxdeg);
        jb->c.pbuf = (float *)malloc(sizeof(float) * (size_t)maxdeg);
        jb->s0 = (int)((int64_t)p->n_samples * t / n_threads);
        jb->s1 = (int)((int64_t)p->n_samples * (t + 1) / n_threads);
        if (n_threads == 1) job_main(jb);
        else pthread_create(&th[t], NULL, job_main, jb);
    }
    int64_t total = 0;
    for (int t = 0; t < n_threads; ++t) {
        if (n_threads > 1) pthread_join(th[t], NULL);
        total += jobs[t].out.n;
    }
    int rc = 0;
    *n_out = total;
    if (total > cap) {
        rc = 3;
    } else {
        int64_t o = 0;
        for (int t = 0; t < n_threads; ++t) {
            ebuf_t *b = &jobs[t].out;
            size_t nb = sizeof(int32_t) * (size_t)b->n;
            if (b->n) {
                memcpy(src + o, b->src, nb);
                memcpy(dst + o, b->dst, nb);
                if (sample) memcpy(sample + o, b->smp, nb);
                if (depth) memcpy(depth + o, b->dep, nb);
            }
            o += b->n;
        }
    }
    for (int t = 0; t < n_threads; ++t) {
        free(jobs[t].c.wbuf); free(jobs[t].c.pbuf);
        free(jobs[t].out.src); free(jobs[t].out.dst);
        free(jobs[t].out.smp); free(jobs[t].out.dep);
    }
    free(jobs); free(th);
    return rc;
}
