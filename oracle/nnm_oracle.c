/* Test infrastructure only -- see nnm_oracle.h.  A plain-C restatement of
 * the reference hot path; file:line citations are into the reference's
 * src/ directory.  It is the parity checker for the CUDA product and is never
 * linked into it. */
#include "nnm_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------ */
/* Distances (vmath.cpp:56-88, distopt.cpp:82-114, distopt.cpp:165-184).
 * One float accumulator, strictly sequential, every operation rounded to
 * float (built with -ffp-contract=off). */
float nno_dist(const float *x, uint64_t i, const float *y, uint64_t j, uint32_t d, int metric) {
    const float *a = x + i * d, *b = y + j * d;
    float res = 0.f;
    if (metric == NNO_L2) {
        for (uint32_t t = 0; t < d; t++) {
            float diff = a[t] - b[t];
            res += diff * diff;
        }
    } else if (metric == NNO_L1) {
        for (uint32_t t = 0; t < d; t++) res += fabsf(a[t] - b[t]);
    } else {
        for (uint32_t t = 0; t < d; t++) {
            float w1 = a[t] - b[t];
            if (a[t] != 0 || b[t] != 0) res += w1 * w1 / (a[t] + b[t]);
        }
    }
    return res;
}

/* ------------------------------------------------------------------ */
/* std::mt19937 (the generator the C++ standard fully specifies). */
typedef struct { uint32_t mt[624]; int idx; } mt_t;

static void mt_seed(mt_t *g, uint32_t s) {
    g->mt[0] = s;
    for (int i = 1; i < 624; i++)
        g->mt[i] = 1812433253u * (g->mt[i - 1] ^ (g->mt[i - 1] >> 30)) + (uint32_t)i;
    g->idx = 624;
}
static uint32_t mt_next(mt_t *g) {
    if (g->idx >= 624) {
        for (int i = 0; i < 624; i++) {
            uint32_t y = (g->mt[i] & 0x80000000u) | (g->mt[(i + 1) % 624] & 0x7fffffffu);
            g->mt[i] = g->mt[(i + 397) % 624] ^ (y >> 1) ^ ((y & 1u) ? 0x9908b0dfu : 0u);
        }
        g->idx = 0;
    }
    uint32_t y = g->mt[g->idx++];
    y ^= y >> 11;
    y ^= (y << 7) & 0x9d2c5680u;
    y ^= (y << 15) & 0xefc60000u;
    y ^= y >> 18;
    return y;
}
void nno_mt19937(uint32_t seed, uint32_t count, uint32_t *out) {
    mt_t g;
    mt_seed(&g, seed);
    for (uint32_t i = 0; i < count; i++) out[i] = mt_next(&g);
}

/* ------------------------------------------------------------------ */
/* glibc rand(): the TYPE_3 additive feedback generator of random_r
 * (degree 31, separation 3), seeded by srandom_r's Park-Miller fill and 310
 * discarded outputs.  std::random_shuffle draws from it. */
typedef struct { int32_t s[31]; int f, r; } grand_t;

static int32_t grand_next(grand_t *g) {
    uint32_t val = (uint32_t)g->s[g->f] + (uint32_t)g->s[g->r];
    g->s[g->f] = (int32_t)val;
    if (++g->f >= 31) { g->f = 0; ++g->r; }
    else if (++g->r >= 31) g->r = 0;
    return (int32_t)(val >> 1);
}
static void grand_seed(grand_t *g, uint32_t seed) {
    if (seed == 0) seed = 1;
    int32_t word = (int32_t)seed;
    g->s[0] = word;
    for (int i = 1; i < 31; i++) {
        long hi = word / 127773, lo = word % 127773;
        word = (int32_t)(16807 * lo - 2836 * hi);
        if (word < 0) word += 2147483647;
        g->s[i] = word;
    }
    g->f = 3;
    g->r = 0;
    for (int i = 0; i < 310; i++) grand_next(g);
}
void nno_glibc_rand(uint32_t seed, uint32_t count, int32_t *out) {
    grand_t g;
    grand_seed(&g, seed);
    for (uint32_t i = 0; i < count; i++) out[i] = grand_next(&g);
}

/* ------------------------------------------------------------------ */
/* Pool entry (pvetex.h:18-30 / kgraph.h:24-36) and libstdc++'s std::sort with
 * the reference's comparator "a.dist < b.dist" (introsort with a
 * median-of-three pivot, heapsort below the depth limit, then insertion sort
 * with threshold 16).  The sort is not stable, so its exact steps decide the
 * order of equal distances and must be reproduced. */
typedef struct { uint32_t id; float dist; uint32_t gd; uint8_t flag; } nbr;

#define NLESS(a, b) ((a).dist < (b).dist)

static void nswap(nbr *a, nbr *b) { nbr t = *a; *a = *b; *b = t; }

static void median_to_first(nbr *res, nbr *a, nbr *b, nbr *c) {
    if (NLESS(*a, *b)) {
        if (NLESS(*b, *c)) nswap(res, b);
        else if (NLESS(*a, *c)) nswap(res, c);
        else nswap(res, a);
    } else if (NLESS(*a, *c)) nswap(res, a);
    else if (NLESS(*b, *c)) nswap(res, c);
    else nswap(res, b);
}
static nbr *unguarded_partition(nbr *first, nbr *last, nbr *pivot) {
    for (;;) {
        while (NLESS(*first, *pivot)) ++first;
        --last;
        while (NLESS(*pivot, *last)) --last;
        if (!(first < last)) return first;
        nswap(first, last);
        ++first;
    }
}
static void heap_push(nbr *first, long hole, long top, nbr v) {
    long parent = (hole - 1) / 2;
    while (hole > top && NLESS(first[parent], v)) {
        first[hole] = first[parent];
        hole = parent;
        parent = (hole - 1) / 2;
    }
    first[hole] = v;
}
static void heap_adjust(nbr *first, long hole, long len, nbr v) {
    long top = hole, second = hole;
    while (second < (len - 1) / 2) {
        second = 2 * (second + 1);
        if (NLESS(first[second], first[second - 1])) second--;
        first[hole] = first[second];
        hole = second;
    }
    if ((len & 1) == 0 && second == (len - 2) / 2) {
        second = 2 * (second + 1);
        first[hole] = first[second - 1];
        hole = second - 1;
    }
    heap_push(first, hole, top, v);
}
static void heap_pop(nbr *first, nbr *last, nbr *result) {
    nbr v = *result;
    *result = *first;
    heap_adjust(first, 0, last - first, v);
}
static void partial_sort_all(nbr *first, nbr *last) {
    long len = last - first;
    if (len >= 2) {
        for (long parent = (len - 2) / 2;; parent--) {
            heap_adjust(first, parent, len, first[parent]);
            if (parent == 0) break;
        }
    }
    while (last - first > 1) {
        --last;
        heap_pop(first, last, last);
    }
}
static void introsort_loop(nbr *first, nbr *last, long depth) {
    while (last - first > 16) {
        if (depth == 0) {
            partial_sort_all(first, last);
            return;
        }
        --depth;
        nbr *mid = first + (last - first) / 2;
        median_to_first(first, first + 1, mid, last - 1);
        nbr *cut = unguarded_partition(first + 1, last, first);
        introsort_loop(cut, last, depth);
        last = cut;
    }
}
static void linear_insert(nbr *last) {
    nbr v = *last;
    nbr *next = last - 1;
    while (NLESS(v, *next)) {
        *last = *next;
        last = next;
        --next;
    }
    *last = v;
}
static void insertion_sort(nbr *first, nbr *last) {
    if (first == last) return;
    for (nbr *i = first + 1; i != last; ++i) {
        if (NLESS(*i, *first)) {
            nbr v = *i;
            memmove(first + 1, first, (size_t)(i - first) * sizeof(nbr));
            *first = v;
        } else {
            linear_insert(i);
        }
    }
}
static void std_sort(nbr *first, uint32_t len) {
    if (len == 0) return;
    nbr *last = first + len;
    long lg = 63 - __builtin_clzll((unsigned long long)len);
    introsort_loop(first, last, 2 * lg);
    if (len > 16) {
        insertion_sort(first, first + 16);
        for (nbr *i = first + 16; i != last; ++i) linear_insert(i);
    } else {
        insertion_sort(first, last);
    }
}
void nno_sort_pool(uint32_t *ids, float *dists, uint8_t *flags, uint32_t len) {
    nbr *t = malloc(sizeof(nbr) * (len ? len : 1));
    for (uint32_t i = 0; i < len; i++) t[i] = (nbr){ids[i], dists[i], 0, flags[i]};
    std_sort(t, len);
    for (uint32_t i = 0; i < len; i++) { ids[i] = t[i].id; dists[i] = t[i].dist; flags[i] = t[i].flag; }
    free(t);
}

/* ------------------------------------------------------------------ */
/* getRndSds (abstractgraph.cpp:7-35; copies at lynndescent.cpp:113-141 and
 * lysearch.cpp:206-233): k distinct ids in [0,N) from k+1 draws. */
static int cmp_u32(const void *a, const void *b) {
    uint32_t x = *(const uint32_t *)a, y = *(const uint32_t *)b;
    return x < y ? -1 : x > y;
}
static void rnd_seeds(mt_t *rng, uint32_t k, uint32_t *addr, uint32_t N) {
    if (N == k) {
        for (uint32_t i = 0; i < k; i++) addr[i] = i;
        return;
    }
    for (uint32_t i = 0; i < k; i++) addr[i] = mt_next(rng) % (uint32_t)(N - k);
    qsort(addr, k, sizeof(uint32_t), cmp_u32);
    for (uint32_t i = 1; i < k; i++)
        if (addr[i] <= addr[i - 1]) addr[i] = addr[i - 1] + 1;
    uint32_t off = mt_next(rng) % N;
    for (uint32_t i = 0; i < k; i++) addr[i] = (addr[i] + off) % N;
}
void nno_rnd_seeds(uint32_t seed, uint32_t rows, uint32_t k, uint32_t n, uint32_t *out) {
    mt_t g;
    mt_seed(&g, seed);
    for (uint32_t r = 0; r < rows; r++) rnd_seeds(&g, k, out + (size_t)r * k, n);
}

/* ------------------------------------------------------------------ */
/* Graph state shared by KGraph, AbstractMerge and LyNNDescent. */
typedef struct { uint32_t id, gid; } ind;                 /* pvetex.h:35-38 */
typedef struct { ind *a; uint32_t n, cap; } ivec;

static void iv_push(ivec *v, uint32_t id, uint32_t gid) {
    if (v->n == v->cap) {
        v->cap = v->cap ? v->cap * 2 : 32;
        v->a = realloc(v->a, sizeof(ind) * v->cap);
    }
    v->a[v->n].id = id;
    v->a[v->n].gid = gid;
    v->n++;
}

enum { MODE_KGRAPH, MODE_SMERGE, MODE_JMERGE, MODE_LY };

typedef struct {
    const float *x;
    uint32_t d, k, n, cap;
    int metric;
    nbr *pool;            /* cap * k */
    ivec *nw, *od, *rnw, *rod;
    nbr *cpn;             /* compensation lists, cap * k */
    uint32_t *cpn_len;
    uint64_t ncmps;
    grand_t *rnd;
    nno_stats *st;
} graph_t;

static void g_init(graph_t *g, const float *x, uint32_t cap, uint32_t d, uint32_t k, int metric,
                   grand_t *rnd, nno_stats *st) {
    memset(g, 0, sizeof(*g));
    g->x = x; g->d = d; g->k = k; g->cap = cap; g->metric = metric;
    g->pool = calloc((size_t)cap * k, sizeof(nbr));
    g->nw = calloc(cap, sizeof(ivec));
    g->od = calloc(cap, sizeof(ivec));
    g->rnw = calloc(cap, sizeof(ivec));
    g->rod = calloc(cap, sizeof(ivec));
    g->cpn = calloc((size_t)cap * k, sizeof(nbr));
    g->cpn_len = calloc(cap, sizeof(uint32_t));
    g->rnd = rnd;
    g->st = st;
}
static void g_free(graph_t *g) {
    for (uint32_t i = 0; i < g->cap; i++) {
        free(g->nw[i].a); free(g->od[i].a); free(g->rnw[i].a); free(g->rod[i].a);
    }
    free(g->nw); free(g->od); free(g->rnw); free(g->rod);
    free(g->pool); free(g->cpn); free(g->cpn_len);
}
static float gdist(graph_t *g, uint32_t a, uint32_t b) {
    return nno_dist(g->x, a, g->x, b, g->d, g->metric);
}

/* UpdateKnnList (pvetex.h:40-85, kgraph.h:42-85). */
static void update_knn(nbr *addr, uint32_t K, nbr nn) {
    uint32_t i = K, j;
    if (addr[K - 1].dist <= nn.dist) return;
    while (i > 0) {
        j = i - 1;
        if (addr[j].dist <= nn.dist) break;
        i = j;
    }
    uint32_t l = i;
    while (l > 0) {
        j = l - 1;
        if (addr[j].dist < nn.dist) break;
        if (addr[j].id == nn.id) return;
        l = j;
    }
    for (j = K - 1; j > i; --j) addr[j] = addr[j - 1];
    addr[j] = nn;
}

static void shuffle(ivec *v, grand_t *r) {             /* std::random_shuffle */
    if (v->n == 0) return;
    for (uint32_t i = 1; i < v->n; i++) {
        uint32_t j = (uint32_t)((long)grand_next(r) % (long)(i + 1));
        if (i != j) { ind t = v->a[i]; v->a[i] = v->a[j]; v->a[j] = t; }
    }
}

static int pair_ok(int mode, ind a, ind b, int verse) {
    if (a.id == b.id) return 0;
    switch (mode) {
    case MODE_KGRAPH: return 1;                                   /* kgraph.cpp:196 */
    case MODE_SMERGE: return a.gid != b.gid;                      /* smerge.cpp:224 */
    case MODE_JMERGE: return a.gid != b.gid || a.gid == 1 || b.gid == 1;   /* jmerge.cpp:191 */
    default: return a.gid != b.gid || a.gid == 1 || b.gid == 1 || verse;   /* lynndescent.cpp:330 */
    }
}

static void join_pair(graph_t *g, int mode, uint32_t n, ind a, ind b, int verse, uint64_t *cc) {
    if (!pair_ok(mode, a, b, verse)) return;
    float dst = gdist(g, a.id, b.id);
    (*cc)++;
    nbr x = {b.id, dst, mode == MODE_KGRAPH ? n : b.gid, 1};
    update_knn(g->pool + (size_t)a.id * g->k, g->k, x);
    nbr y = {a.id, dst, mode == MODE_KGRAPH ? n : a.gid, 1};
    update_knn(g->pool + (size_t)b.id * g->k, g->k, y);
}

/* The NN-Descent iteration loop: kgraph.cpp:98-189, abstractmerge.cpp:78-192,
 * lynndescent.cpp:201-310.  `split` is the first row of the second group
 * (AbstractMerge::preSize, or LyNNDescent's lst_idx with begin_idx 0), used
 * for the group id of reverse entries. */
static void nndescent(graph_t *g, int mode, uint32_t split, int verse) {
    const uint32_t smpl = 100, K = g->k, N = g->n;
    for (;;) {
        for (uint32_t irow = 0; irow < N; irow++) {
            for (uint32_t idim = 0; idim < K; idim++) {
                nbr *nb = &g->pool[(size_t)irow * K + idim];
                float maxd = g->pool[(size_t)nb->id * K + K - 1].dist;
                uint32_t rg = (mode == MODE_KGRAPH) ? 0 : (irow >= split);
                if (nb->flag) {
                    iv_push(&g->nw[irow], nb->id, nb->gd);
                    if (maxd < nb->dist) iv_push(&g->rnw[nb->id], irow, rg);
                    nb->flag = 0;
                } else {
                    iv_push(&g->od[irow], nb->id, nb->gd);
                    if (maxd < nb->dist) iv_push(&g->rod[nb->id], irow, rg);
                }
            }
        }
        for (uint32_t irow = 0; irow < N; irow++) {
            shuffle(&g->rnw[irow], g->rnd);
            if (g->rnw[irow].n > smpl) g->rnw[irow].n = smpl;
            shuffle(&g->rod[irow], g->rnd);
            if (g->rod[irow].n > smpl) g->rod[irow].n = smpl;
            for (uint32_t t = 0; t < g->rnw[irow].n; t++)
                iv_push(&g->nw[irow], g->rnw[irow].a[t].id, g->rnw[irow].a[t].gid);
            for (uint32_t t = 0; t < g->rod[irow].n; t++)
                iv_push(&g->od[irow], g->rod[irow].a[t].id, g->rod[irow].a[t].gid);
        }
        uint64_t cc = 0;
        for (uint32_t n = 0; n < N; n++) {
            ivec *nw = &g->nw[n], *od = &g->od[n];
            for (uint32_t i = 0; i < nw->n; i++) {
                if (mode == MODE_KGRAPH) {                       /* kgraph.h:110-122 */
                    for (uint32_t j = 0; j < nw->n; j++)
                        if (nw->a[i].id < nw->a[j].id) join_pair(g, mode, n, nw->a[i], nw->a[j], verse, &cc);
                } else {                                         /* pvetex.h:111-125 */
                    for (uint32_t j = i + 1; j < nw->n; j++)
                        join_pair(g, mode, n, nw->a[i], nw->a[j], verse, &cc);
                }
                for (uint32_t j = 0; j < od->n; j++)
                    join_pair(g, mode, n, nw->a[i], od->a[j], verse, &cc);
            }
        }
        g->ncmps += cc;
        /* EvaluateDelta + Boost mean over float samples. */
        float sum = 0.f;
        for (uint32_t irow = 0; irow < N; irow++) {
            uint32_t c = 0;
            for (uint32_t t = 0; t < K; t++) c += g->pool[(size_t)irow * K + t].flag ? 1u : 0u;
            sum += (float)c / (float)K;
        }
        float mean = sum / (float)N;
        if (g->st) {
            if (g->st->trace && g->st->trace_len < g->st->trace_cap) g->st->trace[g->st->trace_len] = mean;
            g->st->trace_len++;
        }
        /* On convergence the loop breaks BEFORE clearing the sample lists
         * (kgraph.cpp:167-181, abstractmerge.cpp:221-232,
         * lynndescent.cpp:293-305).  LyNNDescent calls nnDescent once per
         * level on the same graph, so the next level's sampling pass appends
         * to these leftover lists, stale group ids included. */
        if (mean < 0.002f) break;
        for (uint32_t irow = 0; irow < N; irow++) {
            g->nw[irow].n = g->od[irow].n = g->rnw[irow].n = g->rod[irow].n = 0;
        }
    }
}

static void out_pools(graph_t *g, uint32_t *ids, float *dists, uint8_t *flags) {
    for (size_t t = 0; t < (size_t)g->n * g->k; t++) {
        if (ids) ids[t] = g->pool[t].id;
        if (dists) dists[t] = g->pool[t].dist;
        if (flags) flags[t] = g->pool[t].flag;
    }
}

/* KGraph::InitialGraph (kgraph.cpp:56-96) + nndescent. */
static void kgraph_build(graph_t *g, uint32_t seed) {
    const uint32_t K = g->k, N = g->n;
    uint32_t *seeds = malloc(sizeof(uint32_t) * (K + 1));
    mt_t rng;
    mt_seed(&rng, seed);
    for (uint32_t i = 0; i < N; i++) {
        nbr *p = g->pool + (size_t)i * K;
        rnd_seeds(&rng, K + 1, seeds, N);
        uint32_t L = 0;
        for (uint32_t j = 0; j < K + 1; j++) {
            if (seeds[j] == i) continue;
            p[L].id = seeds[j];
            p[L].gd = seeds[j];
            p[L].dist = gdist(g, i, seeds[j]);
            g->ncmps++;
            p[L].flag = 1;
            if (++L >= K) break;
        }
        std_sort(p, K);
    }
    free(seeds);
    nndescent(g, MODE_KGRAPH, 0, 0);
}

int nno_kgraph(const float *x, uint32_t n, uint32_t d, uint32_t k, int metric, uint32_t seed,
               uint32_t *ids, float *dists, uint8_t *flags, nno_stats *st) {
    if (n < k + 2 || k == 0) return -1;
    grand_t rnd;
    grand_seed(&rnd, seed);
    graph_t g;
    g_init(&g, x, n, d, k, metric, &rnd, st);
    g.n = n;
    kgraph_build(&g, seed);
    out_pools(&g, ids, dists, flags);
    if (st) st->ncmps = g.ncmps;
    g_free(&g);
    return 0;
}

/* Builds a sub-graph on rows [b, e) (a KGraph on the cutMat copy) and
 * returns its ids, relative to b. */
static uint32_t *sub_kgraph(const float *x, uint32_t b, uint32_t e, uint32_t d, uint32_t k,
                            int metric, uint32_t seed, grand_t *rnd, nno_stats *st) {
    graph_t g;
    g_init(&g, x + (size_t)b * d, e - b, d, k, metric, rnd, st);
    g.n = e - b;
    kgraph_build(&g, seed);
    uint32_t *ids = malloc(sizeof(uint32_t) * (size_t)g.n * k);
    out_pools(&g, ids, NULL, NULL);
    g_free(&g);
    return ids;
}

/* AbstractMerge::InitSGraph (abstractmerge.cpp:55-76). */
static void init_sgraph(graph_t *g, uint32_t b, const uint32_t *sub, uint32_t gid, uint32_t size) {
    const uint32_t K = g->k;
    for (uint32_t i = 0; i < size; i++) {
        uint32_t row = b + i;
        for (uint32_t j = 0; j < K; j++) {
            nbr *nb = &g->pool[(size_t)row * K + j];
            nb->id = sub[(size_t)i * K + j] + b;
            nb->dist = gdist(g, row, nb->id);
            nb->flag = 1;
            nb->gd = gid;
        }
    }
}

/* Cross-sampling of an already-built row (smerge.cpp:104-150 and :157-203,
 * jmerge.cpp:90-135, lynndescent.cpp:371-415): keep the best K-cut entries,
 * move the worst `cut` to the compensation list, put `cut` random ids of the
 * other group (seed + base, skipping ids already in the pool) in their
 * place, then std::sort.  Returns -1 if fewer than `cut` ids were found. */
static int cross_sample_row(graph_t *g, uint32_t i, mt_t *rng, uint32_t cut, uint32_t draws,
                            uint32_t range, uint32_t base, uint32_t gd, uint32_t *seeds) {
    const uint32_t K = g->k, remain = K - cut;
    nbr *p = g->pool + (size_t)i * K;
    rnd_seeds(rng, draws, seeds, range);
    for (uint32_t j = 0; j < cut; j++) g->cpn[(size_t)i * K + j] = p[j + remain];
    g->cpn_len[i] = cut;
    uint32_t tp[512], ntp = 0;
    for (uint32_t m = 0; m < draws; m++) {
        if (ntp >= cut) break;
        uint32_t rid = seeds[m] + base;
        int dup = 0;
        for (uint32_t l = 0; l < K; l++)
            if (p[l].id == rid) { dup = 1; break; }
        if (!dup) tp[ntp++] = rid;
    }
    if (ntp < cut) return -1;
    for (uint32_t j = 0; j < cut; j++) {
        nbr *nb = &p[j + remain];
        nb->id = tp[j];
        nb->gd = gd;
        nb->flag = 1;
        nb->dist = gdist(g, nb->id, i);
        g->ncmps++;
    }
    std_sort(p, K);
    return 0;
}

/* AbstractMerge::merge2one (abstractmerge.cpp:232-277), lynndescent.cpp:455-500. */
static void merge2one(graph_t *g, uint32_t sz) {
    const uint32_t K = g->k;
    nbr tmp[512];
    for (uint32_t i = 0; i < sz; i++) {
        nbr *p = g->pool + (size_t)i * K, *c = g->cpn + (size_t)i * K;
        uint32_t m = 0, n = 0;
        for (uint32_t t = 0; t < K; t++) {
            if (n >= g->cpn_len[i] || p[m].dist <= c[n].dist) tmp[t] = p[m++];
            else tmp[t] = c[n++];
        }
        memcpy(p, tmp, sizeof(nbr) * K);
    }
    memset(g->cpn_len, 0, sizeof(uint32_t) * g->cap);
}

static int merge_common(int mode, const float *x, uint32_t n, uint32_t d, uint32_t k, int metric,
                        uint32_t seed, uint32_t *ids, float *dists, uint8_t *flags, nno_stats *st) {
    if (k == 0 || k > 256 || n / 2 < k + 2) return -1;
    grand_t rnd;
    grand_seed(&rnd, seed);
    uint32_t pre = n * 5 / 10;                                   /* smerge.cpp:53, jmerge.cpp:47 */
    uint32_t *g1 = sub_kgraph(x, 0, pre, d, k, metric, seed, &rnd, st);
    uint32_t *g2 = mode == MODE_SMERGE ? sub_kgraph(x, pre, n, d, k, metric, seed, &rnd, st) : NULL;
    graph_t g;
    g_init(&g, x, n, d, k, metric, &rnd, st);
    g.n = n;
    init_sgraph(&g, 0, g1, 0, pre);
    if (g2) init_sgraph(&g, pre, g2, 1, n - pre);
    mt_t rng;
    mt_seed(&rng, seed);
    uint32_t cut = mode == MODE_SMERGE ? k * 1 / 2 : k * 3 / 6;  /* smerge.cpp:99, jmerge.cpp:87 */
    uint32_t seeds[1024];
    int rc = 0;
    for (uint32_t i = 0; i < pre && !rc; i++)
        rc = cross_sample_row(&g, i, &rng, cut, 2 * cut, n - pre, pre, 1, seeds);
    if (mode == MODE_SMERGE) {
        for (uint32_t i = pre; i < n && !rc; i++)
            rc = cross_sample_row(&g, i, &rng, cut, 2 * cut, pre, 0, 0, seeds);
    } else {                                                     /* jmerge.cpp:147-171 */
        for (uint32_t i = pre; i < n; i++) {
            nbr *p = g.pool + (size_t)i * k;
            rnd_seeds(&rng, k + 1, seeds, n);
            uint32_t L = 0;
            for (uint32_t j = 0; j < k + 1; j++) {
                if (seeds[j] == i || L >= k) continue;
                nbr *nb = &p[L++];
                nb->id = seeds[j];
                nb->gd = seeds[j] >= pre;
                nb->flag = 1;
                nb->dist = gdist(&g, nb->id, i);
                g.ncmps++;
            }
            std_sort(p, k);
        }
    }
    if (!rc) {
        nndescent(&g, mode, pre, 0);
        merge2one(&g, mode == MODE_SMERGE ? n : pre);
        out_pools(&g, ids, dists, flags);
        if (st) st->ncmps = g.ncmps;
    }
    free(g1);
    free(g2);
    g_free(&g);
    return rc;
}

int nno_smerge(const float *x, uint32_t n, uint32_t d, uint32_t k, int metric, uint32_t seed,
               uint32_t *ids, float *dists, uint8_t *flags, nno_stats *st) {
    return merge_common(MODE_SMERGE, x, n, d, k, metric, seed, ids, dists, flags, st);
}
int nno_jmerge(const float *x, uint32_t n, uint32_t d, uint32_t k, int metric, uint32_t seed,
               uint32_t *ids, float *dists, uint8_t *flags, nno_stats *st) {
    return merge_common(MODE_JMERGE, x, n, d, k, metric, seed, ids, dists, flags, st);
}

/* ------------------------------------------------------------------ */
/* H-Merge (LyNNDescent) with DPG layers. */
typedef struct { uint32_t id; float dist; } dn;
typedef struct { dn *a; uint32_t n, cap; } dvec;

static void dv_resize(dvec *v, uint32_t n) {
    if (n > v->cap) {
        v->cap = n < 8 ? 8 : n * 2;
        v->a = realloc(v->a, sizeof(dn) * v->cap);
    }
    v->n = n;
}

/* LyNNDescent::insert2topk (lynndescent.cpp:546-623). */
static void dpg_insert(dvec *v, uint32_t nid, float dst, uint32_t maxSize) {
    uint32_t topk = v->n, i, j;
    if (topk == 0) {
        dv_resize(v, 1);
        v->a[0].id = nid;
        v->a[0].dist = dst;
        return;
    }
    i = topk;
    if (v->a[topk - 1].dist < dst && topk == maxSize) return;
    if (topk < maxSize && v->a[topk - 1].dist < dst) {
        dv_resize(v, topk + 1);
        v->a[topk].id = nid;
        v->a[topk].dist = dst;
        return;
    }
    while (i > 0) {
        j = i - 1;
        if (v->a[j].dist <= dst) break;
        i = j;
    }
    uint32_t l = i;
    while (l > 0) {
        j = l - 1;
        if (v->a[j].dist < dst) break;
        if (v->a[j].id == nid) return;
        l = j;
    }
    if (topk < maxSize) {
        dv_resize(v, topk + 1);
        j = topk;
    } else {
        j = maxSize - 1;
    }
    while (j > i) {
        v->a[j] = v->a[j - 1];
        --j;
    }
    v->a[j].id = nid;
    v->a[j].dist = dst;
}

typedef struct {
    graph_t g;
    dvec *dpg;          /* LyNNDescent::graph, never cleared between layers */
    uint32_t dpg_rows;
    uint32_t row, M;
    nno_layers *layers;
} hm_t;

/* LyNNDescent::dpg + DelaunayGraph (lynndescent.cpp:502-544, :640-713). */
static void hm_dpg(hm_t *h) {
    graph_t *g = &h->g;
    const uint32_t N = g->n, K = g->k, Mo = K / 2;
    const uint32_t maxM = (N == h->row) ? h->M : h->M / 2;
    if (N > h->dpg_rows) {
        h->dpg = realloc(h->dpg, sizeof(dvec) * N);
        memset(h->dpg + h->dpg_rows, 0, sizeof(dvec) * (N - h->dpg_rows));
        h->dpg_rows = N;
    }
    for (uint32_t i = 0; i < N; i++) {
        dvec *gi = &h->dpg[i];
        for (uint32_t j = 0; j < K; j++) {
            if (gi->n > Mo) break;
            uint32_t nb = g->pool[(size_t)i * K + j].id;
            float dst = gdist(g, i, nb);
            int good = 1;
            for (uint32_t l = 0; l < gi->n; l++)
                if (gdist(g, gi->a[l].id, nb) < dst) good = 0;
            if (good) dpg_insert(gi, nb, dst, Mo);
        }
    }
    for (uint32_t i = 0; i < N; i++) {
        uint32_t num = h->dpg[i].n;
        for (uint32_t j = 0; j < num; j++) {
            dn nn = h->dpg[i].a[j];
            dvec *gt = &h->dpg[nn.id];
            if (gt->n < maxM) {
                dpg_insert(gt, i, nn.dist, maxM);
            } else {
                int ok = 1;
                for (uint32_t t = 0; t < gt->n; t++)
                    if (gdist(g, gt->a[t].id, i) < nn.dist) { ok = 0; break; }
                if (ok) dpg_insert(gt, i, nn.dist, maxM);
            }
        }
    }
    if (h->layers && h->layers->nlayers < 16) {                 /* saveDPGraph (:625-638) */
        uint32_t L = h->layers->nlayers++;
        h->layers->nrows[L] = N;
        uint64_t *off = malloc(sizeof(uint64_t) * ((size_t)N + 1));
        off[0] = 0;
        for (uint32_t i = 0; i < N; i++) off[i + 1] = off[i] + h->dpg[i].n;
        uint32_t *adj = malloc(sizeof(uint32_t) * (off[N] ? off[N] : 1));
        for (uint32_t i = 0; i < N; i++)
            for (uint32_t j = 0; j < h->dpg[i].n; j++) adj[off[i] + j] = h->dpg[i].a[j].id;
        h->layers->off[L] = off;
        h->layers->adj[L] = adj;
    }
}

/* LyNNDescent::appdNwSmpl (lynndescent.cpp:354-452). */
static int hm_append(hm_t *h, uint32_t half, uint32_t bnum, uint32_t *last_id, uint32_t seed) {
    graph_t *g = &h->g;
    const uint32_t K = g->k, sz = g->n, hsize = K - half, lst = *last_id;
    mt_t rng;
    mt_seed(&rng, seed);
    uint32_t seeds[1024];
    for (uint32_t i = 0; i < sz; i++)
        if (cross_sample_row(g, i, &rng, hsize, 2 * half, bnum, lst, 1, seeds)) return -1;
    g->n = sz + bnum;
    for (uint32_t i = sz; i < g->n; i++) {
        nbr *p = g->pool + (size_t)i * K;
        rnd_seeds(&rng, 2 * K, seeds, g->n);
        uint32_t nk = 0;
        for (uint32_t j = 0; j < 2 * K; j++) {
            if (nk >= K) break;
            if (seeds[j] == i) continue;
            p[nk].id = seeds[j];
            p[nk].dist = gdist(g, i, seeds[j]);
            p[nk].flag = 1;
            p[nk].gd = !(seeds[j] < lst);                         /* getGraphId, begin_idx 0 */
            nk++;
            g->ncmps++;
        }
        std_sort(p, K);
    }
    *last_id = lst + bnum;
    return 0;
}

int nno_hmerge(const float *x, uint32_t n, uint32_t d, uint32_t k, uint32_t m, int metric,
               uint32_t seed, uint32_t *ids, float *dists, uint8_t *flags, nno_stats *st,
               nno_layers *layers) {
    const uint32_t N0 = 64;                                       /* lynndescent.cpp:23 */
    if (k == 0 || k + 1 > N0 || 2 * k > 1024 || n <= N0) return -1;
    grand_t rnd;
    grand_seed(&rnd, seed);
    hm_t h;
    memset(&h, 0, sizeof(h));
    h.row = n;
    h.M = m;
    h.layers = layers;
    if (layers) memset(layers, 0, sizeof(*layers));
    graph_t *g = &h.g;
    g_init(g, x, n, d, k, metric, &rnd, st);
    /* init (lynndescent.cpp:143-187) */
    {
        mt_t rng;
        mt_seed(&rng, seed);
        uint32_t seeds[1024];
        for (uint32_t i = 0; i < N0; i++) {
            nbr *p = g->pool + (size_t)i * k;
            rnd_seeds(&rng, k + 1, seeds, N0);
            uint32_t L = 0;
            for (uint32_t j = 0; j < k + 1; j++) {
                if (seeds[j] == i) continue;
                p[L].id = seeds[j];
                p[L].dist = gdist(g, i, seeds[j]);
                g->ncmps++;
                p[L].flag = 1;
                p[L].gd = 0;
                if (++L >= k) break;
            }
            std_sort(p, k);
        }
    }
    g->n = N0;
    uint32_t last_id = N0, total = n - N0, smpl = N0, count_level = 0;
    nndescent(g, MODE_LY, N0, 1);
    hm_dpg(&h);
    count_level++;
    static const uint32_t level[10] = {1, 0, 0, 1, 0, 0, 1, 0, 0, 1};
    int rc = 0;
    while (total != 0 && !rc) {                                   /* buildhgraph (:772-808) */
        if (total > smpl) {
            uint32_t lst = last_id;
            rc = hm_append(&h, k / 2, smpl, &last_id, seed);
            if (rc) break;
            total -= smpl;
            nndescent(g, MODE_LY, lst, 0);
            merge2one(g, lst);
            if (count_level < 10 && level[count_level]) hm_dpg(&h);
            count_level++;
            smpl = g->n;
            for (size_t t = 0; t < (size_t)g->n * k; t++) g->pool[t].gd = 0;   /* setflag */
        } else {
            uint32_t lst = last_id;
            rc = hm_append(&h, k / 2, total, &last_id, seed);
            if (rc) break;
            nndescent(g, MODE_LY, lst, 0);
            merge2one(g, lst);
            hm_dpg(&h);
            count_level++;
            total = 0;
        }
    }
    if (!rc) {
        out_pools(g, ids, dists, flags);
        if (st) st->ncmps = g->ncmps;
    }
    for (uint32_t i = 0; i < h.dpg_rows; i++) free(h.dpg[i].a);
    free(h.dpg);
    g_free(g);
    return rc;
}

void nno_free_layers(nno_layers *layers) {
    for (uint32_t l = 0; l < layers->nlayers; l++) {
        free(layers->off[l]);
        free(layers->adj[l]);
        layers->off[l] = NULL;
        layers->adj[l] = NULL;
    }
    layers->nlayers = 0;
}

/* ------------------------------------------------------------------ */
/* LySearch.  std::priority_queue<pair<float,unsigned>> with CompareByFirst
 * (lysearch.h:37-42) is a max-heap on .first built from libstdc++'s
 * push_heap/pop_heap; its exact steps decide tie order, so they are
 * reproduced. */
typedef struct { float first; uint32_t second; } fpair;
typedef struct { fpair *a; uint32_t n, cap; } pq_t;

static void pq_sift_up(fpair *a, long hole, long top, fpair v) {
    long parent = (hole - 1) / 2;
    while (hole > top && a[parent].first < v.first) {
        a[hole] = a[parent];
        hole = parent;
        parent = (hole - 1) / 2;
    }
    a[hole] = v;
}
static void pq_adjust(fpair *a, long hole, long len, fpair v) {
    long top = hole, second = hole;
    while (second < (len - 1) / 2) {
        second = 2 * (second + 1);
        if (a[second].first < a[second - 1].first) second--;
        a[hole] = a[second];
        hole = second;
    }
    if ((len & 1) == 0 && second == (len - 2) / 2) {
        second = 2 * (second + 1);
        a[hole] = a[second - 1];
        hole = second - 1;
    }
    pq_sift_up(a, hole, top, v);
}
static void pq_push(pq_t *q, float f, uint32_t s) {
    if (q->n == q->cap) {
        q->cap = q->cap ? q->cap * 2 : 64;
        q->a = realloc(q->a, sizeof(fpair) * q->cap);
    }
    fpair v = {f, s};
    q->a[q->n++] = v;
    pq_sift_up(q->a, q->n - 1, 0, v);
}
static void pq_pop(pq_t *q) {
    if (q->n > 1) {
        long last = q->n - 1;
        fpair v = q->a[last];
        q->a[last] = q->a[0];
        pq_adjust(q->a, 0, last, v);
    }
    q->n--;
}

int nno_search(const float *x, uint32_t n, uint32_t d, const nno_layers *layers,
               const float *q, uint32_t nq, uint32_t topk, int metric, uint32_t seed,
               uint32_t *out_ids, float *out_dists, uint64_t *ncmps, uint32_t *entry) {
    return nno_search_ex(x, n, d, layers, q, nq, NULL, topk, topk, NULL, 0, 0, 0, metric, seed, out_ids, out_dists,
                         ncmps, entry);
}

/* The serving form: query i searches with beam width beams[i] (or `beam`)
 * and keeps its first out_k results; with probes (nq x nprobe rows of layer
 * g0) a query starts at the first nearest of its probes, in probe order,
 * and descends from layer g0 instead of from the global entry on layer 0.
 * flat: nndFlatSrch (lysearch.cpp:439-520) -- no descent; the beam starts
 * with getRndSds(mt19937(seed), beam, rows of the last layer) pushed in
 * draw order (the reference seeds a new generator from its clock per query,
 * lysearch.cpp:455, so with the clock frozen every query draws the same). */
int nno_search_ex(const float *x, uint32_t n, uint32_t d, const nno_layers *layers,
                  const float *q, uint32_t nq, const uint32_t *beams, uint32_t beam, uint32_t out_k,
                  const uint32_t *probes, uint32_t nprobe, uint32_t g0, int flat, int metric, uint32_t seed,
                  uint32_t *out_ids, float *out_dists, uint64_t *ncmps, uint32_t *entry) {
    if (!layers || layers->nlayers < 1 || beam == 0 || out_k == 0) return -1;
    const uint32_t L = layers->nlayers;
    if (probes && (nprobe == 0 || g0 >= L)) return -1;
    const uint32_t nlast = layers->nrows[L - 1];
    if (flat)
        for (uint32_t qi = 0; qi < nq; qi++)
            if ((beams ? beams[qi] : beam) > nlast) return -1;
    uint32_t *sds = flat ? malloc(sizeof(uint32_t) * (nlast + 1)) : NULL;
    grand_t rnd;
    grand_seed(&rnd, seed);
    uint32_t enter = (uint32_t)grand_next(&rnd) % layers->nrows[0];  /* lysearch.cpp:382 */
    if (entry) *entry = enter;
    uint8_t *flags = calloc(n, 1);
    uint32_t *pts = malloc(sizeof(uint32_t) * n);
    pq_t top = {0}, cand = {0};
    uint64_t cmps = 0;
    for (uint32_t qi = 0; qi < nq; qi++) {
        const float *qv = q + (size_t)qi * d;
        const uint32_t topk = beams ? beams[qi] : beam;
        uint32_t cur = enter, gstart = 0;
        float cur_d = 0.f;
        if (flat) {
            mt_t rng;
            mt_seed(&rng, seed);
            rnd_seeds(&rng, topk, sds, nlast);
        } else if (probes) {
            gstart = g0;
            cur = probes[(size_t)qi * nprobe];
            cur_d = nno_dist(qv, 0, x, cur, d, metric);
            for (uint32_t j = 1; j < nprobe; j++) {
                const uint32_t pj = probes[(size_t)qi * nprobe + j];
                const float dj = nno_dist(qv, 0, x, pj, d, metric);
                if (dj < cur_d) { cur_d = dj; cur = pj; }
            }
            cmps += nprobe;
        } else {
            cur_d = nno_dist(qv, 0, x, cur, d, metric);
            cmps++;
        }
        for (uint32_t ir = gstart; !flat && ir + 1 < L; ir++) {           /* :397-420 */
            const uint64_t *off = layers->off[ir];
            const uint32_t *adj = layers->adj[ir];
            int moved = 1;
            while (moved) {
                moved = 0;
                const uint64_t b = off[cur], e = off[cur + 1];   /* list of the node at loop entry */
                for (uint64_t t = b; t < e; t++) {
                    uint32_t nn = adj[t];
                    float dd = nno_dist(qv, 0, x, nn, d, metric);
                    cmps++;
                    if (dd < cur_d) { cur_d = dd; cur = nn; moved = 1; }
                }
            }
        }
        /* nndHNSWSrch (:236-322) on the last layer */
        const uint64_t *off = layers->off[L - 1];
        const uint32_t *adj = layers->adj[L - 1];
        uint32_t npts = 0;
        top.n = cand.n = 0;
        if (flat) {
            for (uint32_t i = 0; i < topk; i++) {  /* lysearch.cpp:462-472 */
                const uint32_t s = sds[i];
                const float ds = nno_dist(qv, 0, x, s, d, metric);
                pq_push(&cand, -ds, s);
                pq_push(&top, ds, s);
                flags[s] = 1;
                pts[npts++] = s;
                cmps++;
            }
        } else {
            pq_push(&cand, -cur_d, cur);
            pq_push(&top, cur_d, cur);
            flags[cur] = 1;
            pts[npts++] = cur;
        }
        float lwbnd = top.a[0].first;
        while (cand.n) {
            fpair c = cand.a[0];
            if (-c.first > lwbnd) break;
            pq_pop(&cand);
            for (uint64_t t = off[c.second]; t < off[c.second + 1]; t++) {
                uint32_t cid = adj[t];
                if (flags[cid]) continue;
                flags[cid] = 1;
                pts[npts++] = cid;
                float dst = nno_dist(qv, 0, x, cid, d, metric);
                cmps++;
                if (top.a[0].first > dst || top.n < topk) {
                    pq_push(&cand, -dst, cid);
                    pq_push(&top, dst, cid);
                    if (top.n > topk) pq_pop(&top);
                    lwbnd = top.a[0].first;
                }
            }
        }
        for (uint32_t t = 0; t < out_k; t++) {
            out_ids[(size_t)qi * out_k + t] = 0xffffffffu;
            out_dists[(size_t)qi * out_k + t] = 0.f;
        }
        for (long loc = (long)top.n - 1; loc >= 0; loc--) {
            if ((uint32_t)loc < out_k) {
                out_ids[(size_t)qi * out_k + loc] = top.a[0].second;
                out_dists[(size_t)qi * out_k + loc] = top.a[0].first;
            }
            pq_pop(&top);
        }
        for (uint32_t t = 0; t < npts; t++) flags[pts[t]] = 0;
    }
    if (ncmps) *ncmps = cmps;
    free(top.a);
    free(cand.a);
    free(flags);
    free(pts);
    free(sds);
    return 0;
}
