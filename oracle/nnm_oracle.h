/* Test infrastructure only: a CPU restatement of the nn-merge hot path,
 * used by tests/, __graft_entry__.smoke() and bench.py's CPU baseline leg as
 * the checker.  The product (nn-merge_b200/) never links or calls it.
 *
 * Every routine follows the reference operation for operation, so that under
 * a fixed seed it reproduces the reference's neighbour ids, distances,
 * flags, distance-evaluation counts and iteration counts bit for bit.  It is
 * pinned against the reference itself (oracle/_ref/nnm_ref, built from the
 * reference sources by oracle/Makefile) by tests/test_oracle_vs_ref.py and
 * against the committed fixtures in tests/golden/.
 *
 * Seeding model (mirrors a reference process whose wall clock reads `seed`
 * for the whole run): every phase that constructs std::mt19937(time(NULL))
 * gets mt19937(seed); the process-wide std::rand() stream behind
 * std::random_shuffle starts from srand(seed) at the start of each call. */
#ifndef NNM_ORACLE_H
#define NNM_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { NNO_L2 = 0, NNO_L1 = 1, NNO_CHI2 = 2 };

typedef struct {
    uint64_t ncmps;      /* distance evaluations, counted where the reference counts them */
    uint32_t trace_len;  /* number of NN-Descent iterations run (all loops, in order) */
    uint32_t trace_cap;
    float *trace;        /* convergence mean of each iteration (may be NULL) */
} nno_stats;

/* Search hierarchy: layer g has nrows[g] rows; row i's neighbours are
 * adj[g][off[g][i] .. off[g][i+1]). */
typedef struct {
    uint32_t nlayers;
    uint32_t nrows[16];
    uint64_t *off[16];
    uint32_t *adj[16];
} nno_layers;

float nno_dist(const float *x, uint64_t i, const float *y, uint64_t j, uint32_t d, int metric);

/* KGraph::buildKGraph (kgraph.cpp:217-245).  Outputs n*k each. */
int nno_kgraph(const float *x, uint32_t n, uint32_t d, uint32_t k, int metric, uint32_t seed,
               uint32_t *ids, float *dists, uint8_t *flags, nno_stats *st);
/* Smerge::buildKGraph (smerge.cpp:46-91). ncmps covers the merge phase only. */
int nno_smerge(const float *x, uint32_t n, uint32_t d, uint32_t k, int metric, uint32_t seed,
               uint32_t *ids, float *dists, uint8_t *flags, nno_stats *st);
/* Jmerge::buildKGraph (jmerge.cpp:43-80). ncmps covers the merge phase only. */
int nno_jmerge(const float *x, uint32_t n, uint32_t d, uint32_t k, int metric, uint32_t seed,
               uint32_t *ids, float *dists, uint8_t *flags, nno_stats *st);
/* LyNNDescent::buildhgraph (lynndescent.cpp:735-831).  The DPG layers are
 * returned in *layers (free with nno_free_layers). */
int nno_hmerge(const float *x, uint32_t n, uint32_t d, uint32_t k, uint32_t m, int metric,
               uint32_t seed, uint32_t *ids, float *dists, uint8_t *flags, nno_stats *st,
               nno_layers *layers);
void nno_free_layers(nno_layers *layers);
/* LySearch::knnSearch per-query steps (lysearch.cpp:363-437) at one beam
 * width: greedy descent on layers 0..L-2, nndHNSWSrch on layer L-1. */
int nno_search(const float *x, uint32_t n, uint32_t d, const nno_layers *layers,
               const float *q, uint32_t nq, uint32_t topk, int metric, uint32_t seed,
               uint32_t *out_ids, float *out_dists, uint64_t *ncmps, uint32_t *entry);
/* Serving form: per-query beam widths (beams, or `beam` for all), the first
 * out_k results of each query, and optional learned entries: the first
 * nearest of probes[i*nprobe ..] starts the greedy descent on layer g0.
 * flat != 0: nndFlatSrch (no descent, getRndSds seeds of the last layer). */
int nno_search_ex(const float *x, uint32_t n, uint32_t d, const nno_layers *layers,
                  const float *q, uint32_t nq, const uint32_t *beams, uint32_t beam, uint32_t out_k,
                  const uint32_t *probes, uint32_t nprobe, uint32_t g0, int flat, int metric, uint32_t seed,
                  uint32_t *out_ids, float *out_dists, uint64_t *ncmps, uint32_t *entry);

/* Building blocks exposed for unit tests. */
void nno_glibc_rand(uint32_t seed, uint32_t count, int32_t *out);
void nno_mt19937(uint32_t seed, uint32_t count, uint32_t *out);
void nno_rnd_seeds(uint32_t seed, uint32_t rows, uint32_t k, uint32_t n, uint32_t *out);
void nno_sort_pool(uint32_t *ids, float *dists, uint8_t *flags, uint32_t len);

#ifdef __cplusplus
}
#endif
#endif
