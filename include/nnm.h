/* nnm: B200 (sm_100a) k-NN graph construction, merge and search.
 *
 * C ABI of the drop-in for the nn-merge hot path.  Plain pointers and
 * sizes only.  Every call returns an nnm_status code; nnm_last_error()
 * gives the message of the last failure on a context.
 *
 * Memory: "host" entry points take caller-owned host arrays and copy them
 * to and from the GPU inside the call; "_dev" entry points take device
 * pointers (inputs already resident in HBM).  The library owns its device
 * workspace, which nnm_ctx_destroy frees.  A context is bound to one CUDA
 * device and one stream and is not thread-safe; separate contexts may run
 * concurrently.
 *
 * Seeding: the reference seeds each phase with std::mt19937(time(NULL)) and
 * shuffles with std::rand().  Under NNM_RNG_EXACT every such phase here uses
 * mt19937(opts.seed) and the std::rand() stream starts from srand(opts.seed)
 * at the start of each call -- the reference run with its clock frozen at
 * opts.seed -- so ids, distances, flags, distance counts and iteration
 * counts equal the reference's bit for bit.
 */
#ifndef NNM_H
#define NNM_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    NNM_OK = 0,
    NNM_ERR_INVALID = 1,            /* bad argument (sizes, null pointers, K limits) */
    NNM_ERR_UNSUPPORTED_METRIC = 2, /* distance function the device does not implement */
    NNM_ERR_CUDA = 3,               /* CUDA runtime error */
    NNM_ERR_OOM = 4,                /* device allocation failed */
    NNM_ERR_NO_DEVICE = 5,          /* no usable CUDA device */
    NNM_ERR_CAPACITY = 6            /* a device-side capacity/consistency check failed */
} nnm_status;

/* Distance functions of the reference (space_lp.h:9-53). */
typedef enum {
    NNM_METRIC_L2 = 0,   /* VMath::l2norm: squared L2, vmath.cpp:56-88 */
    NNM_METRIC_L1 = 1,   /* DistOpt::l1norm, distopt.cpp:82-114 */
    NNM_METRIC_CHI2 = 2  /* DistOpt::KSquare, distopt.cpp:165-184 */
} nnm_metric;

typedef enum {
    NNM_RNG_EXACT = 0, /* the reference's mt19937 / std::rand streams: bit-exact results */
    NNM_RNG_FAST = 1   /* counter-based draws (Philox) on the device: same algorithm, different
                          random choices, no host-side streams and no ordering of reverse lists */
} nnm_rng_mode;

/* Kernel of the local join's distance evaluations.  All give the same
   graphs bit for bit.  The tensor-core joins need the L2 metric.  For data
   whose components are all integers in [0, 255] the u8 join computes Gram
   matrices exactly (every squared distance stays below 2^24, where the
   reference's float sum is exact).  The reduced-precision joins (other
   finite data, |components| in [2^-60, 2^50]) compute d~ = |a|^2 + |b|^2 -
   2 G~ from split operands -- BF16: each vector as hi + lo parts, three
   MMAs (d <= 192); FP8: each vector scaled by a power of two and written as
   E4M3 parts hi + mid + lo, six MMAs (d <= 256) -- with a stated bound
   |d~ - d| <= err_c (|a|^2 + |b|^2) against the reference's FP32 distance
   d; a pair side is proposed when its lower bound passes the target's
   filter, and the merge computes the exact FP32 distance of every proposal
   that can still enter the top K, so the graphs equal the FP32 join's. */
typedef enum {
    NNM_JOIN_AUTO = 0,   /* u8 tensor cores for integer data, else FP32 */
    NNM_JOIN_FP32 = 1,   /* FP32 CUDA cores: the reference's sequential sums */
    NNM_JOIN_TENSOR = 2, /* tensor cores: u8, else BF16 hi + lo; NNM_ERR_INVALID when neither applies */
    NNM_JOIN_FP8 = 3     /* tensor cores, FP8 (E4M3) hi + mid + lo with per-vector power-of-two scales */
} nnm_join_kernel;

/* Initial graphs.  NNM_INIT_LEARNED (no counterpart in the reference) needs
   NNM_RNG_FAST and a model set with nnm_set_init_model: every row's initial
   pool is the k nearest among the rows next to it in several orderings of
   the model's 32-bit codes, and the cross-leaf samples of a merge are the
   nearest rows of the other leaves in those orderings. */
typedef enum {
    NNM_INIT_RANDOM = 0, /* the reference's random graphs (getRndSds) */
    NNM_INIT_LEARNED = 1 /* candidates bucketed by the learned codes */
} nnm_init_mode;

/* How nnm_merge_leaves merges its built leaves (no counterpart in the
   reference, which merges two sub-graphs).  ALL: one multi-way merge, every
   row taking cross samples from all other leaves.  TREE (needs
   NNM_RNG_FAST): bottom-up pairwise S-Merges, leaf 2i with leaf 2i + 1, level
   after level, all pairs of a level batched into one NN-Descent run. */
typedef enum {
    NNM_MERGE_ALL = 0,
    NNM_MERGE_TREE = 1
} nnm_merge_order;

typedef struct {
    uint32_t seed;        /* clock value the reference's time(NULL) seeding is frozen at */
    uint32_t rng_mode;    /* nnm_rng_mode */
    uint32_t metric;      /* nnm_metric */
    uint32_t sample_cap;  /* smplNum, reverse-list cap (kgraph.cpp:100): 100 */
    float delta;          /* convergence threshold (abstractgraph.cpp:4): 0.002 */
    uint32_t max_iter;    /* 0: iterate until converged, as the reference */
    uint32_t exact_trace; /* nonzero: record the reference's float mean every iteration */
    uint32_t join_kernel; /* nnm_join_kernel */
    uint32_t init;        /* nnm_init_mode */
    uint32_t audit;       /* nonzero: the reduced-precision joins also compute every pair's exact
                             distance and fail the call (NNM_ERR_CAPACITY) if one lies outside
                             the stated bound -- a test of the bound, slow */
    uint32_t merge_order; /* an nnm_merge_order, read by nnm_merge_leaves */
    uint32_t no_graph;    /* nonzero: launch every kernel directly; zero: the fast tier replays
                             each NN-Descent iteration as a CUDA graph where it can */
    uint32_t tile_rows;   /* u8 tensor-core join: the longest sample lists (entries of a row's
                             new + old lists) joined in tensor-core tiles, 32, 64 or 128 (0: 128);
                             longer lists go to the dp4a pair kernel.  Same graphs either way. */
    uint32_t reserved[3];
} nnm_opts;

typedef struct {
    uint64_t ncmps;          /* distance evaluations of the measured phase, as the reference counts */
    uint64_t sub_ncmps;      /* merges: distance evaluations of the sub-graph builds */
    uint32_t iterations;     /* NN-Descent iterations, all loops */
    uint32_t n_trace;        /* entries written to trace */
    float trace[256];        /* convergence mean per iteration, in order */
    double device_ms;        /* device time of the call (CUDA events) */
} nnm_stats;

/* H-Merge search hierarchy: layer g has nrows[g] rows (a prefix of the data
 * set); row i's neighbours are adj[g][off[g][i] .. off[g][i+1]).  Arrays are
 * allocated by the library (host memory) and freed by nnm_layers_free. */
typedef struct {
    uint32_t nlayers;
    uint32_t nrows[16];
    uint64_t *off[16];
    uint32_t *adj[16];
} nnm_layers;

typedef struct nnm_ctx nnm_ctx;

void nnm_opts_default(nnm_opts *opts);
const char *nnm_status_string(int status);
const char *nnm_last_error(const nnm_ctx *ctx);

/* Creates a context on CUDA device `device`. */
int nnm_ctx_create(int device, nnm_ctx **out);
int nnm_ctx_destroy(nnm_ctx *ctx);

/* KGraph::buildKGraph(mata, K, N, D) (kgraph.cpp:217-245) and the pools it
 * leaves (Neighborx{id,dist,flag}, kgraph.h:24-36).  x: n x d row-major.
 * ids/dists/flags: n x k outputs (any may be NULL). */
int nnm_kgraph_build(nnm_ctx *ctx, const float *x, uint64_t n, uint32_t d, uint32_t k,
                     const nnm_opts *opts, uint32_t *ids, float *dists, uint8_t *flags,
                     nnm_stats *stats);
int nnm_kgraph_build_dev(nnm_ctx *ctx, const float *x_dev, uint64_t n, uint32_t d, uint32_t k,
                         const nnm_opts *opts, uint32_t *ids_dev, float *dists_dev,
                         uint8_t *flags_dev, nnm_stats *stats);

/* Smerge::buildKGraph (smerge.cpp:46-91): NN-Descent on the two halves split
 * at n*5/10, cross sampling, cross-half NN-Descent, merge2one. */
int nnm_smerge(nnm_ctx *ctx, const float *x, uint64_t n, uint32_t d, uint32_t k,
               const nnm_opts *opts, uint32_t *ids, float *dists, uint8_t *flags,
               nnm_stats *stats);

/* Jmerge::buildKGraph (jmerge.cpp:43-80): NN-Descent on the first half,
 * joint NN-Descent with the raw second half, merge2one. */
int nnm_jmerge(nnm_ctx *ctx, const float *x, uint64_t n, uint32_t d, uint32_t k,
               const nnm_opts *opts, uint32_t *ids, float *dists, uint8_t *flags,
               nnm_stats *stats);

/* The two halves of nnm_merge_leaves_dev on the fast tier (rng_mode
 * NNM_RNG_FAST), for a build whose leaves are split over several GPUs (no
 * counterpart in the reference).  nnm_build_leaves_dev: NN-Descent on
 * nleaf consecutive leaves of x (sizes summing to n) as nnm_merge_leaves
 * builds them, without the merge; leaf0 is the index of the first of these
 * leaves among all leaves of the whole build (it fixes their random draws);
 * ids are local to x's rows.  nnm_merge_prebuilt_dev: the merge of
 * nnm_merge_leaves over leaves whose graphs are given (n x k ids of x's rows,
 * distances; ids outside [0, n) are rejected).  Building all leaves in one
 * call and merging them gives nnm_merge_leaves_dev's graph bit for bit.
 * All pointers are device pointers. */
int nnm_build_leaves_dev(nnm_ctx *ctx, const float *x_dev, uint64_t n, uint32_t d, uint32_t k,
                         const uint32_t *leaf_sizes, uint32_t nleaf, uint32_t leaf0, const nnm_opts *opts,
                         uint32_t *ids_dev, float *dists_dev, nnm_stats *stats);
int nnm_merge_prebuilt_dev(nnm_ctx *ctx, const float *x_dev, uint64_t n, uint32_t d, uint32_t k,
                           const uint32_t *leaf_sizes, uint32_t nleaf, const nnm_opts *opts,
                           const uint32_t *ids_in_dev, const float *dists_in_dev, uint32_t *ids_dev,
                           float *dists_dev, uint8_t *flags_dev, nnm_stats *stats);

/* Staged merge: the steps of Smerge::buildKGraph (smerge.cpp:46-91) and
 * Jmerge::buildKGraph (jmerge.cpp:43-80) as separate calls on one session,
 * for callers that drive AbstractMerge's interface (abstractmerge.h:25-37)
 * step by step.  The session holds the vectors and the pools (the
 * reference's MergeType egraph) on the device and behaves as one reference
 * process: the std::rand() stream starts from srand(opts.seed) at
 * nnm_merge_create and continues across the steps; each phase the
 * reference seeds with time(NULL) draws from mt19937(opts.seed).  Run in
 * the reference's order, the steps give the graphs of nnm_smerge /
 * nnm_jmerge bit for bit.  Reference streams only (opts.rng_mode
 * NNM_RNG_EXACT); opts.join_kernel selects the join kernel as elsewhere. */
typedef struct nnm_merge nnm_merge;

/* Which reference class's local join (and initial graph) a step runs. */
typedef enum {
    NNM_MERGE_SMERGE = 1, /* Smerge::localJoin (smerge.cpp:212-235): groups differ */
    NNM_MERGE_JMERGE = 2  /* Jmerge::localJoin (jmerge.cpp:178-203): groups differ or either is 1 */
} nnm_merge_kind;

/* AbstractMerge::InitialMemory(mata, k, n, d) (abstractmerge.cpp:25-35):
 * x is n x d row-major host memory, copied to the device. */
int nnm_merge_create(nnm_ctx *ctx, const float *x, uint64_t n, uint32_t d, uint32_t k,
                     const nnm_opts *opts, nnm_merge **out);
/* KGraph::buildKGraph on cutMat(mata, b, e) (smerge.cpp:56-68): NN-Descent
 * on rows [b, e) alone, continuing the session's std::rand() stream.
 * graph (host, may be NULL): (e - b) x k ids local to the sub-range, as the
 * reference's buildKGraph returns them; ncmps (may be NULL): its distance
 * evaluations. */
int nnm_merge_subgraph(nnm_merge *m, uint32_t b, uint32_t e, uint32_t *graph, uint64_t *ncmps);
/* AbstractMerge::InitSGraph(b, graph, gid, size) (abstractmerge.cpp:55-76):
 * rows [b, b + size) take the host graph's local ids + b in its order,
 * flagged new with group id gid (0 or 1), distances recomputed. */
int nnm_merge_init_sgraph(nnm_merge *m, uint32_t b, const uint32_t *graph, uint32_t gid, uint32_t size);
/* Smerge::InitialGraph (smerge.cpp:94-209) or Jmerge::InitialGraph
 * (jmerge.cpp:83-176) with preSize = pre. */
int nnm_merge_initial_graph(nnm_merge *m, uint32_t kind, uint32_t pre);
/* AbstractMerge::nnDescent (abstractmerge.cpp:78-192) with the local join of
 * `kind`, until the reference's convergence test passes (or opts.max_iter).
 * stats (may be NULL): the step's distance evaluations (ncmps), its
 * iterations and convergence means. */
int nnm_merge_nndescent(nnm_merge *m, uint32_t kind, uint32_t pre, nnm_stats *stats);
/* AbstractMerge::merge2one(sz) (abstractmerge.cpp:232-277): rows [0, sz). */
int nnm_merge_merge2one(nnm_merge *m, uint32_t sz);
/* The pools (n x k; any output may be NULL), host memory. */
int nnm_merge_read(nnm_merge *m, uint32_t *ids, float *dists, uint8_t *flags);
int nnm_merge_free(nnm_merge *m);

/* S-Merge over `nleaf` consecutive leaves of the given sizes (sum = n): every
 * leaf is built with NN-Descent, every row keeps its best k - k/2 entries
 * and samples k/2 ids from the other leaves, and the join pairs only rows of
 * different leaves.  With two leaves of sizes n*5/10 and n - n*5/10 this is
 * nnm_smerge (Smerge::buildKGraph); the reference has no G > 2 form. */
int nnm_merge_leaves(nnm_ctx *ctx, const float *x, uint64_t n, uint32_t d, uint32_t k,
                     const uint32_t *leaf_sizes, uint32_t nleaf, const nnm_opts *opts,
                     uint32_t *ids, float *dists, uint8_t *flags, nnm_stats *stats);
int nnm_merge_leaves_dev(nnm_ctx *ctx, const float *x_dev, uint64_t n, uint32_t d, uint32_t k,
                         const uint32_t *leaf_sizes, uint32_t nleaf, const nnm_opts *opts,
                         uint32_t *ids_dev, float *dists_dev, uint8_t *flags_dev,
                         nnm_stats *stats);

/* LyNNDescent::buildhgraph(src, dst, grd, K, M) (lynndescent.cpp:735-831):
 * H-Merge from 64 rows by doubling J-Merges; DPG layers at 64, 512, 4096,
 * 32768 and n (lynndescent.cpp:502-544, :640-713).  layers may be NULL. */
int nnm_hmerge_build(nnm_ctx *ctx, const float *x, uint64_t n, uint32_t d, uint32_t k, uint32_t m,
                     const nnm_opts *opts, uint32_t *ids, float *dists, uint8_t *flags,
                     nnm_layers *layers, nnm_stats *stats);
void nnm_layers_free(nnm_layers *layers);

/* LySearch::knnSearch per-query steps (lysearch.cpp:363-437) for a batch of
 * queries at one beam width `topk` (the reference's result size equals its
 * beam): entry point rand() % nrows[0] after srand(opts.seed), greedy
 * descent on layers 0..L-2, best-first beam search on layer L-1
 * (nndHNSWSrch, lysearch.cpp:236-322).  out_ids/out_dists: nq x topk,
 * ascending distance; ncmps counts distance evaluations. */
int nnm_search(nnm_ctx *ctx, const float *x, uint64_t n, uint32_t d, const nnm_layers *layers,
               const float *q, uint64_t nq, uint32_t topk, const nnm_opts *opts,
               uint32_t *out_ids, float *out_dists, uint64_t *ncmps);

/* The search hierarchy in device memory, for nnm_search_noalloc: the layout
 * of nnm_layers with device pointers. */
typedef struct {
    uint32_t nlayers;
    uint32_t nrows[16];
    const uint64_t *off[16];
    const uint32_t *adj[16];
} nnm_dev_layers;

/* Search without device allocation.  No counterpart in the reference: it
 * exists for callers that cannot call cudaMalloc -- code running inside a
 * memory pool owned by another framework, a serving process whose device
 * memory budget is fixed at start-up, or a latency path that must not pay
 * the implicit synchronisation of cudaMalloc/cudaFree.  Same results as
 * nnm_search.  The caller passes every input and output in device memory
 * (x: n x d row-major, q: nq x d, out_ids / out_dists: nq x topk) and a CUDA
 * stream (NULL: the legacy default stream); the call allocates nothing.  Its
 * scratch is a fixed array of about 16 MiB in the library's device image,
 * which every GPU that loads the library holds until the process exits.
 * Limits: the last layer has at most 2^20 rows, topk <= 1024, d <= 4096
 * (NNM_ERR_INVALID beyond them); a query needing more than 12288 candidate
 * heap entries fails the call with NNM_ERR_CAPACITY.  The first call on a
 * device looks up the array's device address (cudaGetSymbolAddress) and
 * caches it; under lazy module loading that first call is also where the
 * ~16 MiB are claimed on the device, so a process with a fixed memory
 * budget should make one warm-up call at start-up.  That first call also
 * zeroes the visited bitmaps (8 MiB); later calls zero only the 256-byte
 * counters, since every query clears the bits it set, unless the previous
 * call on the device returned before its kernel finished.  Every call ends by
 * copying its counters to the host and waiting for its stream, so no call
 * may be made while its stream is being captured into a CUDA graph.  All
 * calls share the one array: calls that overlap on the GPU race and must
 * not be issued.  The hierarchy is read as given and is not checked: off[g]
 * must be non-decreasing with off[g][nrows[g]] within adj[g], and every id
 * in adj[g] below nrows[g] (ids out of range end the call with
 * NNM_ERR_CAPACITY after partial output; offsets out of range read out of
 * bounds). */
int nnm_search_noalloc(const float *x_dev, uint64_t n, uint32_t d, const nnm_dev_layers *layers,
                       const float *q_dev, uint64_t nq, uint32_t topk, uint32_t seed, uint32_t metric,
                       uint32_t *out_ids_dev, float *out_dists_dev, uint64_t *ncmps, void *stream);

/* Learned initialisation (no counterpart in the reference).  A 2-layer MLP
 *   u = x * in_scale + in_shift,  h = relu(W1 u + b1),  z = W2 h + b2,
 * d_in = d (<= 256) -> 256 -> 32, evaluated with BF16-rounded weights and
 * FP32 accumulation; a row's code is the sign bits of z (bit o = z_o > 0).
 * Weights are row-major: w1 is 256 x d_in, w2 is 32 x 256.  Training
 * minimises the triplet loss mean(max(0, margin + |t_a - t_p|^2 -
 * |t_a - t_n|^2)), t = tanh(z), over anchors a, graph neighbours p and
 * random rows n, with Adam on FP32 master weights. */
#define NNM_MLP_HIDDEN 256
#define NNM_MLP_OUT 32
typedef struct {
    uint32_t d_in;
    float in_scale, in_shift;
    float *w1, *b1, *w2, *b2; /* caller-owned host arrays */
} nnm_mlp;

typedef struct {
    uint32_t steps;   /* optimiser steps: 400 */
    uint32_t batch;   /* triplets per step: 2048 */
    float lr;         /* Adam step size: 2e-3 */
    float margin;     /* 16 */
    uint32_t seed;
    uint32_t reserved[7];
} nnm_train_opts;

void nnm_train_opts_default(nnm_train_opts *o);
/* Trains `model` in place (its arrays hold the initial weights) on triplets
 * drawn from the k-NN graph `graph` (n x k ids) of x (n x d).  loss_trace:
 * `steps` floats or NULL. */
int nnm_mlp_train(nnm_ctx *ctx, const float *x, uint64_t n, uint32_t d, const uint32_t *graph, uint32_t k,
                  const nnm_train_opts *opts, nnm_mlp *model, float *loss_trace);
/* Loss and gradients (w.r.t. the BF16-rounded weights) of the triplet loss
 * over the given triplets (ntrip x 3 row indices of x: anchor, positive,
 * negative); grad has the model's shapes. */
int nnm_mlp_grad(nnm_ctx *ctx, const nnm_mlp *model, const float *x, uint64_t n, uint32_t d,
                 const uint32_t *triplets, uint32_t ntrip, float margin, float *loss, nnm_mlp *grad);
/* Codes (n) and, when z is not NULL, the outputs (n x 32) of x. */
int nnm_mlp_codes(nnm_ctx *ctx, const nnm_mlp *model, const float *x, uint64_t n, uint32_t d,
                  uint32_t *codes, float *z);
/* The model NNM_INIT_LEARNED builds use (copied to the device); NULL clears it. */
int nnm_set_init_model(nnm_ctx *ctx, const nnm_mlp *model);

/* Serving (LySearch::knnSearch's per-query steps, lysearch.cpp:363-437, on a
 * resident index).  nnm_index_create copies the vectors and the hierarchy
 * to the device once; nnm_index_search then runs batches of queries, each
 * with its own beam width (the reference's topk, lysearch.cpp:236: result
 * heap size), and returns the best out_k results of every query, ascending
 * (padded with id 0xffffffff, distance 0 when a beam holds fewer).
 *
 * Kernels: NNM_SERVE_EXACT is the kernel of nnm_search (the reference's
 * heaps and float sums bit for bit; with beams == NULL, beam == out_k and
 * the default entry it gives nnm_search's results).  NNM_SERVE_FAST
 * computes each distance with a whole warp (coalesced rows, a different
 * float summation order) and keeps the beam as a sorted array in shared
 * memory in place of the two heaps: the same best-first expansion and
 * stopping rule, ties between equal distances broken by id.
 *
 * Entry points: NNM_ENTRY_DEFAULT starts every query at rand() % nrows[0]
 * after srand(seed) and descends greedily from layer 0, as the reference.
 * NNM_ENTRY_LEARNED (no counterpart in the reference) runs the entry
 * network set with nnm_index_set_entry_model: the rows of its layer with
 * the `probes` largest scores are measured, the nearest of them starts the
 * greedy descent on that layer. */
typedef struct nnm_index nnm_index;

typedef enum { NNM_SERVE_EXACT = 0, NNM_SERVE_FAST = 1 } nnm_serve_mode;
typedef enum {
    NNM_ENTRY_DEFAULT = 0, /* LySearch::knnSearch: one global entry, greedy descent from layer 0 */
    NNM_ENTRY_LEARNED = 1, /* the entry network's probes, descent from their layer */
    NNM_ENTRY_FLAT = 2     /* LySearch::nndFlatSrch (lysearch.cpp:439-520): no descent; the beam starts
                              with `beam` distinct rows of the last layer drawn by getRndSds from a fresh
                              mt19937(seed) (the reference reseeds per query from its clock); every
                              beam width must be at most the last layer's rows */
} nnm_entry_mode;

typedef struct {
    uint64_t ncmps;       /* distance evaluations, all queries (entry probes included) */
    uint64_t expansions;  /* beam expansions (nodes whose lists were read), all queries */
    double device_ms;     /* device time of the call's kernels (CUDA events) */
    double predict_ms;    /* of which the entry network */
} nnm_search_stats;

/* The index keeps pointers to nothing the caller owns; it belongs to ctx
 * (its stream and device) and must be freed before ctx is destroyed. */
int nnm_index_create(nnm_ctx *ctx, const float *x, uint64_t n, uint32_t d, const nnm_layers *layers,
                     uint32_t seed, uint32_t metric, nnm_index **out);
int nnm_index_free(nnm_index *ix);
/* beams: nq widths (1..1024) or NULL for `beam` everywhere; out_k <= every width.
 * q, beams, out_ids, out_dists: host arrays (nq x d, nq, nq x out_k). */
int nnm_index_search(nnm_index *ix, const float *q, uint64_t nq, const uint32_t *beams, uint32_t beam,
                     uint32_t out_k, uint32_t serve_mode, uint32_t entry_mode, uint32_t *out_ids,
                     float *out_dists, nnm_search_stats *stats);
/* The same with q, beams, out_ids and out_dists in device memory. */
int nnm_index_search_dev(nnm_index *ix, const float *q_dev, uint64_t nq, const uint32_t *beams_dev,
                         uint32_t beam, uint32_t out_k, uint32_t serve_mode, uint32_t entry_mode,
                         uint32_t *out_ids_dev, float *out_dists_dev, nnm_search_stats *stats);

/* NNM_SERVE_FAST only: a step of a query with beam width ef expands its
 * min(width, max(1, ef / 64)) nearest unexpanded beam entries together and
 * reads their lists as one sequence, so their memory latencies overlap
 * (1: strict best-first order, as the reference).  width is in 1..4,
 * default 4; wider steps may expand a few more nodes. */
int nnm_index_set_width(nnm_index *ix, uint32_t width);
/* Autotuner of the width: times NNM_SERVE_FAST on the sample queries (host
 * arrays, as nnm_index_search takes them) at widths 1..4, `repeats` times
 * each (the fastest kept), sets the fastest and returns it in *width;
 * ms (4 entries, may be NULL) gets each width's device time. */
int nnm_index_tune_width(nnm_index *ix, const float *q, uint64_t nq, const uint32_t *beams, uint32_t beam,
                         uint32_t out_k, uint32_t entry_mode, uint32_t repeats, uint32_t *width, double *ms);

/* Entry-point network (no counterpart in the reference): its classes are
 * rows 0..C-1 of the data set (C <= NNM_ENTRY_MAX_CLASSES), and a learned
 * search starts its greedy descent on the first layer that holds them all.
 * nnm_index_entry_layer gives the default: the deepest layer with at most
 * NNM_ENTRY_MAX_CLASSES rows (C = its rows), else layer 0 with C = 4096.
 *   u = x * in_scale + in_shift,  h = relu(W1 u + b1),  s = W2 h + b2,
 * d_in (<= 256) -> 256 -> C, BF16-rounded weights, FP32 accumulation
 * (inference also rounds h to BF16, the tensor-core operand).
 * Training minimises the softmax cross-entropy of s against the nearest
 * class row (squared L2) of each training row, with Adam on FP32 master
 * weights.  w1 is 256 x d_in, w2 is C x 256 (row-major). */
#define NNM_ENTRY_MAX_CLASSES 4096
typedef struct {
    uint32_t d_in, n_classes;
    float in_scale, in_shift;
    float *w1, *b1, *w2, *b2; /* caller-owned host arrays */
} nnm_entry_mlp;

int nnm_index_entry_layer(const nnm_index *ix, uint32_t *layer, uint32_t *n_classes);
/* Scores (n x C) of x (n x d) as the search computes them: h rounded to
 * BF16, s = W2 h + b2 on the tensor cores (BF16 operands, FP32 sums). */
int nnm_entry_forward(nnm_ctx *ctx, const nnm_entry_mlp *model, const float *x, uint64_t n, uint32_t d,
                      float *scores);
/* The probes a learned search takes for x: the classes of each row's
 * `probes` (1..min(8, C)) largest scores, ties to the lower class, in
 * descending order (n x probes). */
int nnm_entry_probes(nnm_ctx *ctx, const nnm_entry_mlp *model, const float *x, uint64_t n, uint32_t d,
                     uint32_t probes, uint32_t *out);
/* Mean cross-entropy over the rows of x against labels (n classes) and its
 * gradients w.r.t. the BF16-rounded weights; grad has the model's shapes. */
int nnm_entry_grad(nnm_ctx *ctx, const nnm_entry_mlp *model, const float *x, uint64_t n, uint32_t d,
                   const uint32_t *labels, float *loss, nnm_entry_mlp *grad);
/* Trains `model` in place on rows of the index's data set (a seeded sample
 * of at most 262144 rows, labelled on the device by brute force); steps,
 * batch, lr and seed come from opts (margin is unused).  loss_trace: `steps`
 * floats or NULL. */
int nnm_entry_train(nnm_index *ix, nnm_entry_mlp *model, const nnm_train_opts *opts, float *loss_trace);
/* The network NNM_ENTRY_LEARNED uses (copied to the device), probes in
 * 1..min(8, C); NULL clears it. */
int nnm_index_set_entry_model(nnm_index *ix, const nnm_entry_mlp *model, uint32_t probes);

/* Recall@atop of a k-NN graph (Evaluator::getKGraphRecall,
 * evaluator.cpp:258-295, with the ground truth computed on the device): for
 * each of the `nrows` listed rows, the share of its first atop ids (atop
 * <= 16) whose distance is at most the row's atop-th exact nearest distance
 * (brute force over all other rows, the reference's FP32 sums; rows tied at
 * that distance count as hits).  x: n x d, ids: n x k, rows: nrows, all host.
 * d <= 512. */
int nnm_graph_recall(nnm_ctx *ctx, const float *x, uint64_t n, uint32_t d, const uint32_t *ids, uint32_t k,
                     const uint32_t *rows, uint32_t nrows, uint32_t atop, double *recall);

/* Autotuner (no counterpart in the reference) for nnm_merge_leaves_dev:
 * trial builds on the first sample_rows rows of x (leaf sizes scaled to
 * the sample) over a grid of reverse-sample caps (smplNum) and convergence
 * thresholds, each scored with nnm_graph_recall on eval_rows seeded rows
 * and timed with CUDA events; the chosen setting is the fastest whose
 * sample recall@10 is at least target_recall + margin (else the one of the
 * highest recall).  `tuned` is `base` with sample_cap and delta replaced.
 * A sample smaller than the data set usually reads a higher recall than the
 * full build reaches (its clusters are sparser); sample_rows = n tunes on
 * the build itself. */
typedef struct {
    float target_recall;  /* 0.95 */
    float margin;         /* 0.005: the sample's recall is read above the full build's */
    uint32_t sample_rows; /* 200000 (at most n) */
    uint32_t eval_rows;   /* 1000 */
    uint32_t repeats;     /* timed builds per setting, the fastest kept: 2 */
    uint32_t reserved[7];
} nnm_tune_opts;

#define NNM_TUNE_MAX_TRIALS 32
typedef struct {
    uint32_t sample_cap;
    float delta;
    float recall;       /* on the sample */
    uint32_t tile_rows; /* nnm_opts.tile_rows of the trial */
    double ms;          /* device time of the sample build */
} nnm_tune_trial;

typedef struct {
    uint32_t ntrials, chosen; /* trials run; index of the chosen one */
    nnm_tune_trial trials[NNM_TUNE_MAX_TRIALS];
} nnm_tune_result;

void nnm_tune_opts_default(nnm_tune_opts *o);
int nnm_autotune_merge_leaves(nnm_ctx *ctx, const float *x_dev, uint64_t n, uint32_t d, uint32_t k,
                              const uint32_t *leaf_sizes, uint32_t nleaf, const nnm_opts *base,
                              const nnm_tune_opts *topts, nnm_opts *tuned, nnm_tune_result *result);

/* Profiling (no counterpart in the reference, which times whole builds with
 * boost::timer): while enabled, the engine records CUDA events around its
 * local-join and top-K merge kernels and accumulates their device time and
 * algorithmic bytes / flops.  nnm_profile_get writes them as a JSON object. */
int nnm_profile_enable(nnm_ctx *ctx, int on);
int nnm_profile_get(const nnm_ctx *ctx, char *buf, uint64_t buflen);
/* Kernel launches made by this library in this process so far. */
uint64_t nnm_launch_count(void);

#ifdef __cplusplus
}
#endif
#endif
