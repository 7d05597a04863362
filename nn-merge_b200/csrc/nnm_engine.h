// Host-side engine state shared by the NN-Descent driver (nndescent.cu),
// the graph builders (builders.cu), DPG (dpg.cu), search (search.cu) and the
// C ABI (capi.cpp).
#pragma once
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "nnm_nnd.h"
#include "nnm_rng.h"

namespace nnm {

// Grow-only device allocation.
struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    cudaError_t ensure(size_t b) {
        if (b <= bytes) return cudaSuccess;
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
        cudaError_t e = cudaMalloc(&p, b ? b : 16);
        if (e == cudaSuccess) bytes = b;
        return e;
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
    template <class T> T* as() const { return static_cast<T*>(p); }
};

// Scratch for one NN-Descent iteration, sized for the largest graph seen.
struct Workspace {
    DevBuf rcnt, rcur, rtot, roff, rseg, rscr, rcount, rofs, rbuf;
    DevBuf cntpos, bcnt, bcur, boff, bucket, bigrev, nflag, scan_tmp;
    DevBuf npairs, poff, pd, tiers, erows;
    DevBuf kth;  // every row's K-th distance, gathered per iteration
    DevBuf rtier;  // every row's join tier (k_shuffle_append), binned by k_tier_lists
    DevBuf draws, counters, misc;
    DevBuf mlp_err;  // the code network's tensor-core inference: a wait that ran out
    void release_all() {
        DevBuf* all[] = {&rcnt, &rcur, &rtot, &roff, &rseg, &rscr, &rcount, &rofs, &rbuf, &cntpos, &bcnt, &bcur,
                         &boff, &bucket, &bigrev, &nflag, &scan_tmp, &npairs, &poff, &pd, &tiers, &erows, &kth, &rtier,
                         &draws, &counters, &misc, &mlp_err};
        for (auto* b : all) b->release();
    }
};

// Device storage of a graph under construction (owned buffers).
struct GraphStore {
    DevBuf pid, pdist, cpid, cpdist, newL, oldL, newlen, oldlen, rnewT, roldT, rnewTlen, roldTlen, x;
    DevBuf xq, nrm;  // operand copy of the vectors and their squared norms (tensor-core join)
    DevBuf scl;      // FP8 operands: per-row inverse scales
    DevBuf codes, vkeys, vpos, voff;  // learned codes and their sorted views
    DevBuf vfence;                    // every 256th key of each sorted view segment
    void release() {
        DevBuf* all[] = {&pid, &pdist, &cpid, &cpdist, &newL, &oldL, &newlen, &oldlen,
                         &rnewT, &roldT, &rnewTlen, &roldTlen, &x, &xq, &nrm, &scl,
                         &codes, &vkeys, &vpos, &voff, &vfence};
        for (auto* b : all) b->release();
    }
};

// Device time and algorithmic traffic of one kernel class, accumulated
// while profiling is on (CUDA events on the engine's stream).
struct KStat {
    uint64_t launches = 0;
    double ms = 0.0, bytes = 0.0, flops = 0.0;
    double tensor_ops = 0.0;  // multiply-adds x 2 issued to the tensor cores (whole 128 x 128 tiles)
};

struct DevMlp;
struct CodeViews;

struct Ctx {
    int device = 0;
    DevMlp* init_model = nullptr;  // learned-initialisation model (owned)
    bool prof = false;
    GraphStore store;  // graph arrays, reused across calls (grow-only)
    KStat kjoin, kemit, kmerge;
    uint64_t join_rows[5] = {};  // joined rows per list-size tier (while profiling)
    uint64_t join_rows_tc = 0;   // of which on the tensor cores
    // per-iteration record while profiling (the most recent iterations)
    struct IterLog {
        uint32_t n, rows[5];
        uint64_t pairs, proposals, flags, ncmps, sum_s;
        float ms_join, ms_emit, ms_merge;
    };
    std::vector<IterLog> iter_log;
    // audit of the reduced-precision joins (while profiling): the largest
    // |d~ - d| / (|a|^2 + |b|^2) seen and the bound coefficient it is held to
    float audit_max = 0.f, audit_err_c = 0.f;
    // reduced-precision joins (while profiling): proposals carrying d~, and
    // those the merge computed exactly
    uint64_t approx_props = 0, rechecks = 0;
    cudaEvent_t ev[8] = {};
    // executable whole-iteration graphs of the fast tier, one per join mode,
    // refreshed by cudaGraphExecUpdate at each NN-Descent call
    struct IterGraph {
        cudaGraphExec_t exec = nullptr;
        uint64_t launches = 0;
    } iter_graph[4];
    cudaStream_t stream = nullptr;
    Workspace ws;
    IterCounters* h_counters = nullptr;  // pinned
    std::string last_error;
    double last_device_ms = 0.0;
    uint64_t kernel_launches = 0;
};

// A graph under construction: raw device pointers, so that a sub-graph
// (an S-/J-Merge leaf) can run NN-Descent in place inside its parent's
// arrays.
struct GraphDev {
    uint32_t n_cap = 0, n = 0, K = 0, d = 0, dp = 0;
    int metric = L2;
    const float* x = nullptr;       // n_cap x dp on the device
    // Tensor-core join (set by tc_prepare when it applies): n_cap x kq bytes
    // of u8 vectors (kq = d rounded up to 32) or BF16 vectors (kq = 2 x d
    // rounded up to 16), zero padded, and squared norms.
    const uint8_t* xq = nullptr;
    const uint32_t* nrm = nullptr;
    uint32_t kq = 0;
    uint32_t tc_kind = 0;  // 0: u8 copy (exact); 1: BF16 hi + lo parts; 2: FP8 hi + mid + lo parts
    float err_c = 0.f;     // reduced precision: |d~ - d| <= err_c (|a|^2 + |b|^2)
    const float* scl = nullptr;  // FP8: per-row inverse scales 2^-e
    uint32_t join_kernel = 0;       // nnm_join_kernel
    // Learned initialisation: codes of rows [0, n_cap) and, inside a merge,
    // the parent's code views with this graph's leaf index.
    uint32_t init = 0;              // nnm_init_mode
    const uint32_t* codes = nullptr;
    const CodeViews* views = nullptr;
    uint32_t view_leaf = 0;
    uint32_t* pid = nullptr;        // pools, n_cap x K
    float* pdist = nullptr;
    uint32_t* cpid = nullptr;       // compensation lists, n_cap x K (cut used)
    float* cpdist = nullptr;
    uint32_t cut = 0;
    uint32_t *newL = nullptr, *oldL = nullptr, *newlen = nullptr, *oldlen = nullptr;  // sample lists
    uint32_t capn = 0, capo = 0;
    uint32_t *rnewT = nullptr, *roldT = nullptr, *rnewTlen = nullptr, *roldTlen = nullptr;  // H-Merge carry
    bool carry = false;        // lists of the last converged iteration are still present
    GlibcBase gbase;
    uint64_t gpos = 0;         // std::rand() outputs consumed since srand(seed)
    uint32_t seed = 0;
    uint32_t smpl = 100;
    float delta = 0.002f;
    uint32_t max_iter = 0;     // 0: iterate until the reference's convergence test passes
    bool exact_trace = false;  // record the reference's float mean every iteration
    bool audit = false;        // reduced-precision joins: check every pair against its bound
    bool merge_tree = false;   // multi-leaf merges: bottom-up pairwise levels instead of all at once
    bool no_graph = false;     // launch every kernel directly (no CUDA graphs)
    uint32_t tile_rows = 128;  // u8 tensor-core join: longest lists in tensor-core tiles (32, 64, 128)
    // Fast tier: counter-based random draws (Philox keyed by the seed) in
    // place of the reference's sequential streams, so the initial graphs and
    // samples are drawn on the device and reverse lists need no ordering.
    bool fast = false;
    uint32_t phase = 0;        // Philox counter of the next sampling phase
    uint64_t ncmps = 0;
    uint32_t iters = 0;
    std::vector<float> trace;
};

// Philox phases of the fast tier's multi-leaf build: the leaves' initial
// draws use phases 0 .. nleaf - 1, the leaf run's iterations start at
// LEAF_PHASE0, the merge's draws at MERGE_PHASE0 -- so that the merge does
// not depend on how the leaves were built (one run or one per rank).
constexpr uint32_t LEAF_PHASE0 = 1u << 24;
constexpr uint32_t MERGE_PHASE0 = 1u << 28;

#define NNM_CUDA_TRY(expr)                                                         \
    do {                                                                           \
        cudaError_t _e = (expr);                                                   \
        if (_e != cudaSuccess) {                                                   \
            ctx.last_error = std::string(#expr) + ": " + cudaGetErrorString(_e);   \
            return _e == cudaErrorMemoryAllocation ? 4 : 3;                        \
        }                                                                          \
    } while (0)

// Allocates pools and list storage for up to n_cap rows into `store` and
// points g at it.  with_carry sizes the lists for one level of carried-over
// sample lists and keeps the truncated reverse lists (H-Merge).
int graph_alloc(Ctx& ctx, GraphStore& store, GraphDev& g, bool with_carry);
// Runs NN-Descent iterations until the reference's convergence test passes
// (or max_iter).  split: first row of group 1 for the group id of reverse
// entries; leaf_off/nleaf: group boundaries for MODE_SMERGE.
int run_nndescent(Ctx& ctx, GraphDev& g, JoinMode mode, uint32_t split, uint32_t verse,
                  const uint32_t* d_leaf_off, uint32_t nleaf);

}  // namespace nnm
