// H-Merge hierarchy: DPG layers (dpg.cu) and batched LySearch (search.cu).
#pragma once
#include <cstdint>

#include "../../include/nnm.h"
#include "nnm_engine.h"

namespace nnm {

constexpr uint32_t SEARCH_MAX_BEAM = 1024;

// Device state of LyNNDescent::graph, which the reference never clears
// between layers (lynndescent.cpp:644): each layer starts from the previous
// layer's lists for the rows it already had.
struct DpgState {
    DevBuf gid, gdist, glen;      // current lists
    DevBuf g1id, g1dist, g1len;   // after the forward (occlusion) pass
    DevBuf sid, sdist, slen;      // snapshots guessed for the reverse pass
    DevBuf tid, tdist, tlen;      // snapshots recomputed from the guess
    DevBuf ecnt, ecur, eoff, ev, escr, bigseg, counters, tmp;
    uint32_t cap = 0, K = 0, M = 0, rows = 0, n_cap = 0;
    uint32_t last_rounds = 0;
    void release() {
        DevBuf* all[] = {&gid, &gdist, &glen, &g1id, &g1dist, &g1len, &sid, &sdist, &slen, &tid, &tdist,
                         &tlen, &ecnt, &ecur, &eoff, &ev, &escr, &bigseg, &counters, &tmp};
        for (auto* b : all) b->release();
    }
};

int dpg_init(Ctx& ctx, DpgState& s, uint32_t n_cap, uint32_t K, uint32_t M);
// Builds the DPG layer of g's current rows (LyNNDescent::dpg) and appends it
// to `out` (host CSR) when out is non-null.
int dpg_layer(Ctx& ctx, DpgState& s, GraphDev& g, nnm_layers* out);

struct DevEntry;  // entry network (entry.cu)

// A resident search hierarchy (nnm_index): vectors (n x dp), every layer's
// offsets rebased onto one adjacency array, and the search scratch.
struct IndexDev {
    uint32_t n = 0, d = 0, dp = 0, L = 0, metric = 0, seed = 0, entry = 0;
    uint32_t nrows[16] = {};
    uint64_t off_base[16] = {};
    DevBuf x, off, adj;
    DevBuf visited, vlist, cand, ctr;          // per-warp scratch and counters
    DevBuf qpad, beams, probes, hid, scores, out;  // per-call staging
    DevBuf flat_off, flat_pool;                // flat-search seeds of every beam width <= flat_max
    uint32_t flat_max = 0;
    DevEntry* net = nullptr;                   // entry network, owned
    uint32_t nprobe = 0, entry_layer = 0, n_classes = 0;
    uint32_t width = 4;  // fast kernel: most unexpanded entries expanded together
    void release();
};

// One batch of queries against an index; every pointer is device memory.
struct SearchReq {
    const float* q;           // nq x dp
    uint32_t nq;
    const uint32_t* beams;    // nq widths or null: `beam` for all
    uint32_t beam, beam_max, out_k;
    const uint32_t* probes;   // nq x nprobe rows of layer g0, or null: default entry
    uint32_t nprobe, g0;
    uint32_t flat;            // nndFlatSrch: getRndSds seeds of the last layer, no descent
    const uint32_t* flat_off;
    const uint32_t* flat_pool;
    uint32_t* out_ids;        // nq x out_k
    float* out_d;             // nq x out_k or null
};

int index_upload(Ctx& ctx, IndexDev& ix, const float* x, uint64_t n, uint32_t d, const nnm_layers* layers,
                 uint32_t seed, uint32_t metric);
// The caller zeroes ix.ctr (64 bytes: query counter, self-check flags,
// distance and expansion counts) before a run.
int index_run_exact(Ctx& ctx, IndexDev& ix, const SearchReq& r);
int index_run_fast(Ctx& ctx, IndexDev& ix, const SearchReq& r);
// Seeds of nndFlatSrch for every beam width up to beam_max (cached).
int index_flat_seeds(Ctx& ctx, IndexDev& ix, uint32_t beam_max);
// Waits for the stream, reads the distance and expansion counts of the last
// run and turns its self-check flags into an error.
int index_counters(Ctx& ctx, IndexDev& ix, uint64_t* ncmps, uint64_t* nexp);

int search_host(Ctx& ctx, const float* x, uint64_t n, uint32_t d, const nnm_layers* layers, const float* q,
                uint64_t nq, uint32_t topk, uint32_t seed, int metric, uint32_t* out_ids, float* out_dists,
                uint64_t* ncmps);

}  // namespace nnm
