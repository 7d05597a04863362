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

int search_host(Ctx& ctx, const float* x, uint64_t n, uint32_t d, const nnm_layers* layers, const float* q,
                uint64_t nq, uint32_t topk, uint32_t seed, int metric, uint32_t* out_ids, float* out_dists,
                uint64_t* ncmps);

}  // namespace nnm
