// Graph builders on the device: the reference's initial graphs, merges and
// the H-Merge level scheduler, driving run_nndescent (nndescent.cu).
//
//   kgraph_build   KGraph::buildKGraph        (kgraph.cpp:56-96, :217-245)
//   merge_leaves   Smerge::buildKGraph        (smerge.cpp:46-209) for two
//                  halves; the same steps over G leaves for G > 2
//   jmerge_build   Jmerge::buildKGraph        (jmerge.cpp:43-176)
//   hmerge_build   LyNNDescent::buildhgraph   (lynndescent.cpp:143-187,
//                  :354-500, :717-831)
//
// Random draws: each phase that the reference seeds with
// std::mt19937(time(NULL)) gets mt19937(seed) here (the reference run with a
// clock frozen at `seed`); the draws are generated on the host in row order
// and copied to the device, where each row's kernel warp consumes its fixed
// share.  std::rand() continues across phases from srand(seed).
#include <algorithm>
#include <vector>

#include "nnm_builders.h"
#include "nnm_join.h"
#include "nnm_learned.h"
#include "nnm_launch.h"
#include "nnm_scan.h"

namespace nnm {
namespace {
constexpr unsigned FULL = 0xffffffffu;
constexpr int WPB = 8;  // warps per block in the per-row kernels

struct InitArgs {
    const float* x;
    uint32_t dp, K;
    int metric;
    uint32_t* pid;
    float* pdist;
    const uint32_t* draws;   // draws of row0 first
    uint32_t draws_per_row;  // 0 when getRndSds is the identity
    uint32_t nseed, range;   // getRndSds(k = nseed, N = range)
    uint32_t row0, row1;
    uint32_t gd_split;       // gd = (id >= gd_split); 0xffffffff: gd = 0
    IterCounters* ctr;
};

// KGraph::InitialGraph (kgraph.cpp:56-96), Jmerge::InitialGraph new rows
// (jmerge.cpp:147-171), LyNNDescent::init (lynndescent.cpp:143-187) and the
// new rows of appdNwSmpl (:418-446): the first K seeds that are not the row
// itself, their distances, std::sort.
__global__ void k_init_rows(InitArgs a) {
    __shared__ uint32_t seeds[WPB][72];
    __shared__ SortEnt ents[WPB][MAXK];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t row = a.row0 + blockIdx.x * WPB + w;
    if (row >= a.row1) return;
    if (lane == 0)
        rnd_seeds_dev(a.draws + (size_t)(row - a.row0) * a.draws_per_row, a.nseed, a.range, seeds[w]);
    __syncwarp();
    uint32_t taken = 0;
    for (uint32_t b = 0; b < a.nseed && taken < a.K; b += 32) {
        uint32_t j = b + lane;
        uint32_t s = j < a.nseed ? seeds[w][j] : row;
        bool ok = j < a.nseed && s != row;
        unsigned bal = __ballot_sync(FULL, ok);
        uint32_t r = taken + __popc(bal & ((1u << lane) - 1u));
        if (ok && r < a.K) ents[w][r].id = s;
        taken += __popc(bal);
    }
    __syncwarp();
    if (taken < a.K) {
        if (lane == 0) atomicOr(&a.ctr->error, (unsigned)DERR_CROSS_SAMPLE);
        return;
    }
    if (lane < (int)a.K) {
        uint32_t s = ents[w][lane].id;
        float d = dist_seq_rt(a.metric, a.x + (size_t)row * a.dp, a.x + (size_t)s * a.dp, a.dp);
        uint32_t gd = (a.gd_split != 0xffffffffu && s >= a.gd_split) ? GD_BIT : 0u;
        ents[w][lane] = SortEnt{d, s | gd | FLAG_BIT};
    }
    __syncwarp();
    if (lane == 0) std_sort_dev(ents[w], (int)a.K);
    __syncwarp();
    if (lane < (int)a.K) {
        a.pid[(size_t)row * a.K + lane] = ents[w][lane].id;
        a.pdist[(size_t)row * a.K + lane] = ents[w][lane].dist;
    }
}

struct CrossArgs {
    const float* x;
    uint32_t dp, K;
    int metric;
    uint32_t* pid;
    float* pdist;
    uint32_t* cpid;
    float* cpdist;
    const uint32_t* draws;
    uint32_t draws_per_row;
    uint32_t nseed, cut;
    uint32_t row0, row1;
    // seed s of row r maps to the id: own leaf [lo, hi) of r is skipped, i.e.
    // id = s < lo ? s : s + (hi - lo); range = rows outside the leaf.
    const uint32_t* leaf_off;  // null: a single other group [base, base+range)
    uint32_t nleaf;
    uint32_t base, range;
    uint32_t gd_new;
    IterCounters* ctr;
};

__device__ __forceinline__ uint32_t leaf_index(uint32_t id, const uint32_t* off, uint32_t nleaf) {
    uint32_t lo = 0, hi = nleaf;
    while (hi - lo > 1) {
        uint32_t mid = (lo + hi) >> 1;
        if (id >= off[mid]) lo = mid;
        else hi = mid;
    }
    return lo;
}

// Cross sampling of built rows: Smerge::InitialGraph (smerge.cpp:94-209),
// Jmerge::InitialGraph old rows (jmerge.cpp:90-135), appdNwSmpl old rows
// (lynndescent.cpp:371-415).  The worst `cut` pool entries move to the
// compensation list and `cut` random ids of the other group(s) that are not
// already in the pool take their place; then std::sort.
__global__ void k_cross_sample(CrossArgs a) {
    __shared__ uint32_t seeds[WPB][72];
    __shared__ SortEnt ents[WPB][MAXK];
    __shared__ uint32_t fresh[WPB][MAXK];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t row = a.row0 + blockIdx.x * WPB + w;
    if (row >= a.row1) return;
    const uint32_t K = a.K, remain = K - a.cut;
    uint32_t lo = a.base, hi = a.base, range = a.range;
    if (a.leaf_off) {
        uint32_t g = leaf_index(row, a.leaf_off, a.nleaf);
        lo = a.leaf_off[g];
        hi = a.leaf_off[g + 1];
        range = a.leaf_off[a.nleaf] - (hi - lo);
    }
    if (lane == 0)
        rnd_seeds_dev(a.draws + (size_t)(row - a.row0) * a.draws_per_row, a.nseed, range, seeds[w]);
    if (lane < (int)K) {
        ents[w][lane] = SortEnt{a.pdist[(size_t)row * K + lane], a.pid[(size_t)row * K + lane]};
    }
    __syncwarp();
    if (lane < (int)a.cut) {
        a.cpid[(size_t)row * K + lane] = ents[w][remain + lane].id;
        a.cpdist[(size_t)row * K + lane] = ents[w][remain + lane].dist;
    }
    uint32_t taken = 0;
    for (uint32_t b = 0; b < a.nseed && taken < a.cut; b += 32) {
        uint32_t m = b + lane;
        uint32_t rid = 0;
        bool ok = false;
        if (m < a.nseed) {
            uint32_t s = seeds[w][m];
            rid = a.leaf_off ? (s < lo ? s : s + (hi - lo)) : s + a.base;
            ok = true;
            for (uint32_t l = 0; l < K; l++)
                if ((ents[w][l].id & ID_MASK) == rid) ok = false;
        }
        unsigned bal = __ballot_sync(FULL, ok);
        uint32_t r = taken + __popc(bal & ((1u << lane) - 1u));
        if (ok && r < a.cut) fresh[w][r] = rid;
        taken += __popc(bal);
    }
    __syncwarp();
    if (taken < a.cut) {
        if (lane == 0) atomicOr(&a.ctr->error, (unsigned)DERR_CROSS_SAMPLE);
        return;
    }
    if (lane < (int)a.cut) {
        uint32_t id = fresh[w][lane];
        float d = dist_seq_rt(a.metric, a.x + (size_t)id * a.dp, a.x + (size_t)row * a.dp, a.dp);
        ents[w][remain + lane] = SortEnt{d, id | (a.gd_new ? GD_BIT : 0u) | FLAG_BIT};
    }
    __syncwarp();
    if (lane == 0) std_sort_dev(ents[w], (int)K);
    __syncwarp();
    if (lane < (int)K) {
        a.pid[(size_t)row * K + lane] = ents[w][lane].id;
        a.pdist[(size_t)row * K + lane] = ents[w][lane].dist;
    }
}

// Fast tier: initial graphs and cross samples from Philox draws.  Per row,
// keep the best `keep` pool entries (their worst K - keep move to the
// compensation list), then draw K - keep distinct ids -- not the row itself,
// not already in the pool -- from the row's id space, compute their
// distances and sort the pool.  Each lane draws one candidate per round;
// duplicates within a round are resolved with __match_any_sync.
struct FastArgs {
    const float* x;
    uint32_t dp, K;
    int metric;
    uint32_t* pid;
    float* pdist;
    uint32_t* cpid;
    float* cpdist;
    uint32_t row0, row1;
    uint32_t keep;
    uint32_t range, base;      // ids base + [0, range) ...
    const uint32_t* leaf_off;  // ... or, when set, all rows outside the row's own leaf
    uint32_t nleaf;
    uint32_t gd_new;           // 0: gd 0, 1: gd 1, 2: gd = (id >= gd_split)
    uint32_t gd_split;
    uint32_t seed, phase;
    IterCounters* ctr;
    uint32_t partner;          // with leaf_off: draw from the partner leaf (leaf ^ 1) only; a row
                               // whose leaf has no partner keeps its pool
};

__global__ void k_fast_rows(FastArgs a) {
    __shared__ SortEnt ents[WPB][MAXK];
    __shared__ uint32_t fresh[WPB][MAXK];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t row = a.row0 + blockIdx.x * WPB + w;
    if (row >= a.row1) return;
    const uint32_t K = a.K;
    uint32_t need = K - a.keep;
    uint32_t lo = a.base, span = 0, range = a.range;
    if (a.leaf_off) {
        uint32_t g = leaf_index(row, a.leaf_off, a.nleaf);
        if (a.partner) {  // ids lo + [0, range) of the partner leaf
            const uint32_t p = g ^ 1u;
            if (p >= a.nleaf) return;  // unpaired at this level: the pool stays
            lo = a.leaf_off[p];
            range = a.leaf_off[p + 1] - lo;
        } else {
            lo = a.leaf_off[g];
            span = a.leaf_off[g + 1] - lo;
            range = a.leaf_off[a.nleaf] - span;
        }
    }
    if (lane < (int)K && a.keep) ents[w][lane] = SortEnt{a.pdist[(size_t)row * K + lane], a.pid[(size_t)row * K + lane]};
    __syncwarp();
    if (a.keep && lane < (int)need) {
        a.cpid[(size_t)row * K + lane] = ents[w][a.keep + lane].id;
        a.cpdist[(size_t)row * K + lane] = ents[w][a.keep + lane].dist;
    }
    const Philox ph{a.seed, 0x6e6e6d02u};
    uint32_t taken = 0;
    for (uint32_t round = 0; taken < need && round < 64; round++) {
        const uint32_t s = bounded(ph(row, a.phase, round, (uint32_t)lane).x, range);
        const uint32_t id = (a.leaf_off && !a.partner) ? (s < lo ? s : s + span) : s + (a.leaf_off ? lo : a.base);
        bool ok = id != row;
        for (uint32_t l = 0; l < K && ok; l++)
            if (a.keep && (ents[w][l].id & ID_MASK) == id) ok = false;
        for (uint32_t l = 0; l < taken && ok; l++)
            if (fresh[w][l] == id) ok = false;
        const unsigned same = __match_any_sync(FULL, id);
        if ((int)(__ffs(same) - 1) != lane) ok = false;  // first lane of equal draws
        const unsigned bal = __ballot_sync(FULL, ok);
        const uint32_t r = taken + __popc(bal & ((1u << lane) - 1u));
        __syncwarp();
        if (ok && r < need) fresh[w][r] = id;
        taken += __popc(bal);
        __syncwarp();
    }
    if (taken < need) {
        if (lane == 0) atomicOr(&a.ctr->error, (unsigned)DERR_CROSS_SAMPLE);
        return;
    }
    if (lane < (int)need) {
        const uint32_t id = fresh[w][lane];
        const float d = dist_seq_rt(a.metric, a.x + (size_t)row * a.dp, a.x + (size_t)id * a.dp, a.dp);
        const uint32_t gd = a.gd_new == 1 ? GD_BIT : (a.gd_new == 2 && id >= a.gd_split ? GD_BIT : 0u);
        ents[w][a.keep + lane] = SortEnt{d, id | gd | FLAG_BIT};
    }
    __syncwarp();
    if (lane == 0) std_sort_dev(ents[w], (int)K);
    __syncwarp();
    if (lane < (int)K) {
        a.pid[(size_t)row * K + lane] = ents[w][lane].id;
        a.pdist[(size_t)row * K + lane] = ents[w][lane].dist;
    }
}

// merge2one (abstractmerge.cpp:232-277, lynndescent.cpp:455-500): merge each
// pool with its compensation list, pool first on equal distances, keep K.
// The reference does not look for ids that are in both lists -- after an
// H-Merge level a compensation id can be back in the pool, and most rows of
// the reference's H-Merge output then hold duplicate ids.  The exact path
// keeps that; with `dedupe` (fast tier) such compensation entries are
// dropped, so every row keeps K distinct ids.
__global__ void k_merge2one(uint32_t* pid, float* pdist, const uint32_t* cpid, const float* cpdist, uint32_t K,
                            uint32_t cut, uint32_t rows, uint32_t dedupe) {
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t row = blockIdx.x * WPB + w;
    if (row >= rows) return;
    uint32_t pe = 0, ce = 0;
    float pd = 0.f, cd = 0.f;
    if (lane < (int)K) {
        pe = pid[(size_t)row * K + lane];
        pd = pdist[(size_t)row * K + lane];
    }
    if (lane < (int)cut) {
        ce = cpid[(size_t)row * K + lane];
        cd = cpdist[(size_t)row * K + lane];
    }
    bool keepc = lane < (int)cut;
    if (dedupe)
        for (uint32_t j = 0; j < K; j++)
            if ((__shfl_sync(FULL, pe, j) & ID_MASK) == (ce & ID_MASK)) keepc = false;
    const unsigned km = __ballot_sync(FULL, keepc);
    uint32_t pp = lane, cp = __popc(km & ((1u << lane) - 1u));
    for (uint32_t j = 0; j < K; j++) {
        float od = __shfl_sync(FULL, pd, j);
        float oc = __shfl_sync(FULL, cd, j);
        if (j < cut && ((km >> j) & 1u) && oc < pd) pp++;  // compensation entries strictly smaller come first
        if (od <= cd) cp++;                                // pool entries with equal distance win
    }
    __syncwarp();
    if (lane < (int)K && pp < K) {
        pid[(size_t)row * K + pp] = pe;
        pdist[(size_t)row * K + pp] = pd;
    }
    if (keepc && cp < K) {
        pid[(size_t)row * K + cp] = ce;
        pdist[(size_t)row * K + cp] = cd;
    }
}

// Sub-graph ids become global ids; every entry is flagged new with the
// sub-graph's group id (AbstractMerge::InitSGraph, abstractmerge.cpp:55-76;
// the distances are recomputed there with the same arithmetic, so the
// sub-graph's own values are kept).
__global__ void k_rebase(uint32_t* pid, size_t count, uint32_t add, uint32_t gd) {
    size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= count) return;
    pid[t] = ((pid[t] & ID_MASK) + add) | (gd ? GD_BIT : 0u) | FLAG_BIT;
}

// AbstractMerge::InitSGraph (abstractmerge.cpp:55-76) from a caller's
// graph: rows [b, b + rows) take the graph's local ids + b, in the graph's
// order, flagged new with group id `gd`, distances recomputed (a warp per
// row, a lane per entry).
__global__ void k_init_sgraph(const float* x, uint32_t dp, int metric, uint32_t K, const uint32_t* graph, uint32_t b,
                              uint32_t rows, uint32_t gd, uint32_t* pid, float* pdist) {
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t i = blockIdx.x * WPB + w;
    if (i >= rows || lane >= (int)K) return;
    const uint32_t row = b + i, id = graph[(size_t)i * K + lane] + b;
    pid[(size_t)row * K + lane] = id | (gd ? GD_BIT : 0u) | FLAG_BIT;
    pdist[(size_t)row * K + lane] = dist_seq_rt(metric, x + (size_t)row * dp, x + (size_t)id * dp, dp);
}

// setflag (lynndescent.cpp:717-732): all group ids to 0.
__global__ void k_clear_gd(uint32_t* pid, size_t count) {
    size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < count) pid[t] &= ~GD_BIT;
}

__global__ void k_export(const uint32_t* pid, const float* pdist, size_t count, uint32_t* ids, float* dists,
                         uint8_t* flags) {
    size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= count) return;
    uint32_t e = pid[t];
    if (ids) ids[t] = e & ID_MASK;
    if (dists) dists[t] = pdist[t];
    if (flags) flags[t] = (uint8_t)(e >> 31);
}

__global__ void k_pad_copy(const float* src, float* dst, uint64_t n, uint32_t d, uint32_t dp) {
    uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n * dp) return;
    uint64_t r = t / dp;
    uint32_t c = (uint32_t)(t - r * dp);
    dst[t] = c < d ? src[r * d + c] : 0.f;
}

}  // namespace

unsigned blocks_for(size_t n, unsigned per) { return (unsigned)((n + per - 1) / per); }

namespace {

// Host-generated mt19937 stream for `rows` rows of `per_row` draws each.
int upload_draws(Ctx& ctx, uint32_t seed_or_state_unused, std::vector<uint32_t>& host, size_t count) {
    (void)seed_or_state_unused;
    NNM_CUDA_TRY(ctx.ws.draws.ensure(std::max<size_t>(count, 1) * 4));
    if (count)
        NNM_CUDA_TRY(cudaMemcpyAsync(ctx.ws.draws.p, host.data(), count * 4, cudaMemcpyHostToDevice, ctx.stream));
    return 0;
}

// Draws consumed by one getRndSds(k, N) call.
inline uint32_t sds_draws(uint32_t k, uint32_t N) { return N == k ? 0u : k + 1u; }

}  // namespace

int check_counters(Ctx& ctx) {
    IterCounters* ctr = ctx.ws.counters.as<IterCounters>();
    NNM_CUDA_TRY(cudaMemcpyAsync(ctx.h_counters, ctr, sizeof(IterCounters), cudaMemcpyDeviceToHost, ctx.stream));
    NNM_CUDA_TRY(cudaStreamSynchronize(ctx.stream));
    if (ctx.h_counters->error) {
        ctx.last_error = ctx.h_counters->error & DERR_CROSS_SAMPLE
                             ? "random sampling found too few distinct candidates (graph too small for K)"
                             : "device capacity check failed";
        return 6;
    }
    return 0;
}

namespace {

int reset_counters(Ctx& ctx) {
    NNM_CUDA_TRY(ctx.ws.counters.ensure(sizeof(IterCounters) + 64));
    NNM_CUDA_TRY(cudaMemsetAsync(ctx.ws.counters.p, 0, sizeof(IterCounters), ctx.stream));
    return 0;
}

}  // namespace

int upload_vectors(Ctx& ctx, GraphStore& s, GraphDev& g, const float* x, bool x_on_device) {
    g.dp = (g.d + 3) & ~3u;
    const size_t elems = (size_t)g.n_cap * g.dp;
    NNM_CUDA_TRY(s.x.ensure(elems * 4));
    if (g.dp == g.d) {
        NNM_CUDA_TRY(cudaMemcpyAsync(s.x.p, x, elems * 4, x_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                                     ctx.stream));
    } else {
        const float* src = x;
        DevBuf tmp;
        if (!x_on_device) {
            NNM_CUDA_TRY(tmp.ensure((size_t)g.n_cap * g.d * 4));
            NNM_CUDA_TRY(cudaMemcpyAsync(tmp.p, x, (size_t)g.n_cap * g.d * 4, cudaMemcpyHostToDevice, ctx.stream));
            src = tmp.as<float>();
        }
        k_pad_copy<<<blocks_for(elems, 256), 256, 0, ctx.stream>>>(src, s.x.as<float>(), g.n_cap, g.d, g.dp); count_launch();
        NNM_CUDA_TRY(cudaStreamSynchronize(ctx.stream));
        tmp.release();
    }
    g.x = s.x.as<float>();
    if (g.init == NNM_INIT_LEARNED) {
        if (!ctx.init_model || ctx.init_model->d != g.d) {
            ctx.last_error = "NNM_INIT_LEARNED needs a model for this dimension (nnm_set_init_model)";
            return 1;
        }
        NNM_CUDA_TRY(s.codes.ensure((size_t)g.n_cap * 4));
        int rc = mlp_codes_dev(ctx, *ctx.init_model, g.x, g.n_cap, g.dp, s.codes.as<uint32_t>(), nullptr);
        if (rc) return rc;
        g.codes = s.codes.as<uint32_t>();
    }
    return tc_prepare(ctx, s, g);
}

int export_graph(Ctx& ctx, const GraphDev& g, uint32_t* ids, float* dists, uint8_t* flags, bool host_out) {
    const size_t cnt = (size_t)g.n * g.K;
    if (!host_out) {
        k_export<<<blocks_for(cnt, 256), 256, 0, ctx.stream>>>(g.pid, g.pdist, cnt, ids, dists, flags); count_launch();
        NNM_CUDA_TRY(cudaGetLastError());
        return 0;
    }
    DevBuf& tmp = ctx.ws.misc;
    NNM_CUDA_TRY(tmp.ensure(cnt * 9 + 64));
    uint32_t* di = tmp.as<uint32_t>();
    float* dd = reinterpret_cast<float*>(di + cnt);
    uint8_t* df = reinterpret_cast<uint8_t*>(dd + cnt);
    k_export<<<blocks_for(cnt, 256), 256, 0, ctx.stream>>>(g.pid, g.pdist, cnt, di, dd, df); count_launch();
    if (ids) NNM_CUDA_TRY(cudaMemcpyAsync(ids, di, cnt * 4, cudaMemcpyDeviceToHost, ctx.stream));
    if (dists) NNM_CUDA_TRY(cudaMemcpyAsync(dists, dd, cnt * 4, cudaMemcpyDeviceToHost, ctx.stream));
    if (flags) NNM_CUDA_TRY(cudaMemcpyAsync(flags, df, cnt, cudaMemcpyDeviceToHost, ctx.stream));
    NNM_CUDA_TRY(cudaStreamSynchronize(ctx.stream));
    return 0;
}

// KGraph on rows [0, g.n) of g (x, pid, pdist already offset by the caller).
static int fast_rows(Ctx& ctx, GraphDev& g, uint32_t row0, uint32_t row1, uint32_t keep, uint32_t range,
                     uint32_t base, const uint32_t* leaf_off, uint32_t nleaf, uint32_t gd_new, uint32_t gd_split,
                     uint32_t partner = 0) {
    int rc;
    if ((rc = reset_counters(ctx))) return rc;
    FastArgs fa{g.x, g.dp, g.K, g.metric, g.pid, g.pdist, g.cpid, g.cpdist, row0, row1, keep, range, base,
                leaf_off, nleaf, gd_new, gd_split, g.seed, g.phase++, ctx.ws.counters.as<IterCounters>(), partner};
    k_fast_rows<<<blocks_for(row1 - row0, WPB), WPB * 32, 0, ctx.stream>>>(fa); count_launch();
    NNM_CUDA_TRY(cudaGetLastError());
    return check_counters(ctx);
}

// Fast tier: the initial graph of g's rows (learned or random), local ids.
static int fast_init(Ctx& ctx, GraphDev& g) {
    const uint32_t n = g.n;
    int rc;
    if (g.init == NNM_INIT_LEARNED) {
        if (g.views) {
            rc = learned_rows(ctx, g, *g.views, g.view_leaf);
        } else {
            CodeViews vw;
            rc = views_build(ctx, g, {0u, n}, vw);
            if (!rc) rc = learned_rows(ctx, g, vw, 0);
        }
    } else {
        rc = fast_rows(ctx, g, 0, n, 0, n, 0, nullptr, 0, 0, 0);
    }
    if (rc) return rc;
    g.ncmps += (uint64_t)n * g.K;
    return 0;
}

int kgraph_build(Ctx& ctx, GraphDev& g) {
    const uint32_t K = g.K, n = g.n;
    if (g.fast) {
        int rc = fast_init(ctx, g);
        if (rc) return rc;
        return run_nndescent(ctx, g, MODE_KGRAPH, 0, 0, nullptr, 0);
    }
    const uint32_t per = sds_draws(K + 1, n);
    std::vector<uint32_t> h((size_t)n * per);
    gen_mt19937(g.seed, h.size(), h.data());
    int rc = upload_draws(ctx, g.seed, h, h.size());
    if (rc) return rc;
    if ((rc = reset_counters(ctx))) return rc;
    InitArgs ia{g.x, g.dp, K, g.metric, g.pid, g.pdist, ctx.ws.draws.as<uint32_t>(), per, K + 1, n, 0, n,
                0xffffffffu, ctx.ws.counters.as<IterCounters>()};
    k_init_rows<<<blocks_for(n, WPB), WPB * 32, 0, ctx.stream>>>(ia); count_launch();
    NNM_CUDA_TRY(cudaGetLastError());
    if ((rc = check_counters(ctx))) return rc;
    g.ncmps += (uint64_t)n * K;
    return run_nndescent(ctx, g, MODE_KGRAPH, 0, 0, nullptr, 0);
}

// A view of rows [b, e) of parent as a stand-alone graph (shared arrays).
static GraphDev sub_view(const GraphDev& p, uint32_t b, uint32_t e) {
    GraphDev s = p;
    s.n_cap = s.n = e - b;
    s.x = p.x + (size_t)b * p.dp;
    if (p.codes) s.codes = p.codes + b;
    s.views = nullptr;
    if (p.xq) {
        s.xq = p.xq + (size_t)b * p.kq;
        s.nrm = p.nrm + b;
        if (p.scl) s.scl = p.scl + b;  // FP8 operands: the rows' scales with their rows
    }
    s.pid = p.pid + (size_t)b * p.K;
    s.pdist = p.pdist + (size_t)b * p.K;
    s.cpid = p.cpid + (size_t)b * p.K;
    s.cpdist = p.cpdist + (size_t)b * p.K;
    s.ncmps = 0;
    s.iters = 0;
    s.trace.clear();
    s.carry = false;
    return s;
}

static void absorb(GraphDev& p, const GraphDev& s) {
    p.gpos = s.gpos;
    p.iters += s.iters;
    p.trace.insert(p.trace.end(), s.trace.begin(), s.trace.end());
}

// Smerge::InitialGraph (smerge.cpp:94-209) over G leaves, reference
// streams: one mt19937(seed) for all rows in order, getRndSds(2 cut) over the
// rows outside the row's leaf, the worst `cut` entries to the compensation
// list.  d_leaf_off: the leaf boundaries on the device.
static int cross_sample_leaves(Ctx& ctx, GraphDev& g, const std::vector<uint32_t>& leaf_off,
                               const uint32_t* d_leaf_off) {
    const uint32_t K = g.K, n = g.n, nleaf = (uint32_t)leaf_off.size() - 1;
    int rc;
    g.cut = K * 1 / 2;
    size_t total = 0;
    std::vector<uint32_t> per(nleaf);
    for (uint32_t l = 0; l < nleaf; l++) {
        uint32_t range = n - (leaf_off[l + 1] - leaf_off[l]);
        per[l] = sds_draws(2 * g.cut, range);
        total += (size_t)(leaf_off[l + 1] - leaf_off[l]) * per[l];
    }
    std::vector<uint32_t> h(total);
    gen_mt19937(g.seed, total, h.data());
    if ((rc = upload_draws(ctx, g.seed, h, total))) return rc;
    if ((rc = reset_counters(ctx))) return rc;
    size_t off = 0;
    for (uint32_t l = 0; l < nleaf; l++) {
        uint32_t r0 = leaf_off[l], r1 = leaf_off[l + 1];
        CrossArgs ca{g.x, g.dp, K, g.metric, g.pid, g.pdist, g.cpid, g.cpdist,
                     ctx.ws.draws.as<uint32_t>() + off, per[l], 2 * g.cut, g.cut, r0, r1,
                     d_leaf_off, nleaf, 0, 0, nleaf == 2 ? (l == 0 ? 1u : 0u) : 0u,
                     ctx.ws.counters.as<IterCounters>()};
        k_cross_sample<<<blocks_for(r1 - r0, WPB), WPB * 32, 0, ctx.stream>>>(ca); count_launch();
        off += (size_t)(r1 - r0) * per[l];
    }
    NNM_CUDA_TRY(cudaGetLastError());
    if ((rc = check_counters(ctx))) return rc;
    g.ncmps += (uint64_t)n * g.cut;
    return 0;
}

// Jmerge::InitialGraph (jmerge.cpp:83-176), reference streams: the built
// rows [0, pre) cross-sample `cut` ids of the raw rows, the raw rows [pre, n)
// take K random ids of all rows; one mt19937(seed), built rows first.
static int jmerge_initial_exact(Ctx& ctx, GraphDev& g, uint32_t pre) {
    const uint32_t K = g.K, n = g.n;
    int rc;
    g.cut = K * 3 / 6;  // jmerge.cpp:87
    const uint32_t per_old = sds_draws(2 * g.cut, n - pre), per_new = sds_draws(K + 1, n);
    size_t total = (size_t)pre * per_old + (size_t)(n - pre) * per_new;
    std::vector<uint32_t> h(total);
    gen_mt19937(g.seed, total, h.data());
    if ((rc = upload_draws(ctx, g.seed, h, total))) return rc;
    if ((rc = reset_counters(ctx))) return rc;
    CrossArgs ca{g.x, g.dp, K, g.metric, g.pid, g.pdist, g.cpid, g.cpdist, ctx.ws.draws.as<uint32_t>(), per_old,
                 2 * g.cut, g.cut, 0, pre, nullptr, 0, pre, n - pre, 1, ctx.ws.counters.as<IterCounters>()};
    k_cross_sample<<<blocks_for(pre, WPB), WPB * 32, 0, ctx.stream>>>(ca); count_launch();
    InitArgs ia{g.x, g.dp, K, g.metric, g.pid, g.pdist, ctx.ws.draws.as<uint32_t>() + (size_t)pre * per_old,
                per_new, K + 1, n, pre, n, pre, ctx.ws.counters.as<IterCounters>()};
    k_init_rows<<<blocks_for(n - pre, WPB), WPB * 32, 0, ctx.stream>>>(ia); count_launch();
    NNM_CUDA_TRY(cudaGetLastError());
    if ((rc = check_counters(ctx))) return rc;
    g.ncmps += (uint64_t)pre * g.cut + (uint64_t)(n - pre) * K;
    return 0;
}

// Bottom-up pairwise merge of built leaves (fast tier): at each level leaf
// 2i is S-Merged with leaf 2i + 1 (an odd last leaf waits for the next
// level), and all pairs of a level share one NN-Descent run -- every row's
// cross samples come from its partner leaf only, so no list mixes pairs --
// then merge2one; the merged pairs are the next level's leaves.  On entry
// the leaves hold their graphs (global ids).
static int merge_tree_levels(Ctx& ctx, GraphDev& g, std::vector<uint32_t> off) {
    const uint32_t K = g.K;
    int rc;
    g.cut = K * 1 / 2;
    DevBuf& lo = ctx.ws.misc;
    NNM_CUDA_TRY(lo.ensure(off.size() * 4 + 64));
    while (off.size() > 2) {
        const uint32_t nl = (uint32_t)off.size() - 1;
        const uint32_t pend = (nl & 1u) ? off[nl - 1] : off[nl];  // rows of paired leaves
        NNM_CUDA_TRY(cudaMemcpyAsync(lo.p, off.data(), off.size() * 4, cudaMemcpyHostToDevice, ctx.stream));
        // InitSGraph of both sub-graphs of every pair: all entries new
        k_rebase<<<blocks_for((size_t)pend * K, 256), 256, 0, ctx.stream>>>(g.pid, (size_t)pend * K, 0u, 0u); count_launch();
        if ((rc = fast_rows(ctx, g, 0, pend, K - g.cut, 0, 0, lo.as<uint32_t>(), nl, 0, 0, 1))) return rc;
        g.ncmps += (uint64_t)pend * g.cut;
        if ((rc = run_nndescent(ctx, g, MODE_SMERGE, off[1], 0, lo.as<uint32_t>(), nl))) return rc;
        k_merge2one<<<blocks_for(pend, WPB), WPB * 32, 0, ctx.stream>>>(g.pid, g.pdist, g.cpid, g.cpdist, K, g.cut,
                                                                       pend, 1u); count_launch();
        NNM_CUDA_TRY(cudaGetLastError());
        std::vector<uint32_t> nxt;
        for (size_t i = 0; i < off.size(); i += 2) nxt.push_back(off[i]);
        if (nxt.back() != off.back()) nxt.push_back(off.back());
        off.swap(nxt);
        NNM_CUDA_TRY(cudaStreamSynchronize(ctx.stream));  // `off` on the host changes before the next copy
    }
    return 0;
}

// Fast tier, step 1 of a multi-leaf build: NN-Descent on every leaf, in
// place (smerge.cpp:56-68), all leaves in one run: each leaf's initial graph
// holds only rows of that leaf and reverse lists come from the pools, so no
// list ever mixes leaves -- one launch sequence for leaves of any sizes.
// leaf0: the index of the first leaf among all leaves of the build (the
// leaves' initial draws).  Pools end with ids of g's rows.
static int fast_leaf_builds(Ctx& ctx, GraphDev& g, const std::vector<uint32_t>& leaf_off, uint32_t leaf0,
                            const CodeViews* vw, uint64_t* subc) {
    const uint32_t K = g.K, nleaf = (uint32_t)leaf_off.size() - 1;
    int rc;
    for (uint32_t l = 0; l < nleaf; l++) {
        GraphDev s = sub_view(g, leaf_off[l], leaf_off[l + 1]);
        if (vw) {
            s.views = vw;
            s.view_leaf = l;
        }
        s.phase = g.phase + leaf0 + l;  // independent draws per leaf
        if ((rc = fast_init(ctx, s))) return rc;
        *subc += s.ncmps;
        const size_t cnt = (size_t)s.n * K;
        k_rebase<<<blocks_for(cnt, 256), 256, 0, ctx.stream>>>(s.pid, cnt, leaf_off[l], 0u); count_launch();
    }
    g.phase = LEAF_PHASE0;  // the leaf run's draws do not depend on how the leaves were split
    const uint64_t before = g.ncmps;
    if ((rc = run_nndescent(ctx, g, MODE_KGRAPH, 0, 0, nullptr, 0))) return rc;
    *subc += g.ncmps - before;
    g.ncmps = before;
    return 0;
}

// Fast tier, steps 2-4 of a multi-leaf build on leaves whose graphs are in
// g's pools (ids of g's rows): InitSGraph (all entries new, group ids),
// cross sampling from the other leaves (learned or random), NN-Descent with
// the cross-leaf join, merge2one -- or the bottom-up tree.  The merge's
// draws start at a fixed phase, so they do not depend on the leaf runs.
static int fast_merge_phase(Ctx& ctx, GraphDev& g, const std::vector<uint32_t>& leaf_off, const CodeViews* vw) {
    const uint32_t K = g.K, n = g.n, nleaf = (uint32_t)leaf_off.size() - 1;
    int rc;
    g.phase = MERGE_PHASE0;
    for (uint32_t l = 0; l < nleaf; l++) {
        const size_t cnt = (size_t)(leaf_off[l + 1] - leaf_off[l]) * K;
        k_rebase<<<blocks_for(cnt, 256), 256, 0, ctx.stream>>>(g.pid + (size_t)leaf_off[l] * K, cnt, 0u,
                                                              nleaf == 2 ? l : 0u); count_launch();
    }
    if (g.merge_tree) return merge_tree_levels(ctx, g, leaf_off);
    g.cut = K * 1 / 2;
    DevBuf& lo = ctx.ws.misc;
    NNM_CUDA_TRY(lo.ensure(leaf_off.size() * 4 + 64));
    NNM_CUDA_TRY(cudaMemcpyAsync(lo.p, leaf_off.data(), leaf_off.size() * 4, cudaMemcpyHostToDevice, ctx.stream));
    rc = vw ? learned_cross(ctx, g, *vw, lo.as<uint32_t>())
            : fast_rows(ctx, g, 0, n, K - g.cut, 0, 0, lo.as<uint32_t>(), nleaf, 0, 0);
    if (rc) return rc;
    g.ncmps += (uint64_t)n * g.cut;
    if ((rc = run_nndescent(ctx, g, MODE_SMERGE, leaf_off[1], 0, lo.as<uint32_t>(), nleaf))) return rc;
    k_merge2one<<<blocks_for(n, WPB), WPB * 32, 0, ctx.stream>>>(g.pid, g.pdist, g.cpid, g.cpdist, K, g.cut, n, 1u); count_launch();
    NNM_CUDA_TRY(cudaGetLastError());
    return 0;
}

int build_leaves(Ctx& ctx, GraphDev& g, const std::vector<uint32_t>& leaf_off, uint32_t leaf0, uint64_t* ncmps) {
    CodeViews vw;
    const bool learned = g.init == NNM_INIT_LEARNED;
    int rc;
    if (learned && (rc = views_build(ctx, g, leaf_off, vw))) return rc;
    uint64_t c = 0;
    if ((rc = fast_leaf_builds(ctx, g, leaf_off, leaf0, learned ? &vw : nullptr, &c))) return rc;
    if (ncmps) *ncmps = c;
    return 0;
}

// Pools from a caller's device arrays (n x K ids of g's rows, distances);
// ids outside [0, n) fail with DERR_CROSS_SAMPLE's status.
__global__ void k_check_ids(const uint32_t* ids, size_t count, uint32_t n, IterCounters* ctr) {
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < count && ids[t] >= n) atomicOr(&ctr->error, (unsigned)DERR_LIST_CAP);
}

int load_pools(Ctx& ctx, GraphDev& g, const uint32_t* ids_dev, const float* dists_dev) {
    const size_t cnt = (size_t)g.n * g.K;
    int rc;
    if ((rc = reset_counters(ctx))) return rc;
    k_check_ids<<<blocks_for(cnt, 256), 256, 0, ctx.stream>>>(ids_dev, cnt, g.n, ctx.ws.counters.as<IterCounters>()); count_launch();
    NNM_CUDA_TRY(cudaGetLastError());
    IterCounters* ctr = ctx.ws.counters.as<IterCounters>();
    NNM_CUDA_TRY(cudaMemcpyAsync(ctx.h_counters, ctr, sizeof(IterCounters), cudaMemcpyDeviceToHost, ctx.stream));
    NNM_CUDA_TRY(cudaStreamSynchronize(ctx.stream));
    if (ctx.h_counters->error) {
        ctx.last_error = "leaf graph ids must lie in [0, n)";
        return 1;
    }
    NNM_CUDA_TRY(cudaMemcpyAsync(g.pid, ids_dev, cnt * 4, cudaMemcpyDeviceToDevice, ctx.stream));
    NNM_CUDA_TRY(cudaMemcpyAsync(g.pdist, dists_dev, cnt * 4, cudaMemcpyDeviceToDevice, ctx.stream));
    return 0;
}

int merge_prebuilt(Ctx& ctx, GraphDev& g, const std::vector<uint32_t>& leaf_off) {
    CodeViews vw;
    const bool learned = g.init == NNM_INIT_LEARNED;
    int rc;
    if (learned && (rc = views_build(ctx, g, leaf_off, vw))) return rc;
    return fast_merge_phase(ctx, g, leaf_off, learned ? &vw : nullptr);
}

int merge_leaves(Ctx& ctx, GraphDev& g, const std::vector<uint32_t>& leaf_off, uint64_t* sub_ncmps) {
    const uint32_t K = g.K;
    int rc;
    uint64_t subc = 0;
    CodeViews vw;
    const bool learned = g.fast && g.init == NNM_INIT_LEARNED;
    if (learned && (rc = views_build(ctx, g, leaf_off, vw))) return rc;
    if (g.fast) {
        if ((rc = fast_leaf_builds(ctx, g, leaf_off, 0, learned ? &vw : nullptr, &subc))) return rc;
        if (sub_ncmps) *sub_ncmps = subc;
        return fast_merge_phase(ctx, g, leaf_off, learned ? &vw : nullptr);
    }
    // reference streams: one KGraph per leaf, the std::rand() stream running on
    const uint32_t n = g.n, nleaf = (uint32_t)leaf_off.size() - 1;
    for (uint32_t l = 0; l < nleaf; l++) {
        GraphDev s = sub_view(g, leaf_off[l], leaf_off[l + 1]);
        if ((rc = kgraph_build(ctx, s))) return rc;
        subc += s.ncmps;
        absorb(g, s);
        size_t cnt = (size_t)s.n * K;
        k_rebase<<<blocks_for(cnt, 256), 256, 0, ctx.stream>>>(s.pid, cnt, leaf_off[l], nleaf == 2 ? l : 0u); count_launch();
    }
    if (sub_ncmps) *sub_ncmps = subc;
    // 2. cross sampling (smerge.cpp:94-209)
    g.cut = K * 1 / 2;
    DevBuf& lo = ctx.ws.misc;
    NNM_CUDA_TRY(lo.ensure(leaf_off.size() * 4 + 64));
    NNM_CUDA_TRY(cudaMemcpyAsync(lo.p, leaf_off.data(), leaf_off.size() * 4, cudaMemcpyHostToDevice, ctx.stream));
    if ((rc = cross_sample_leaves(ctx, g, leaf_off, lo.as<uint32_t>()))) return rc;
    // 3. NN-Descent with the cross-group join, 4. merge2one
    if ((rc = run_nndescent(ctx, g, MODE_SMERGE, leaf_off[1], 0, lo.as<uint32_t>(), nleaf))) return rc;
    k_merge2one<<<blocks_for(n, WPB), WPB * 32, 0, ctx.stream>>>(g.pid, g.pdist, g.cpid, g.cpdist, K, g.cut, n, g.fast ? 1u : 0u); count_launch();
    NNM_CUDA_TRY(cudaGetLastError());
    return 0;
}

int jmerge_build(Ctx& ctx, GraphDev& g, uint64_t* sub_ncmps) {
    const uint32_t K = g.K, n = g.n, pre = n * 5 / 10;  // jmerge.cpp:47
    int rc;
    GraphDev s = sub_view(g, 0, pre);
    if ((rc = kgraph_build(ctx, s))) return rc;
    if (sub_ncmps) *sub_ncmps = s.ncmps;
    absorb(g, s);
    k_rebase<<<blocks_for((size_t)pre * K, 256), 256, 0, ctx.stream>>>(g.pid, (size_t)pre * K, 0, 0); count_launch();
    g.cut = K * 3 / 6;                                    // jmerge.cpp:87
    if (g.fast) {
        if ((rc = fast_rows(ctx, g, 0, pre, K - g.cut, n - pre, pre, nullptr, 0, 1, 0))) return rc;
        if ((rc = fast_rows(ctx, g, pre, n, 0, n, 0, nullptr, 0, 2, pre))) return rc;
        g.ncmps += (uint64_t)pre * g.cut + (uint64_t)(n - pre) * K;
        if ((rc = run_nndescent(ctx, g, MODE_JMERGE, pre, 0, nullptr, 0))) return rc;
        k_merge2one<<<blocks_for(pre, WPB), WPB * 32, 0, ctx.stream>>>(g.pid, g.pdist, g.cpid, g.cpdist, K, g.cut, pre, g.fast ? 1u : 0u); count_launch();
        NNM_CUDA_TRY(cudaGetLastError());
        return 0;
    }
    if ((rc = jmerge_initial_exact(ctx, g, pre))) return rc;
    if ((rc = run_nndescent(ctx, g, MODE_JMERGE, pre, 0, nullptr, 0))) return rc;
    k_merge2one<<<blocks_for(pre, WPB), WPB * 32, 0, ctx.stream>>>(g.pid, g.pdist, g.cpid, g.cpdist, K, g.cut, pre, g.fast ? 1u : 0u); count_launch();
    NNM_CUDA_TRY(cudaGetLastError());
    return 0;
}

int hmerge_build(Ctx& ctx, GraphDev& g, const LayerHook& on_layer) {
    const uint32_t N0 = 64, K = g.K, row = g.n_cap;  // lynndescent.cpp:23
    int rc;
    // init: 64 rows, random K-NN (lynndescent.cpp:143-187)
    if (g.fast) {
        if ((rc = fast_rows(ctx, g, 0, N0, 0, N0, 0, nullptr, 0, 0, 0))) return rc;
        g.ncmps += (uint64_t)N0 * K;
    } else {
        const uint32_t per = sds_draws(K + 1, N0);
        std::vector<uint32_t> h((size_t)N0 * per);
        gen_mt19937(g.seed, h.size(), h.data());
        if ((rc = upload_draws(ctx, g.seed, h, h.size()))) return rc;
        if ((rc = reset_counters(ctx))) return rc;
        InitArgs ia{g.x, g.dp, K, g.metric, g.pid, g.pdist, ctx.ws.draws.as<uint32_t>(), per, K + 1, N0, 0, N0,
                    0xffffffffu, ctx.ws.counters.as<IterCounters>()};
        k_init_rows<<<blocks_for(N0, WPB), WPB * 32, 0, ctx.stream>>>(ia); count_launch();
        if ((rc = check_counters(ctx))) return rc;
        g.ncmps += (uint64_t)N0 * K;
    }
    g.n = N0;
    uint32_t last_id = N0, total = row - N0, smpl = N0, count_level = 0;
    if ((rc = run_nndescent(ctx, g, MODE_LY, N0, 1, nullptr, 0))) return rc;
    if ((rc = on_layer(ctx, g))) return rc;
    count_level++;
    static const uint32_t level[10] = {1, 0, 0, 1, 0, 0, 1, 0, 0, 1};  // lynndescent.cpp:771
    const uint32_t half = K / 2, hsize = K - half;
    while (total != 0) {
        const bool last = !(total > smpl);
        const uint32_t bnum = last ? total : smpl;
        const uint32_t sz = g.n, lst = last_id;
        // appdNwSmpl (lynndescent.cpp:354-452): one mt19937(seed), old rows then new rows
        if (g.fast) {
            g.cut = hsize;
            if ((rc = fast_rows(ctx, g, 0, sz, half, bnum, lst, nullptr, 0, 1, 0))) return rc;
            if ((rc = fast_rows(ctx, g, sz, sz + bnum, 0, sz + bnum, 0, nullptr, 0, 2, lst))) return rc;
        }
        if (!g.fast) {
            const uint32_t per_old = sds_draws(2 * half, bnum), per_new = sds_draws(2 * K, sz + bnum);
            size_t tot = (size_t)sz * per_old + (size_t)bnum * per_new;
            std::vector<uint32_t> h(tot);
            gen_mt19937(g.seed, tot, h.data());
            if ((rc = upload_draws(ctx, g.seed, h, tot))) return rc;
            if ((rc = reset_counters(ctx))) return rc;
            g.cut = hsize;
            CrossArgs ca{g.x, g.dp, K, g.metric, g.pid, g.pdist, g.cpid, g.cpdist, ctx.ws.draws.as<uint32_t>(), per_old,
                         2 * half, hsize, 0, sz, nullptr, 0, lst, bnum, 1, ctx.ws.counters.as<IterCounters>()};
            k_cross_sample<<<blocks_for(sz, WPB), WPB * 32, 0, ctx.stream>>>(ca); count_launch();
            InitArgs ia{g.x, g.dp, K, g.metric, g.pid, g.pdist, ctx.ws.draws.as<uint32_t>() + (size_t)sz * per_old,
                        per_new, 2 * K, sz + bnum, sz, sz + bnum, lst, ctx.ws.counters.as<IterCounters>()};
            k_init_rows<<<blocks_for(bnum, WPB), WPB * 32, 0, ctx.stream>>>(ia); count_launch();
            NNM_CUDA_TRY(cudaGetLastError());
            if ((rc = check_counters(ctx))) return rc;
        }
        g.ncmps += (uint64_t)sz * hsize + (uint64_t)bnum * K;
        g.n = sz + bnum;
        last_id = lst + bnum;
        total -= bnum;
        if ((rc = run_nndescent(ctx, g, MODE_LY, lst, 0, nullptr, 0))) return rc;
        k_merge2one<<<blocks_for(sz, WPB), WPB * 32, 0, ctx.stream>>>(g.pid, g.pdist, g.cpid, g.cpdist, K, hsize, sz, g.fast ? 1u : 0u); count_launch();
        NNM_CUDA_TRY(cudaGetLastError());
        if (last || (count_level < 10 && level[count_level]))
            if ((rc = on_layer(ctx, g))) return rc;
        count_level++;
        if (!last) {
            smpl = g.n;
            size_t cnt = (size_t)g.n * K;
            k_clear_gd<<<blocks_for(cnt, 256), 256, 0, ctx.stream>>>(g.pid, cnt); count_launch();  // setflag
        }
    }
    NNM_CUDA_TRY(cudaGetLastError());
    return 0;
}

// ---------------------------------------------------------------------------
// Staged merge: the steps of Smerge/Jmerge::buildKGraph as separate calls on
// one graph (reference streams).  The graph is one reference process: the
// std::rand() stream continues from step to step, each phase that the
// reference seeds with time(NULL) draws from mt19937(seed).

int stage_subgraph(Ctx& ctx, GraphDev& g, uint32_t b, uint32_t e, uint64_t* ncmps) {
    GraphDev s = sub_view(g, b, e);
    int rc = kgraph_build(ctx, s);
    if (rc) return rc;
    if (ncmps) *ncmps = s.ncmps;
    absorb(g, s);
    return 0;
}

int stage_init_sgraph(Ctx& ctx, GraphDev& g, uint32_t b, const uint32_t* d_graph, uint32_t gid, uint32_t rows) {
    k_init_sgraph<<<blocks_for(rows, WPB), WPB * 32, 0, ctx.stream>>>(g.x, g.dp, g.metric, g.K, d_graph, b, rows,
                                                                   gid, g.pid, g.pdist); count_launch();
    NNM_CUDA_TRY(cudaGetLastError());
    return 0;
}

int stage_initial_graph(Ctx& ctx, GraphDev& g, JoinMode mode, uint32_t pre, const uint32_t* d_leaf_off) {
    if (mode == MODE_SMERGE) return cross_sample_leaves(ctx, g, {0u, pre, g.n}, d_leaf_off);
    return jmerge_initial_exact(ctx, g, pre);
}

int stage_nndescent(Ctx& ctx, GraphDev& g, JoinMode mode, uint32_t pre, const uint32_t* d_leaf_off) {
    if (mode == MODE_SMERGE) return run_nndescent(ctx, g, MODE_SMERGE, pre, 0, d_leaf_off, 2);
    return run_nndescent(ctx, g, MODE_JMERGE, pre, 0, nullptr, 0);
}

int stage_merge2one(Ctx& ctx, GraphDev& g, uint32_t sz) {
    k_merge2one<<<blocks_for(sz, WPB), WPB * 32, 0, ctx.stream>>>(g.pid, g.pdist, g.cpid, g.cpdist, g.K, g.cut, sz,
                                                                 g.fast ? 1u : 0u); count_launch();
    NNM_CUDA_TRY(cudaGetLastError());
    return 0;
}

}  // namespace nnm
