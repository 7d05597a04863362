// C ABI (include/nnm.h) over the device engine.
#include <cstdio>
#include <cstring>
#include <memory>
#include <random>
#include <string>
#include <vector>

#include "../../include/nnm.h"
#include "nnm_builders.h"
#include "nnm_entry.h"
#include "nnm_eval.h"
#include "nnm_hier.h"
#include "nnm_launch.h"
#include "nnm_learned.h"

struct nnm_ctx {
    nnm::Ctx c;
};

struct nnm_index {
    nnm_ctx* ctx;
    nnm::IndexDev ix;
};

// A staged merge: its own graph arrays (the reference's egraph), so that
// other calls on the context between the steps leave it alone.
struct nnm_merge {
    nnm_ctx* ctx;
    nnm::GraphStore store;
    nnm::GraphDev g;
    nnm::DevBuf leaf_off, graph;  // {0, pre, n}; a caller's graph for InitSGraph
};

namespace {

using nnm::Ctx;
using nnm::GraphDev;
using nnm::GraphStore;

int fail(nnm_ctx* ctx, int code, const std::string& msg) {
    if (ctx) ctx->c.last_error = msg;
    return code;
}

bool opts_ok(nnm_ctx* ctx, const nnm_opts* o, int* rc) {
    if (o->metric > NNM_METRIC_CHI2) {
        *rc = fail(ctx, NNM_ERR_UNSUPPORTED_METRIC, "metric must be NNM_METRIC_L2, _L1 or _CHI2");
        return false;
    }
    if (o->rng_mode != NNM_RNG_EXACT && o->rng_mode != NNM_RNG_FAST) {
        *rc = fail(ctx, NNM_ERR_INVALID, "unknown rng_mode");
        return false;
    }
    if (o->sample_cap == 0 || o->sample_cap > 4096) {
        *rc = fail(ctx, NNM_ERR_INVALID, "sample_cap must be in [1, 4096]");
        return false;
    }
    if (o->join_kernel > NNM_JOIN_FP8) {
        *rc = fail(ctx, NNM_ERR_INVALID, "unknown join_kernel");
        return false;
    }
    if (o->init > NNM_INIT_LEARNED) {
        *rc = fail(ctx, NNM_ERR_INVALID, "unknown init");
        return false;
    }
    if (o->tile_rows != 0 && o->tile_rows != 32 && o->tile_rows != 64 && o->tile_rows != 128) {
        *rc = fail(ctx, NNM_ERR_INVALID, "tile_rows must be 0, 32, 64 or 128");
        return false;
    }
    if (o->merge_order > NNM_MERGE_TREE) {
        *rc = fail(ctx, NNM_ERR_INVALID, "unknown merge_order");
        return false;
    }
    if (o->merge_order == NNM_MERGE_TREE && o->rng_mode != NNM_RNG_FAST) {
        *rc = fail(ctx, NNM_ERR_INVALID, "NNM_MERGE_TREE needs rng_mode NNM_RNG_FAST");
        return false;
    }
    if (o->init == NNM_INIT_LEARNED && o->rng_mode != NNM_RNG_FAST) {
        *rc = fail(ctx, NNM_ERR_INVALID, "NNM_INIT_LEARNED needs rng_mode NNM_RNG_FAST");
        return false;
    }
    return true;
}

void setup_graph(GraphDev& g, const nnm_opts& o, uint64_t n, uint32_t d, uint32_t k) {
    g.n_cap = g.n = (uint32_t)n;
    g.K = k;
    g.d = d;
    g.metric = (int)o.metric;
    g.seed = o.seed;
    g.gbase = nnm::glibc_base(o.seed);
    g.gpos = 0;  // srand(seed) at the start of the call
    g.smpl = o.sample_cap;
    g.delta = o.delta;
    g.max_iter = o.max_iter;
    g.exact_trace = o.exact_trace != 0;
    g.fast = o.rng_mode == NNM_RNG_FAST;
    g.join_kernel = o.join_kernel;
    g.audit = o.audit != 0;
    g.merge_tree = o.merge_order == NNM_MERGE_TREE;
    g.no_graph = o.no_graph != 0;
    g.tile_rows = o.tile_rows ? o.tile_rows : 128u;
    g.init = o.init;
    g.phase = 0;
}

void fill_stats(nnm_stats* st, const GraphDev& g, uint64_t sub, float ms) {
    if (!st) return;
    st->ncmps = g.ncmps;
    st->sub_ncmps = sub;
    st->iterations = g.iters;
    st->n_trace = (uint32_t)std::min<size_t>(g.trace.size(), 256);
    for (uint32_t i = 0; i < st->n_trace; i++) st->trace[i] = g.trace[i];
    st->device_ms = ms;
}

struct EventTimer {
    cudaEvent_t a = nullptr, b = nullptr;
    cudaStream_t s;
    explicit EventTimer(cudaStream_t st) : s(st) {
        cudaEventCreate(&a);
        cudaEventCreate(&b);
        cudaEventRecord(a, s);
    }
    float stop() {
        float ms = 0.f;
        cudaEventRecord(b, s);
        cudaEventSynchronize(b);
        cudaEventElapsedTime(&ms, a, b);
        return ms;
    }
    ~EventTimer() {
        cudaEventDestroy(a);
        cudaEventDestroy(b);
    }
};

enum Kind { KIND_KGRAPH, KIND_LEAVES, KIND_JMERGE };

int build_common(nnm_ctx* ctx, Kind kind, const float* x, bool dev, uint64_t n, uint32_t d, uint32_t k,
                 const uint32_t* leaf_sizes, uint32_t nleaf, const nnm_opts* opts, uint32_t* ids, float* dists,
                 uint8_t* flags, nnm_stats* stats) {
    if (!ctx) return NNM_ERR_INVALID;
    if (!x || n == 0 || d == 0) return fail(ctx, NNM_ERR_INVALID, "x must be non-null with n, d > 0");
    if (k == 0 || k > (uint32_t)nnm::MAXK) return fail(ctx, NNM_ERR_INVALID, "k must be in [1, 32]");
    if (n >= (1ull << 30)) return fail(ctx, NNM_ERR_INVALID, "n must be below 2^30");
    nnm_opts o;
    if (opts) o = *opts;
    else nnm_opts_default(&o);
    int rc;
    if (!opts_ok(ctx, &o, &rc)) return rc;
    std::vector<uint32_t> off;
    if (kind == KIND_LEAVES) {
        if (!leaf_sizes || nleaf < 2 || nleaf > 1024) return fail(ctx, NNM_ERR_INVALID, "need 2..1024 leaves");
        off.push_back(0);
        for (uint32_t l = 0; l < nleaf; l++) {
            if (leaf_sizes[l] < k + 2) return fail(ctx, NNM_ERR_INVALID, "every leaf needs at least k+2 rows");
            off.push_back(off.back() + leaf_sizes[l]);
        }
        if (off.back() != n) return fail(ctx, NNM_ERR_INVALID, "leaf sizes must sum to n");
    } else if (kind == KIND_JMERGE) {
        if (n * 5 / 10 < k + 2) return fail(ctx, NNM_ERR_INVALID, "n too small for k");
    } else if (n < k + 2) {
        return fail(ctx, NNM_ERR_INVALID, "n must be at least k+2");
    }
    Ctx& c = ctx->c;
    if (cudaSetDevice(c.device) != cudaSuccess) return fail(ctx, NNM_ERR_NO_DEVICE, "cudaSetDevice failed");
    GraphStore& store = c.store;
    GraphDev g;
    setup_graph(g, o, n, d, k);
    uint64_t sub = 0;
    EventTimer tm(c.stream);
    rc = nnm::upload_vectors(c, store, g, x, dev);
    if (!rc) rc = nnm::graph_alloc(c, store, g, false);
    if (!rc) {
        if (kind == KIND_KGRAPH) rc = nnm::kgraph_build(c, g);
        else if (kind == KIND_LEAVES) rc = nnm::merge_leaves(c, g, off, &sub);
        else rc = nnm::jmerge_build(c, g, &sub);
    }
    if (!rc) rc = nnm::export_graph(c, g, ids, dists, flags, !dev);
    float ms = tm.stop();
    if (!rc) {
        cudaError_t e = cudaStreamSynchronize(c.stream);
        if (e != cudaSuccess) rc = fail(ctx, NNM_ERR_CUDA, cudaGetErrorString(e));
    }
    if (!rc) fill_stats(stats, g, sub, ms);
    return rc;
}

bool mlp_ok(nnm_ctx* ctx, const nnm_mlp* m, uint32_t d) {
    if (!m || !m->w1 || !m->b1 || !m->w2 || !m->b2) {
        fail(ctx, NNM_ERR_INVALID, "model arrays must be non-null");
        return false;
    }
    if (m->d_in != d || d == 0 || d > nnm::MLP_MAX_D) {
        fail(ctx, NNM_ERR_INVALID, "model d_in must equal d and be in [1, 256]");
        return false;
    }
    return true;
}

// Vectors to the device (zero-padded rows) without any join preparation.
int upload_plain(Ctx& c, GraphStore& st, GraphDev& g, const float* x, uint64_t n, uint32_t d) {
    g.n_cap = g.n = (uint32_t)n;
    g.d = d;
    g.join_kernel = NNM_JOIN_FP32;
    g.init = NNM_INIT_RANDOM;
    return nnm::upload_vectors(c, st, g, x, false);
}

// Runs one step of a staged merge: sets the device, returns the step's
// status after its work has finished.
template <class F>
int merge_step(nnm_merge* m, F&& step) {
    if (!m) return NNM_ERR_INVALID;
    Ctx& c = m->ctx->c;
    if (cudaSetDevice(c.device) != cudaSuccess) return fail(m->ctx, NNM_ERR_NO_DEVICE, "cudaSetDevice failed");
    int rc = step(c);
    if (!rc) {
        cudaError_t e = cudaStreamSynchronize(c.stream);
        if (e != cudaSuccess) rc = fail(m->ctx, NNM_ERR_CUDA, cudaGetErrorString(e));
    }
    return rc;
}

bool merge_kind_ok(nnm_merge* m, uint32_t kind, uint32_t pre) {
    if (kind != NNM_MERGE_SMERGE && kind != NNM_MERGE_JMERGE) {
        fail(m->ctx, NNM_ERR_INVALID, "kind must be NNM_MERGE_SMERGE or NNM_MERGE_JMERGE");
        return false;
    }
    if (pre < m->g.K + 2 || pre >= m->g.n || (kind == NNM_MERGE_SMERGE && m->g.n - pre < m->g.K + 2)) {
        fail(m->ctx, NNM_ERR_INVALID, "pre must leave at least k+2 rows on its built side(s)");
        return false;
    }
    return true;
}
}  // namespace

extern "C" {

void nnm_opts_default(nnm_opts* o) {
    std::memset(o, 0, sizeof(*o));
    o->seed = 0;
    o->rng_mode = NNM_RNG_EXACT;
    o->metric = NNM_METRIC_L2;
    o->sample_cap = 100;  // kgraph.cpp:100
    o->delta = 0.002f;    // abstractgraph.cpp:4
    o->max_iter = 0;
    o->exact_trace = 0;
}

const char* nnm_status_string(int s) {
    switch (s) {
    case NNM_OK: return "ok";
    case NNM_ERR_INVALID: return "invalid argument";
    case NNM_ERR_UNSUPPORTED_METRIC: return "unsupported metric";
    case NNM_ERR_CUDA: return "CUDA error";
    case NNM_ERR_OOM: return "out of device memory";
    case NNM_ERR_NO_DEVICE: return "no CUDA device";
    case NNM_ERR_CAPACITY: return "device capacity check failed";
    default: return "unknown status";
    }
}

const char* nnm_last_error(const nnm_ctx* ctx) { return ctx ? ctx->c.last_error.c_str() : "null context"; }

int nnm_ctx_create(int device, nnm_ctx** out) {
    if (!out) return NNM_ERR_INVALID;
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count <= device || device < 0) return NNM_ERR_NO_DEVICE;
    if (cudaSetDevice(device) != cudaSuccess) return NNM_ERR_NO_DEVICE;
    std::unique_ptr<nnm_ctx> ctx(new nnm_ctx());
    ctx->c.device = device;
    if (cudaStreamCreateWithFlags(&ctx->c.stream, cudaStreamNonBlocking) != cudaSuccess) return NNM_ERR_CUDA;
    if (cudaMallocHost(&ctx->c.h_counters, sizeof(nnm::IterCounters) * 2) != cudaSuccess) return NNM_ERR_CUDA;
    if (nnm::glibc_tables_init() != cudaSuccess) return NNM_ERR_CUDA;
    *out = ctx.release();
    return NNM_OK;
}

int nnm_ctx_destroy(nnm_ctx* ctx) {
    if (!ctx) return NNM_OK;
    cudaSetDevice(ctx->c.device);
    cudaStreamSynchronize(ctx->c.stream);
    for (auto& e : ctx->c.ev)
        if (e) cudaEventDestroy(e);
    for (auto& ig : ctx->c.iter_graph)
        if (ig.exec) cudaGraphExecDestroy(ig.exec);
    ctx->c.ws.release_all();
    ctx->c.store.release();
    if (ctx->c.init_model) {
        ctx->c.init_model->release();
        delete ctx->c.init_model;
    }
    if (ctx->c.h_counters) cudaFreeHost(ctx->c.h_counters);
    if (ctx->c.stream) cudaStreamDestroy(ctx->c.stream);
    delete ctx;
    return NNM_OK;
}

int nnm_kgraph_build(nnm_ctx* ctx, const float* x, uint64_t n, uint32_t d, uint32_t k, const nnm_opts* opts,
                     uint32_t* ids, float* dists, uint8_t* flags, nnm_stats* stats) {
    return build_common(ctx, KIND_KGRAPH, x, false, n, d, k, nullptr, 0, opts, ids, dists, flags, stats);
}

int nnm_kgraph_build_dev(nnm_ctx* ctx, const float* x, uint64_t n, uint32_t d, uint32_t k, const nnm_opts* opts,
                         uint32_t* ids, float* dists, uint8_t* flags, nnm_stats* stats) {
    return build_common(ctx, KIND_KGRAPH, x, true, n, d, k, nullptr, 0, opts, ids, dists, flags, stats);
}

int nnm_smerge(nnm_ctx* ctx, const float* x, uint64_t n, uint32_t d, uint32_t k, const nnm_opts* opts,
               uint32_t* ids, float* dists, uint8_t* flags, nnm_stats* stats) {
    uint32_t sizes[2] = {(uint32_t)(n * 5 / 10), (uint32_t)(n - n * 5 / 10)};  // smerge.cpp:53
    return build_common(ctx, KIND_LEAVES, x, false, n, d, k, sizes, 2, opts, ids, dists, flags, stats);
}

int nnm_jmerge(nnm_ctx* ctx, const float* x, uint64_t n, uint32_t d, uint32_t k, const nnm_opts* opts,
               uint32_t* ids, float* dists, uint8_t* flags, nnm_stats* stats) {
    return build_common(ctx, KIND_JMERGE, x, false, n, d, k, nullptr, 0, opts, ids, dists, flags, stats);
}

int nnm_merge_leaves(nnm_ctx* ctx, const float* x, uint64_t n, uint32_t d, uint32_t k, const uint32_t* leaf_sizes,
                     uint32_t nleaf, const nnm_opts* opts, uint32_t* ids, float* dists, uint8_t* flags,
                     nnm_stats* stats) {
    return build_common(ctx, KIND_LEAVES, x, false, n, d, k, leaf_sizes, nleaf, opts, ids, dists, flags, stats);
}

int nnm_merge_leaves_dev(nnm_ctx* ctx, const float* x, uint64_t n, uint32_t d, uint32_t k,
                         const uint32_t* leaf_sizes, uint32_t nleaf, const nnm_opts* opts, uint32_t* ids,
                         float* dists, uint8_t* flags, nnm_stats* stats) {
    return build_common(ctx, KIND_LEAVES, x, true, n, d, k, leaf_sizes, nleaf, opts, ids, dists, flags, stats);
}

namespace {
// The two halves of a fast-tier multi-leaf build on device arrays.
int leaves_common(nnm_ctx* ctx, bool merge, const float* x, uint64_t n, uint32_t d, uint32_t k,
                  const uint32_t* leaf_sizes, uint32_t nleaf, uint32_t leaf0, const nnm_opts* opts,
                  const uint32_t* ids_in, const float* dists_in, uint32_t* ids, float* dists, uint8_t* flags,
                  nnm_stats* stats) {
    if (!ctx) return NNM_ERR_INVALID;
    if (!x || n == 0 || d == 0) return fail(ctx, NNM_ERR_INVALID, "x must be non-null with n, d > 0");
    if (k == 0 || k > (uint32_t)nnm::MAXK) return fail(ctx, NNM_ERR_INVALID, "k must be in [1, 32]");
    if (n >= (1ull << 30)) return fail(ctx, NNM_ERR_INVALID, "n must be below 2^30");
    if (merge && (!ids_in || !dists_in)) return fail(ctx, NNM_ERR_INVALID, "the leaves' graphs must be given");
    nnm_opts o;
    if (opts) o = *opts;
    else nnm_opts_default(&o);
    int rc;
    if (!opts_ok(ctx, &o, &rc)) return rc;
    if (o.rng_mode != NNM_RNG_FAST) return fail(ctx, NNM_ERR_INVALID, "split leaf builds need rng_mode NNM_RNG_FAST");
    if (!leaf_sizes || nleaf < (merge ? 2u : 1u) || nleaf > 1024) return fail(ctx, NNM_ERR_INVALID, "bad leaf count");
    std::vector<uint32_t> off(1, 0);
    for (uint32_t l = 0; l < nleaf; l++) {
        if (leaf_sizes[l] < k + 2) return fail(ctx, NNM_ERR_INVALID, "every leaf needs at least k+2 rows");
        off.push_back(off.back() + leaf_sizes[l]);
    }
    if (off.back() != n) return fail(ctx, NNM_ERR_INVALID, "leaf sizes must sum to n");
    Ctx& c = ctx->c;
    if (cudaSetDevice(c.device) != cudaSuccess) return fail(ctx, NNM_ERR_NO_DEVICE, "cudaSetDevice failed");
    GraphDev g;
    setup_graph(g, o, n, d, k);
    uint64_t sub = 0;
    EventTimer tm(c.stream);
    rc = nnm::upload_vectors(c, c.store, g, x, true);
    if (!rc) rc = nnm::graph_alloc(c, c.store, g, false);
    if (!rc) {
        if (merge) {
            rc = nnm::load_pools(c, g, ids_in, dists_in);
            if (!rc) rc = nnm::merge_prebuilt(c, g, off);
        } else {
            rc = nnm::build_leaves(c, g, off, leaf0, &sub);
        }
    }
    if (!rc) rc = nnm::export_graph(c, g, ids, dists, flags, false);
    float ms = tm.stop();
    if (!rc) {
        cudaError_t e = cudaStreamSynchronize(c.stream);
        if (e != cudaSuccess) rc = fail(ctx, NNM_ERR_CUDA, cudaGetErrorString(e));
    }
    if (!rc) {
        if (!merge) g.ncmps = 0;
        fill_stats(stats, g, sub, ms);
    }
    return rc;
}
}  // namespace

int nnm_build_leaves_dev(nnm_ctx* ctx, const float* x_dev, uint64_t n, uint32_t d, uint32_t k,
                         const uint32_t* leaf_sizes, uint32_t nleaf, uint32_t leaf0, const nnm_opts* opts,
                         uint32_t* ids_dev, float* dists_dev, nnm_stats* stats) {
    return leaves_common(ctx, false, x_dev, n, d, k, leaf_sizes, nleaf, leaf0, opts, nullptr, nullptr, ids_dev,
                         dists_dev, nullptr, stats);
}

int nnm_merge_prebuilt_dev(nnm_ctx* ctx, const float* x_dev, uint64_t n, uint32_t d, uint32_t k,
                           const uint32_t* leaf_sizes, uint32_t nleaf, const nnm_opts* opts,
                           const uint32_t* ids_in_dev, const float* dists_in_dev, uint32_t* ids_dev,
                           float* dists_dev, uint8_t* flags_dev, nnm_stats* stats) {
    return leaves_common(ctx, true, x_dev, n, d, k, leaf_sizes, nleaf, 0, opts, ids_in_dev, dists_in_dev, ids_dev,
                         dists_dev, flags_dev, stats);
}

int nnm_merge_create(nnm_ctx* ctx, const float* x, uint64_t n, uint32_t d, uint32_t k, const nnm_opts* opts,
                     nnm_merge** out) {
    if (!ctx) return NNM_ERR_INVALID;
    if (!out) return fail(ctx, NNM_ERR_INVALID, "out must be non-null");
    *out = nullptr;
    if (!x || n == 0 || d == 0) return fail(ctx, NNM_ERR_INVALID, "x must be non-null with n, d > 0");
    if (k == 0 || k > (uint32_t)nnm::MAXK) return fail(ctx, NNM_ERR_INVALID, "k must be in [1, 32]");
    if (n >= (1ull << 30)) return fail(ctx, NNM_ERR_INVALID, "n must be below 2^30");
    if (n < k + 2) return fail(ctx, NNM_ERR_INVALID, "n must be at least k+2");
    nnm_opts o;
    if (opts) o = *opts;
    else nnm_opts_default(&o);
    int rc;
    if (!opts_ok(ctx, &o, &rc)) return rc;
    if (o.rng_mode != NNM_RNG_EXACT)
        return fail(ctx, NNM_ERR_INVALID, "the staged merge runs the reference's streams (NNM_RNG_EXACT)");
    Ctx& c = ctx->c;
    if (cudaSetDevice(c.device) != cudaSuccess) return fail(ctx, NNM_ERR_NO_DEVICE, "cudaSetDevice failed");
    std::unique_ptr<nnm_merge> m(new nnm_merge());
    m->ctx = ctx;
    setup_graph(m->g, o, n, d, k);
    rc = nnm::upload_vectors(c, m->store, m->g, x, false);
    if (!rc) rc = nnm::graph_alloc(c, m->store, m->g, false);
    if (!rc) {
        cudaError_t e = m->leaf_off.ensure(64);
        if (e == cudaSuccess) e = cudaStreamSynchronize(c.stream);
        if (e != cudaSuccess) rc = fail(ctx, NNM_ERR_CUDA, cudaGetErrorString(e));
    }
    if (rc) {
        m->store.release();
        m->leaf_off.release();
        return rc;
    }
    *out = m.release();
    return NNM_OK;
}


int nnm_merge_subgraph(nnm_merge* m, uint32_t b, uint32_t e, uint32_t* graph, uint64_t* ncmps) {
    if (!m) return NNM_ERR_INVALID;
    if (b >= e || e > m->g.n || e - b < m->g.K + 2)
        return fail(m->ctx, NNM_ERR_INVALID, "need 0 <= b < e <= n with at least k+2 rows");
    return merge_step(m, [&](Ctx& ctx) {
        uint64_t nc = 0;
        int rc = nnm::stage_subgraph(ctx, m->g, b, e, &nc);
        if (!rc && graph) {
            nnm::GraphDev s = m->g;
            s.n = e - b;
            s.pid = m->g.pid + (size_t)b * m->g.K;
            s.pdist = m->g.pdist + (size_t)b * m->g.K;
            rc = nnm::export_graph(ctx, s, graph, nullptr, nullptr, true);
        }
        if (!rc && ncmps) *ncmps = nc;
        return rc;
    });
}

int nnm_merge_init_sgraph(nnm_merge* m, uint32_t b, const uint32_t* graph, uint32_t gid, uint32_t size) {
    if (!m) return NNM_ERR_INVALID;
    const uint32_t K = m->g.K;
    if (!graph || size == 0 || (uint64_t)b + size > m->g.n)
        return fail(m->ctx, NNM_ERR_INVALID, "need a graph and 0 < size with b + size <= n");
    if (gid > 1) return fail(m->ctx, NNM_ERR_INVALID, "gid must be 0 or 1");
    for (size_t t = 0; t < (size_t)size * K; t++)
        if (graph[t] >= size) return fail(m->ctx, NNM_ERR_INVALID, "graph ids must be local to the sub-range");
    return merge_step(m, [&](Ctx& ctx) {
        const size_t bytes = (size_t)size * K * 4;
        NNM_CUDA_TRY(m->graph.ensure(bytes));
        NNM_CUDA_TRY(cudaMemcpyAsync(m->graph.p, graph, bytes, cudaMemcpyHostToDevice, ctx.stream));
        return nnm::stage_init_sgraph(ctx, m->g, b, m->graph.as<uint32_t>(), gid, size);
    });
}

int nnm_merge_initial_graph(nnm_merge* m, uint32_t kind, uint32_t pre) {
    if (!m) return NNM_ERR_INVALID;
    if (!merge_kind_ok(m, kind, pre)) return NNM_ERR_INVALID;
    return merge_step(m, [&](Ctx& ctx) {
        const uint32_t off[3] = {0u, pre, m->g.n};
        NNM_CUDA_TRY(cudaMemcpyAsync(m->leaf_off.p, off, sizeof(off), cudaMemcpyHostToDevice, ctx.stream));
        NNM_CUDA_TRY(cudaStreamSynchronize(ctx.stream));  // off lives on this stack
        return nnm::stage_initial_graph(ctx, m->g, kind == NNM_MERGE_SMERGE ? nnm::MODE_SMERGE : nnm::MODE_JMERGE, pre,
                                        m->leaf_off.as<uint32_t>());
    });
}

int nnm_merge_nndescent(nnm_merge* m, uint32_t kind, uint32_t pre, nnm_stats* stats) {
    if (!m) return NNM_ERR_INVALID;
    if (!merge_kind_ok(m, kind, pre)) return NNM_ERR_INVALID;
    return merge_step(m, [&](Ctx& ctx) {
        const uint32_t off[3] = {0u, pre, m->g.n};
        NNM_CUDA_TRY(cudaMemcpyAsync(m->leaf_off.p, off, sizeof(off), cudaMemcpyHostToDevice, ctx.stream));
        NNM_CUDA_TRY(cudaStreamSynchronize(ctx.stream));
        GraphDev& g = m->g;
        const uint64_t c0 = g.ncmps;
        const uint32_t it0 = g.iters;
        const size_t t0 = g.trace.size();
        EventTimer tm(ctx.stream);
        int rc = nnm::stage_nndescent(ctx, g, kind == NNM_MERGE_SMERGE ? nnm::MODE_SMERGE : nnm::MODE_JMERGE, pre,
                                      m->leaf_off.as<uint32_t>());
        const float ms = tm.stop();
        if (!rc && stats) {
            GraphDev part;
            part.ncmps = g.ncmps - c0;
            part.iters = g.iters - it0;
            part.trace.assign(g.trace.begin() + t0, g.trace.end());
            fill_stats(stats, part, 0, ms);
        }
        return rc;
    });
}

int nnm_merge_merge2one(nnm_merge* m, uint32_t sz) {
    if (!m) return NNM_ERR_INVALID;
    if (sz == 0 || sz > m->g.n) return fail(m->ctx, NNM_ERR_INVALID, "sz must be in [1, n]");
    if (m->g.cut == 0) return fail(m->ctx, NNM_ERR_INVALID, "merge2one needs an initial graph (its compensation lists)");
    return merge_step(m, [&](Ctx& ctx) { return nnm::stage_merge2one(ctx, m->g, sz); });
}

int nnm_merge_read(nnm_merge* m, uint32_t* ids, float* dists, uint8_t* flags) {
    if (!m) return NNM_ERR_INVALID;
    return merge_step(m, [&](Ctx& ctx) { return nnm::export_graph(ctx, m->g, ids, dists, flags, true); });
}

int nnm_merge_free(nnm_merge* m) {
    if (!m) return NNM_OK;
    cudaSetDevice(m->ctx->c.device);
    cudaStreamSynchronize(m->ctx->c.stream);
    m->store.release();
    m->leaf_off.release();
    m->graph.release();
    delete m;
    return NNM_OK;
}

int nnm_hmerge_build(nnm_ctx* ctx, const float* x, uint64_t n, uint32_t d, uint32_t k, uint32_t m,
                     const nnm_opts* opts, uint32_t* ids, float* dists, uint8_t* flags, nnm_layers* layers,
                     nnm_stats* stats) {
    if (!ctx) return NNM_ERR_INVALID;
    if (!x || n <= 64 || d == 0) return fail(ctx, NNM_ERR_INVALID, "need x non-null, n > 64, d > 0");
    if (k == 0 || k + 1 > 64 || k > (uint32_t)nnm::MAXK) return fail(ctx, NNM_ERR_INVALID, "k must be in [1, 32]");
    if (m == 0 || m > 64) return fail(ctx, NNM_ERR_INVALID, "m must be in [1, 64]");
    if (n >= (1ull << 30)) return fail(ctx, NNM_ERR_INVALID, "n must be below 2^30");
    nnm_opts o;
    if (opts) o = *opts;
    else nnm_opts_default(&o);
    int rc;
    if (!opts_ok(ctx, &o, &rc)) return rc;
    Ctx& c = ctx->c;
    if (cudaSetDevice(c.device) != cudaSuccess) return fail(ctx, NNM_ERR_NO_DEVICE, "cudaSetDevice failed");
    GraphStore& store = c.store;
    GraphDev g;
    setup_graph(g, o, n, d, k);
    nnm::DpgState dpg;
    if (layers) std::memset(layers, 0, sizeof(*layers));
    EventTimer tm(c.stream);
    rc = nnm::upload_vectors(c, store, g, x, false);
    if (!rc) rc = nnm::graph_alloc(c, store, g, true);
    if (!rc) rc = nnm::dpg_init(c, dpg, g.n_cap, k, m);
    if (!rc)
        rc = nnm::hmerge_build(c, g, [&](Ctx& cc, GraphDev& gg) { return nnm::dpg_layer(cc, dpg, gg, layers); });
    if (!rc) rc = nnm::export_graph(c, g, ids, dists, flags, true);
    float ms = tm.stop();
    dpg.release();
    if (!rc) fill_stats(stats, g, 0, ms);
    else if (layers) nnm_layers_free(layers);
    return rc;
}

int nnm_profile_enable(nnm_ctx* ctx, int on) {
    if (!ctx) return NNM_ERR_INVALID;
    if (on && !ctx->c.ev[0]) {
        cudaSetDevice(ctx->c.device);
        for (auto& e : ctx->c.ev)
            if (cudaEventCreate(&e) != cudaSuccess) return fail(ctx, NNM_ERR_CUDA, "cudaEventCreate failed");
    }
    ctx->c.prof = on != 0;
    ctx->c.kjoin = ctx->c.kemit = ctx->c.kmerge = nnm::KStat();
    for (auto& r : ctx->c.join_rows) r = 0;
    ctx->c.join_rows_tc = 0;
    ctx->c.iter_log.clear();
    ctx->c.audit_max = ctx->c.audit_err_c = 0.f;
    ctx->c.approx_props = ctx->c.rechecks = 0;
    return NNM_OK;
}

int nnm_profile_get(const nnm_ctx* ctx, char* buf, uint64_t buflen) {
    if (!ctx || !buf || buflen == 0) return NNM_ERR_INVALID;
    const nnm::Ctx& c = ctx->c;
    std::string js;
    char tmp[512];
    std::snprintf(tmp, sizeof tmp,
                  "{\"join\": {\"launches\": %llu, \"ms\": %.6f, \"bytes\": %.1f, \"flops\": %.1f, \"tensor_ops\": %.1f}, "
                  "\"emit\": {\"launches\": %llu, \"ms\": %.6f, \"bytes\": %.1f, \"tensor_ops\": %.1f}, "
                  "\"merge\": {\"launches\": %llu, \"ms\": %.6f, \"bytes\": %.1f}, ",
                  (unsigned long long)c.kjoin.launches, c.kjoin.ms, c.kjoin.bytes, c.kjoin.flops, c.kjoin.tensor_ops,
                  (unsigned long long)c.kemit.launches, c.kemit.ms, c.kemit.bytes, c.kemit.tensor_ops,
                  (unsigned long long)c.kmerge.launches, c.kmerge.ms, c.kmerge.bytes);
    js += tmp;
    std::snprintf(tmp, sizeof tmp,
                  "\"audit\": {\"max_rel\": %.9g, \"err_c\": %.9g}, "
                  "\"approx\": {\"proposals\": %llu, \"rechecks\": %llu}, ",
                  (double)c.audit_max, (double)c.audit_err_c, (unsigned long long)c.approx_props,
                  (unsigned long long)c.rechecks);
    js += tmp;
    std::snprintf(tmp, sizeof tmp, "\"rows\": {\"tiers\": [%llu, %llu, %llu, %llu, %llu], \"tensor\": %llu}, \"iters\": [",
                  (unsigned long long)c.join_rows[0], (unsigned long long)c.join_rows[1],
                  (unsigned long long)c.join_rows[2], (unsigned long long)c.join_rows[3],
                  (unsigned long long)c.join_rows[4], (unsigned long long)c.join_rows_tc);
    js += tmp;
    for (size_t i = 0; i < c.iter_log.size(); i++) {
        const auto& L = c.iter_log[i];
        std::snprintf(tmp, sizeof tmp,
                      "%s[%u, [%u, %u, %u, %u, %u], %llu, %llu, %llu, %llu, %llu, %.4f, %.4f, %.4f]", i ? ", " : "",
                      L.n, L.rows[0], L.rows[1], L.rows[2], L.rows[3], L.rows[4], (unsigned long long)L.pairs,
                      (unsigned long long)L.proposals, (unsigned long long)L.flags, (unsigned long long)L.ncmps,
                      (unsigned long long)L.sum_s, L.ms_join, L.ms_emit, L.ms_merge);
        js += tmp;
    }
    js += "]}";
    if (js.size() + 1 > buflen) return NNM_ERR_INVALID;
    std::memcpy(buf, js.c_str(), js.size() + 1);
    return NNM_OK;
}

uint64_t nnm_launch_count(void) { return nnm::launch_counter().load(); }

void nnm_train_opts_default(nnm_train_opts* o) {
    std::memset(o, 0, sizeof(*o));
    o->steps = 400;
    o->batch = 2048;
    o->lr = 2e-3f;
    o->margin = 16.f;
    o->seed = 0;
}

int nnm_set_init_model(nnm_ctx* ctx, const nnm_mlp* model) {
    if (!ctx) return NNM_ERR_INVALID;
    Ctx& c = ctx->c;
    if (!model) {
        if (c.init_model) {
            c.init_model->release();
            delete c.init_model;
            c.init_model = nullptr;
        }
        return NNM_OK;
    }
    if (!mlp_ok(ctx, model, model->d_in)) return NNM_ERR_INVALID;
    if (cudaSetDevice(c.device) != cudaSuccess) return fail(ctx, NNM_ERR_NO_DEVICE, "cudaSetDevice failed");
    if (!c.init_model) c.init_model = new nnm::DevMlp();
    return nnm::mlp_upload(c, *c.init_model, *model);
}

int nnm_mlp_codes(nnm_ctx* ctx, const nnm_mlp* model, const float* x, uint64_t n, uint32_t d, uint32_t* codes,
                  float* z) {
    if (!ctx || !x || !codes || n == 0 || n >= (1ull << 30)) return NNM_ERR_INVALID;
    if (!mlp_ok(ctx, model, d)) return NNM_ERR_INVALID;
    Ctx& c = ctx->c;
    if (cudaSetDevice(c.device) != cudaSuccess) return fail(ctx, NNM_ERR_NO_DEVICE, "cudaSetDevice failed");
    nnm::DevMlp m;
    GraphStore st;
    GraphDev g;
    int rc = nnm::mlp_upload(c, m, *model);
    if (!rc) rc = upload_plain(c, st, g, x, n, d);
    nnm::DevBuf dc, dz;
    if (!rc && (dc.ensure(n * 4) != cudaSuccess || (z && dz.ensure(n * 32 * 4) != cudaSuccess)))
        rc = fail(ctx, NNM_ERR_OOM, "device allocation failed");
    if (!rc) rc = nnm::mlp_codes_dev(c, m, g.x, (uint32_t)n, g.dp, dc.as<uint32_t>(), z ? dz.as<float>() : nullptr);
    // the engine's stream is non-blocking: wait for it before the plain copies
    if (!rc && cudaStreamSynchronize(c.stream) != cudaSuccess) rc = fail(ctx, NNM_ERR_CUDA, "kernel failed");
    if (!rc && cudaMemcpy(codes, dc.p, n * 4, cudaMemcpyDeviceToHost) != cudaSuccess) rc = NNM_ERR_CUDA;
    if (!rc && z && cudaMemcpy(z, dz.p, n * 32 * 4, cudaMemcpyDeviceToHost) != cudaSuccess) rc = NNM_ERR_CUDA;
    m.release();
    dc.release();
    dz.release();
    st.release();
    return rc;
}

int nnm_mlp_grad(nnm_ctx* ctx, const nnm_mlp* model, const float* x, uint64_t n, uint32_t d,
                 const uint32_t* triplets, uint32_t ntrip, float margin, float* loss, nnm_mlp* grad) {
    if (!ctx || !x || !triplets || !loss || !grad || ntrip == 0 || n == 0 || n >= (1ull << 30)) return NNM_ERR_INVALID;
    if (!mlp_ok(ctx, model, d) || !mlp_ok(ctx, grad, d)) return NNM_ERR_INVALID;
    for (uint64_t i = 0; i < 3ull * ntrip; i++)
        if (triplets[i] >= n) return fail(ctx, NNM_ERR_INVALID, "triplet index out of range");
    Ctx& c = ctx->c;
    if (cudaSetDevice(c.device) != cudaSuccess) return fail(ctx, NNM_ERR_NO_DEVICE, "cudaSetDevice failed");
    GraphStore st;
    GraphDev g;
    int rc = upload_plain(c, st, g, x, n, d);
    if (!rc) rc = nnm::mlp_grad(c, *model, g.x, (uint32_t)n, g.dp, triplets, ntrip, margin, loss, *grad);
    st.release();
    return rc;
}

int nnm_mlp_train(nnm_ctx* ctx, const float* x, uint64_t n, uint32_t d, const uint32_t* graph, uint32_t k,
                  const nnm_train_opts* opts, nnm_mlp* model, float* loss_trace) {
    if (!ctx || !x || !graph || n < 2 || n >= (1ull << 30) || k == 0) return NNM_ERR_INVALID;
    if (!mlp_ok(ctx, model, d)) return NNM_ERR_INVALID;
    nnm_train_opts o;
    if (opts) o = *opts;
    else nnm_train_opts_default(&o);
    if (o.steps == 0 || o.batch == 0 || o.batch > (1u << 20)) return fail(ctx, NNM_ERR_INVALID, "bad steps/batch");
    for (uint64_t i = 0; i < n * k; i++)
        if (graph[i] >= n) return fail(ctx, NNM_ERR_INVALID, "graph id out of range");
    Ctx& c = ctx->c;
    if (cudaSetDevice(c.device) != cudaSuccess) return fail(ctx, NNM_ERR_NO_DEVICE, "cudaSetDevice failed");
    GraphStore st;
    GraphDev g;
    nnm::DevBuf gd;
    int rc = upload_plain(c, st, g, x, n, d);
    if (!rc && gd.ensure(n * k * 4) != cudaSuccess) rc = fail(ctx, NNM_ERR_OOM, "device allocation failed");
    if (!rc && cudaMemcpy(gd.p, graph, n * k * 4, cudaMemcpyHostToDevice) != cudaSuccess) rc = NNM_ERR_CUDA;
    if (!rc) rc = nnm::mlp_train(c, g.x, (uint32_t)n, g.dp, gd.as<uint32_t>(), k, o, *model, loss_trace);
    gd.release();
    st.release();
    return rc;
}

void nnm_layers_free(nnm_layers* layers) {
    if (!layers) return;
    for (uint32_t l = 0; l < layers->nlayers && l < 16; l++) {
        std::free(layers->off[l]);
        std::free(layers->adj[l]);
        layers->off[l] = nullptr;
        layers->adj[l] = nullptr;
    }
    layers->nlayers = 0;
}

int nnm_search(nnm_ctx* ctx, const float* x, uint64_t n, uint32_t d, const nnm_layers* layers, const float* q,
               uint64_t nq, uint32_t topk, const nnm_opts* opts, uint32_t* out_ids, float* out_dists,
               uint64_t* ncmps) {
    if (!ctx) return NNM_ERR_INVALID;
    if (!x || !q || !layers || layers->nlayers < 1 || layers->nlayers > 16 || !out_ids)
        return fail(ctx, NNM_ERR_INVALID, "x, q, layers and out_ids are required");
    if (topk == 0 || topk > nnm::SEARCH_MAX_BEAM) return fail(ctx, NNM_ERR_INVALID, "topk must be in [1, 1024]");
    if (n >= (1ull << 30) || layers->nrows[layers->nlayers - 1] > n)
        return fail(ctx, NNM_ERR_INVALID, "layers do not match the data set");
    nnm_opts o;
    if (opts) o = *opts;
    else nnm_opts_default(&o);
    int rc;
    if (!opts_ok(ctx, &o, &rc)) return rc;
    Ctx& c = ctx->c;
    if (cudaSetDevice(c.device) != cudaSuccess) return fail(ctx, NNM_ERR_NO_DEVICE, "cudaSetDevice failed");
    return nnm::search_host(c, x, n, d, layers, q, nq, topk, o.seed, (int)o.metric, out_ids, out_dists, ncmps);
}

int nnm_graph_recall(nnm_ctx* ctx, const float* x, uint64_t n, uint32_t d, const uint32_t* ids, uint32_t k,
                     const uint32_t* rows, uint32_t nrows, uint32_t atop, double* recall) {
    if (!ctx || !x || !ids || !recall || (nrows && !rows) || n < 2 || n >= (1ull << 30) || d == 0 || d > 512 ||
        k == 0 || atop == 0 || atop > (uint32_t)nnm::EVAL_MAX_ATOP || atop > k)
        return ctx ? fail(ctx, NNM_ERR_INVALID, "recall: bad arguments (atop <= min(16, k), d <= 512)")
                   : NNM_ERR_INVALID;
    for (uint32_t i = 0; i < nrows; i++)
        if (rows[i] >= n) return fail(ctx, NNM_ERR_INVALID, "recall: row out of range");
    Ctx& c = ctx->c;
    if (cudaSetDevice(c.device) != cudaSuccess) return fail(ctx, NNM_ERR_NO_DEVICE, "cudaSetDevice failed");
    GraphStore st;
    GraphDev g;
    nnm::DevBuf ib, rb;
    int rc = upload_plain(c, st, g, x, n, d);
    if (!rc && (ib.ensure(n * k * 4) != cudaSuccess || rb.ensure((size_t)nrows * 4 + 4) != cudaSuccess))
        rc = fail(ctx, NNM_ERR_OOM, "device allocation failed");
    if (!rc && (cudaMemcpy(ib.p, ids, n * k * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
                (nrows && cudaMemcpy(rb.p, rows, (size_t)nrows * 4, cudaMemcpyHostToDevice) != cudaSuccess)))
        rc = NNM_ERR_CUDA;
    if (!rc)
        rc = nnm::graph_recall_dev(c, g.x, (uint32_t)n, g.dp, NNM_METRIC_L2, ib.as<uint32_t>(), k, rb.as<uint32_t>(),
                                   nrows, atop, recall);
    st.release();
    ib.release();
    rb.release();
    return rc;
}

void nnm_tune_opts_default(nnm_tune_opts* o) {
    std::memset(o, 0, sizeof(*o));
    o->target_recall = 0.95f;
    o->margin = 0.005f;
    o->sample_rows = 200000;
    o->eval_rows = 1000;
    o->repeats = 2;
}

int nnm_autotune_merge_leaves(nnm_ctx* ctx, const float* x_dev, uint64_t n, uint32_t d, uint32_t k,
                              const uint32_t* leaf_sizes, uint32_t nleaf, const nnm_opts* base,
                              const nnm_tune_opts* topts, nnm_opts* tuned, nnm_tune_result* result) {
    if (!ctx || !x_dev || !leaf_sizes || !tuned || nleaf < 2 || n < 2 || d == 0 || d > 512 || k < 10)
        return ctx ? fail(ctx, NNM_ERR_INVALID, "autotune: bad arguments (k >= 10, d <= 512)") : NNM_ERR_INVALID;
    nnm_opts b;
    if (base) b = *base;
    else nnm_opts_default(&b);
    nnm_tune_opts t;
    if (topts) t = *topts;
    else nnm_tune_opts_default(&t);
    if (t.repeats == 0) t.repeats = 1;
    Ctx& c = ctx->c;
    if (cudaSetDevice(c.device) != cudaSuccess) return fail(ctx, NNM_ERR_NO_DEVICE, "cudaSetDevice failed");
    // the sample: the first ns rows, leaves scaled to it
    const uint32_t ns = (uint32_t)std::min<uint64_t>(n, std::max<uint32_t>(t.sample_rows, 1000));
    std::vector<uint32_t> ls(nleaf);
    uint64_t acc = 0, tot = 0;
    for (uint32_t l = 0; l < nleaf; l++) tot += leaf_sizes[l];
    if (tot != n) return fail(ctx, NNM_ERR_INVALID, "leaf sizes must sum to n");
    for (uint32_t l = 0; l < nleaf; l++) {
        acc += leaf_sizes[l];
        ls[l] = (uint32_t)(acc * ns / n);
    }
    for (uint32_t l = nleaf - 1; l > 0; l--) ls[l] -= ls[l - 1];
    for (uint32_t l = 0; l < nleaf; l++)
        if (ls[l] < k + 2) return fail(ctx, NNM_ERR_INVALID, "autotune: a sampled leaf is too small");
    const uint32_t ne = std::min(t.eval_rows, ns);
    std::vector<uint32_t> rows(ne);
    {
        // seeded distinct rows: a stride walk from a seeded start
        std::mt19937 rng(b.seed + 77u);
        const uint64_t step = ns / ne, start = rng() % std::max<uint64_t>(step, 1);
        for (uint32_t i = 0; i < ne; i++) rows[i] = (uint32_t)(start + (uint64_t)i * step);
    }
    nnm::DevBuf ib, rb, xp;
    auto done = [&](int rc) {
        ib.release();
        rb.release();
        xp.release();
        return rc;
    };
    const uint32_t dp = (d + 3) & ~3u;
    if (ib.ensure((size_t)ns * k * 4) != cudaSuccess || rb.ensure((size_t)ne * 4) != cudaSuccess ||
        (dp != d && xp.ensure((size_t)ns * dp * 4) != cudaSuccess))
        return done(fail(ctx, NNM_ERR_OOM, "device allocation failed"));
    if (cudaMemcpy(rb.p, rows.data(), (size_t)ne * 4, cudaMemcpyHostToDevice) != cudaSuccess) return done(NNM_ERR_CUDA);
    const float* xe = x_dev;
    if (dp != d) {
        if (cudaMemset2D(xp.p, dp * 4, 0, dp * 4, ns) != cudaSuccess ||
            cudaMemcpy2D(xp.p, dp * 4, x_dev, d * 4, d * 4, ns, cudaMemcpyDeviceToDevice) != cudaSuccess)
            return done(NNM_ERR_CUDA);
        xe = xp.as<float>();
    }
    // the reference's cap (100) and convergence threshold (0.002) first
    static const uint32_t caps[] = {100, 88, 76, 64, 48};
    static const float deltas[] = {0.002f, 0.008f, 0.016f};
    nnm_tune_result res;
    std::memset(&res, 0, sizeof(res));
    int best = -1, best_rec = 0;
    for (uint32_t cap : caps)
        for (float dl : deltas) {
            nnm_opts o = b;
            o.sample_cap = cap;
            o.delta = dl;
            double ms = 1e30;
            for (uint32_t r = 0; r < t.repeats; r++) {
                nnm_stats stt;
                int rc = nnm_merge_leaves_dev(ctx, x_dev, ns, d, k, ls.data(), nleaf, &o, ib.as<uint32_t>(), nullptr,
                                              nullptr, &stt);
                if (rc) return done(rc);
                ms = std::min(ms, stt.device_ms);
            }
            double rec = 0.0;
            int rc = nnm::graph_recall_dev(c, xe, ns, dp, (int)o.metric, ib.as<uint32_t>(), k, rb.as<uint32_t>(), ne,
                                           10, &rec);
            if (rc) return done(rc);
            const uint32_t i = res.ntrials++;
            res.trials[i] = nnm_tune_trial{cap, dl, (float)rec, b.tile_rows ? b.tile_rows : 128u, ms};
            if (rec >= (double)(t.target_recall + t.margin) && (best < 0 || ms < res.trials[best].ms)) best = (int)i;
            if (rec > res.trials[best_rec].recall) best_rec = (int)i;
        }
    res.chosen = best >= 0 ? (uint32_t)best : (uint32_t)best_rec;
    // then the tile shape at the chosen cap and threshold: the longest lists
    // joined in tensor-core tiles (the graphs are the same; only time decides)
    for (uint32_t tr : {64u, 32u}) {
        nnm_opts o = b;
        o.sample_cap = res.trials[res.chosen].sample_cap;
        o.delta = res.trials[res.chosen].delta;
        o.tile_rows = tr;
        double ms = 1e30;
        for (uint32_t r = 0; r < t.repeats; r++) {
            nnm_stats stt;
            int rc = nnm_merge_leaves_dev(ctx, x_dev, ns, d, k, ls.data(), nleaf, &o, ib.as<uint32_t>(), nullptr,
                                          nullptr, &stt);
            if (rc) return done(rc);
            ms = std::min(ms, stt.device_ms);
        }
        const uint32_t i = res.ntrials++;
        res.trials[i] = nnm_tune_trial{o.sample_cap, o.delta, res.trials[res.chosen].recall, tr, ms};
        if (ms < res.trials[res.chosen].ms) res.chosen = i;
    }
    *tuned = b;
    tuned->sample_cap = res.trials[res.chosen].sample_cap;
    tuned->delta = res.trials[res.chosen].delta;
    tuned->tile_rows = res.trials[res.chosen].tile_rows;
    if (result) *result = res;
    return done(0);
}

int nnm_index_create(nnm_ctx* ctx, const float* x, uint64_t n, uint32_t d, const nnm_layers* layers, uint32_t seed,
                     uint32_t metric, nnm_index** out) {
    if (!ctx || !out) return NNM_ERR_INVALID;
    *out = nullptr;
    if (!x || !layers || n == 0 || d == 0 || layers->nlayers < 1 || layers->nlayers > 16)
        return fail(ctx, NNM_ERR_INVALID, "x and 1..16 layers are required, n, d > 0");
    if (n >= (1ull << 30) || layers->nrows[layers->nlayers - 1] > n)
        return fail(ctx, NNM_ERR_INVALID, "layers do not match the data set");
    if (metric > NNM_METRIC_CHI2) return fail(ctx, NNM_ERR_UNSUPPORTED_METRIC, "unknown metric");
    Ctx& c = ctx->c;
    if (cudaSetDevice(c.device) != cudaSuccess) return fail(ctx, NNM_ERR_NO_DEVICE, "cudaSetDevice failed");
    std::unique_ptr<nnm_index> h(new nnm_index());
    h->ctx = ctx;
    int rc = nnm::index_upload(c, h->ix, x, n, d, layers, seed, metric);
    if (!rc && cudaStreamSynchronize(c.stream) != cudaSuccess) rc = fail(ctx, NNM_ERR_CUDA, "index upload failed");
    if (rc) {
        h->ix.release();
        return rc;
    }
    *out = h.release();
    return NNM_OK;
}

int nnm_index_free(nnm_index* h) {
    if (!h) return NNM_OK;
    cudaSetDevice(h->ctx->c.device);
    cudaStreamSynchronize(h->ctx->c.stream);
    if (h->ix.net) {
        h->ix.net->release();
        delete h->ix.net;
    }
    h->ix.release();
    delete h;
    return NNM_OK;
}

namespace {
int index_search_impl(nnm_index* h, const float* q, uint64_t nq, const uint32_t* beams, uint32_t beam,
                      uint32_t out_k, uint32_t smode, uint32_t emode, uint32_t* out_ids, float* out_d,
                      nnm_search_stats* stats, bool dev) {
    if (!h) return NNM_ERR_INVALID;
    nnm_ctx* ctx = h->ctx;
    Ctx& c = ctx->c;
    nnm::IndexDev& ix = h->ix;
    if (stats) std::memset(stats, 0, sizeof(*stats));
    if (nq == 0) return NNM_OK;
    if (!q || !out_ids) return fail(ctx, NNM_ERR_INVALID, "q and out_ids are required");
    if (nq >= (1ull << 31)) return fail(ctx, NNM_ERR_INVALID, "nq must be below 2^31");
    if (smode > NNM_SERVE_FAST || emode > NNM_ENTRY_FLAT) return fail(ctx, NNM_ERR_INVALID, "unknown mode");
    if (emode == NNM_ENTRY_LEARNED && !ix.net) return fail(ctx, NNM_ERR_INVALID, "no entry model set");
    if (out_k == 0) return fail(ctx, NNM_ERR_INVALID, "out_k must be positive");
    uint32_t bmax = beam;
    if (beams && !dev) {
        bmax = 0;
        for (uint64_t i = 0; i < nq; i++) {
            if (beams[i] < out_k || beams[i] > nnm::SEARCH_MAX_BEAM)
                return fail(ctx, NNM_ERR_INVALID, "every beam width must be in [out_k, 1024]");
            bmax = std::max(bmax, beams[i]);
        }
    } else if (beam < out_k || beam > nnm::SEARCH_MAX_BEAM) {
        return fail(ctx, NNM_ERR_INVALID, "beam must be in [out_k, 1024]");
    }
    if (cudaSetDevice(c.device) != cudaSuccess) return fail(ctx, NNM_ERR_NO_DEVICE, "cudaSetDevice failed");
    cudaStream_t st = c.stream;
    const uint32_t d = ix.d, dp = ix.dp;
    auto cu = [&](cudaError_t e) {
        if (e == cudaSuccess) return 0;
        c.last_error = cudaGetErrorString(e);
        return e == cudaErrorMemoryAllocation ? (int)NNM_ERR_OOM : (int)NNM_ERR_CUDA;
    };
    int rc = 0;
    // queries with rows of dp floats
    const float* qd = q;
    if (!dev || dp != d) {
        if ((rc = cu(ix.qpad.ensure((size_t)nq * dp * 4)))) return rc;
        const cudaMemcpyKind kind = dev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
        if (dp == d) rc = cu(cudaMemcpyAsync(ix.qpad.p, q, (size_t)nq * d * 4, kind, st));
        else {
            rc = cu(cudaMemset2DAsync(ix.qpad.p, dp * 4, 0, dp * 4, nq, st));
            if (!rc) rc = cu(cudaMemcpy2DAsync(ix.qpad.p, dp * 4, q, d * 4, d * 4, nq, kind, st));
        }
        if (rc) return rc;
        qd = ix.qpad.as<float>();
    }
    const uint32_t* bd = beams;
    if (beams && !dev) {
        if ((rc = cu(ix.beams.ensure((size_t)nq * 4)))) return rc;
        if ((rc = cu(cudaMemcpyAsync(ix.beams.p, beams, (size_t)nq * 4, cudaMemcpyHostToDevice, st)))) return rc;
        bd = ix.beams.as<uint32_t>();
    }
    uint32_t* oi = out_ids;
    float* od = out_d;
    if (!dev) {
        if ((rc = cu(ix.out.ensure((size_t)nq * out_k * 8)))) return rc;
        oi = ix.out.as<uint32_t>();
        od = out_d ? reinterpret_cast<float*>(oi + (size_t)nq * out_k) : nullptr;
    }
    nnm::SearchReq r{};
    r.q = qd;
    r.nq = (uint32_t)nq;
    r.beams = bd;
    r.beam = beam;
    r.beam_max = bmax;
    r.out_k = out_k;
    r.out_ids = oi;
    r.out_d = od;
    if ((rc = cu(cudaMemsetAsync(ix.ctr.p, 0, 64, st)))) return rc;
    cudaEvent_t ev[3];
    for (auto& e : ev) cudaEventCreate(&e);
    cudaEventRecord(ev[0], st);
    if (emode == NNM_ENTRY_LEARNED) {
        rc = cu(ix.probes.ensure((size_t)nq * ix.nprobe * 4));
        if (!rc)
            rc = nnm::entry_predict(c, ix, qd, (uint32_t)nq, ix.probes.as<uint32_t>(),
                                    reinterpret_cast<unsigned*>(ix.ctr.as<unsigned char>() + 4));
        r.probes = ix.probes.as<uint32_t>();
        r.nprobe = ix.nprobe;
        r.g0 = ix.entry_layer;
    } else if (emode == NNM_ENTRY_FLAT) {
        rc = nnm::index_flat_seeds(c, ix, bmax);
        r.flat = 1;
        r.flat_off = ix.flat_off.as<uint32_t>();
        r.flat_pool = ix.flat_pool.as<uint32_t>();
    }
    cudaEventRecord(ev[1], st);
    if (!rc) rc = smode == NNM_SERVE_FAST ? nnm::index_run_fast(c, ix, r) : nnm::index_run_exact(c, ix, r);
    cudaEventRecord(ev[2], st);
    uint64_t ncmps = 0, nexp = 0;
    if (!rc) rc = nnm::index_counters(c, ix, &ncmps, &nexp);
    if (!rc && !dev) {
        rc = cu(cudaMemcpyAsync(out_ids, oi, (size_t)nq * out_k * 4, cudaMemcpyDeviceToHost, st));
        if (!rc && out_d) rc = cu(cudaMemcpyAsync(out_d, od, (size_t)nq * out_k * 4, cudaMemcpyDeviceToHost, st));
        if (!rc) rc = cu(cudaStreamSynchronize(st));
    }
    if (!rc && stats) {
        float a = 0.f, b = 0.f;
        cudaEventElapsedTime(&a, ev[0], ev[1]);
        cudaEventElapsedTime(&b, ev[1], ev[2]);
        stats->ncmps = ncmps;
        stats->expansions = nexp;
        stats->predict_ms = a;
        stats->device_ms = a + b;
    }
    for (auto& e : ev) cudaEventDestroy(e);
    return rc;
}

bool entry_ok(nnm_ctx* ctx, const nnm_entry_mlp* m, uint32_t d) {
    if (!m || !m->w1 || !m->b1 || !m->w2 || !m->b2) {
        fail(ctx, NNM_ERR_INVALID, "model arrays must be non-null");
        return false;
    }
    if (m->d_in != d || d == 0 || d > nnm::ENTRY_MAX_D) {
        fail(ctx, NNM_ERR_INVALID, "model d_in must equal d and be in [1, 256]");
        return false;
    }
    if (m->n_classes == 0 || m->n_classes > nnm::ENTRY_MAX_C) {
        fail(ctx, NNM_ERR_INVALID, "n_classes must be in [1, 4096]");
        return false;
    }
    return true;
}
}  // namespace

int nnm_index_search(nnm_index* ix, const float* q, uint64_t nq, const uint32_t* beams, uint32_t beam, uint32_t out_k,
                     uint32_t serve_mode, uint32_t entry_mode, uint32_t* out_ids, float* out_dists,
                     nnm_search_stats* stats) {
    return index_search_impl(ix, q, nq, beams, beam, out_k, serve_mode, entry_mode, out_ids, out_dists, stats, false);
}

int nnm_index_search_dev(nnm_index* ix, const float* q, uint64_t nq, const uint32_t* beams, uint32_t beam,
                         uint32_t out_k, uint32_t serve_mode, uint32_t entry_mode, uint32_t* out_ids,
                         float* out_dists, nnm_search_stats* stats) {
    return index_search_impl(ix, q, nq, beams, beam, out_k, serve_mode, entry_mode, out_ids, out_dists, stats, true);
}

int nnm_index_set_width(nnm_index* h, uint32_t width) {
    if (!h) return NNM_ERR_INVALID;
    if (width < 1 || width > 4) return fail(h->ctx, NNM_ERR_INVALID, "width must be in [1, 4]");
    h->ix.width = width;
    return NNM_OK;
}

int nnm_index_tune_width(nnm_index* h, const float* q, uint64_t nq, const uint32_t* beams, uint32_t beam,
                         uint32_t out_k, uint32_t entry_mode, uint32_t repeats, uint32_t* width, double* ms) {
    if (!h || !width || nq == 0) return h ? fail(h->ctx, NNM_ERR_INVALID, "tune: queries and width are required")
                                          : NNM_ERR_INVALID;
    std::vector<uint32_t> ids((size_t)nq * out_k);
    const uint32_t keep = h->ix.width;
    double best = 1e300;
    uint32_t bw = keep;
    for (uint32_t w = 1; w <= 4; w++) {
        h->ix.width = w;
        double t = 1e300;
        for (uint32_t r = 0; r < std::max(1u, repeats); r++) {
            nnm_search_stats st;
            int rc = index_search_impl(h, q, nq, beams, beam, out_k, NNM_SERVE_FAST, entry_mode, ids.data(), nullptr,
                                       &st, false);
            if (rc) {
                h->ix.width = keep;
                return rc;
            }
            t = std::min(t, st.device_ms - st.predict_ms);
        }
        if (ms) ms[w - 1] = t;
        if (t < best) {
            best = t;
            bw = w;
        }
    }
    h->ix.width = bw;
    *width = bw;
    return NNM_OK;
}

int nnm_index_entry_layer(const nnm_index* h, uint32_t* layer, uint32_t* n_classes) {
    if (!h || !layer || !n_classes) return NNM_ERR_INVALID;
    const nnm::IndexDev& ix = h->ix;
    for (int g = (int)ix.L - 1; g >= 0; g--)
        if (ix.nrows[g] <= nnm::ENTRY_MAX_C) {
            *layer = (uint32_t)g;
            *n_classes = ix.nrows[g];
            return NNM_OK;
        }
    *layer = 0;  // rows 0..4095, a prefix of the top layer
    *n_classes = nnm::ENTRY_MAX_C;
    return NNM_OK;
}

namespace {
// Scores (when scores is non-null) or probes of x through the inference kernels.
int entry_infer_host(nnm_ctx* ctx, const nnm_entry_mlp* model, const float* x, uint64_t n, uint32_t d,
                     float* scores, uint32_t P, uint32_t* probes) {
    Ctx& c = ctx->c;
    if (cudaSetDevice(c.device) != cudaSuccess) return fail(ctx, NNM_ERR_NO_DEVICE, "cudaSetDevice failed");
    nnm::DevEntry m;
    GraphStore st;
    GraphDev g;
    nnm::DevBuf hb, ob, eb;
    const size_t out_bytes = scores ? n * model->n_classes * 4 : n * P * 4;
    int rc = nnm::entry_upload(c, m, *model);
    if (!rc) rc = upload_plain(c, st, g, x, n, d);
    if (!rc && (hb.ensure(n * nnm::ENTRY_H * 2) != cudaSuccess || ob.ensure(out_bytes) != cudaSuccess ||
                eb.ensure(16) != cudaSuccess))
        rc = fail(ctx, NNM_ERR_OOM, "device allocation failed");
    if (!rc && cudaMemsetAsync(eb.p, 0, 16, c.stream) != cudaSuccess) rc = NNM_ERR_CUDA;
    if (!rc)
        rc = nnm::entry_infer(c, m, g.x, (uint32_t)n, g.dp, hb.p, scores ? ob.as<float>() : nullptr, P,
                              scores ? nullptr : ob.as<uint32_t>(), eb.as<unsigned>());
    if (!rc && cudaStreamSynchronize(c.stream) != cudaSuccess) rc = fail(ctx, NNM_ERR_CUDA, "entry inference failed");
    unsigned e = 0;
    if (!rc && cudaMemcpy(&e, eb.p, 4, cudaMemcpyDeviceToHost) != cudaSuccess) rc = NNM_ERR_CUDA;
    if (!rc && e) rc = fail(ctx, NNM_ERR_CAPACITY, "entry inference: a bounded wait ran out");
    if (!rc && cudaMemcpy(scores ? (void*)scores : (void*)probes, ob.p, out_bytes, cudaMemcpyDeviceToHost) !=
                   cudaSuccess)
        rc = NNM_ERR_CUDA;
    m.release();
    st.release();
    hb.release();
    ob.release();
    eb.release();
    return rc;
}
}  // namespace

int nnm_entry_forward(nnm_ctx* ctx, const nnm_entry_mlp* model, const float* x, uint64_t n, uint32_t d,
                      float* scores) {
    if (!ctx || !x || !scores || n == 0 || n >= (1ull << 30)) return NNM_ERR_INVALID;
    if (!entry_ok(ctx, model, d)) return NNM_ERR_INVALID;
    return entry_infer_host(ctx, model, x, n, d, scores, 0, nullptr);
}

int nnm_entry_probes(nnm_ctx* ctx, const nnm_entry_mlp* model, const float* x, uint64_t n, uint32_t d,
                     uint32_t probes, uint32_t* out) {
    if (!ctx || !x || !out || n == 0 || n >= (1ull << 30)) return NNM_ERR_INVALID;
    if (!entry_ok(ctx, model, d)) return NNM_ERR_INVALID;
    if (probes == 0 || probes > (uint32_t)nnm::ENTRY_MAX_PROBES || probes > model->n_classes)
        return fail(ctx, NNM_ERR_INVALID, "probes must be in [1, min(8, n_classes)]");
    return entry_infer_host(ctx, model, x, n, d, nullptr, probes, out);
}

int nnm_entry_grad(nnm_ctx* ctx, const nnm_entry_mlp* model, const float* x, uint64_t n, uint32_t d,
                   const uint32_t* labels, float* loss, nnm_entry_mlp* grad) {
    if (!ctx || !x || !labels || !loss || !grad || n == 0 || n >= (1ull << 24)) return NNM_ERR_INVALID;
    if (!entry_ok(ctx, model, d) || !entry_ok(ctx, grad, d)) return NNM_ERR_INVALID;
    if (grad->n_classes != model->n_classes) return fail(ctx, NNM_ERR_INVALID, "grad must have the model's shapes");
    for (uint64_t i = 0; i < n; i++)
        if (labels[i] >= model->n_classes) return fail(ctx, NNM_ERR_INVALID, "label out of range");
    Ctx& c = ctx->c;
    if (cudaSetDevice(c.device) != cudaSuccess) return fail(ctx, NNM_ERR_NO_DEVICE, "cudaSetDevice failed");
    GraphStore st;
    GraphDev g;
    int rc = upload_plain(c, st, g, x, n, d);
    if (!rc) rc = nnm::entry_grad(c, *model, g.x, (uint32_t)n, g.dp, labels, loss, *grad);
    st.release();
    return rc;
}

int nnm_entry_train(nnm_index* h, nnm_entry_mlp* model, const nnm_train_opts* opts, float* loss_trace) {
    if (!h) return NNM_ERR_INVALID;
    nnm_ctx* ctx = h->ctx;
    nnm::IndexDev& ix = h->ix;
    if (!entry_ok(ctx, model, ix.d)) return NNM_ERR_INVALID;
    if (model->n_classes > ix.n) return fail(ctx, NNM_ERR_INVALID, "more classes than rows");
    if (ix.metric != NNM_METRIC_L2) return fail(ctx, NNM_ERR_UNSUPPORTED_METRIC, "entry training needs L2");
    nnm_train_opts o;
    if (opts) o = *opts;
    else nnm_train_opts_default(&o);
    if (o.steps == 0 || o.batch == 0 || o.batch > (1u << 16)) return fail(ctx, NNM_ERR_INVALID, "bad training opts");
    Ctx& c = ctx->c;
    if (cudaSetDevice(c.device) != cudaSuccess) return fail(ctx, NNM_ERR_NO_DEVICE, "cudaSetDevice failed");
    return nnm::entry_train(c, ix, 0, o, *model, loss_trace);
}

int nnm_index_set_entry_model(nnm_index* h, const nnm_entry_mlp* model, uint32_t probes) {
    if (!h) return NNM_ERR_INVALID;
    nnm_ctx* ctx = h->ctx;
    nnm::IndexDev& ix = h->ix;
    Ctx& c = ctx->c;
    if (cudaSetDevice(c.device) != cudaSuccess) return fail(ctx, NNM_ERR_NO_DEVICE, "cudaSetDevice failed");
    if (!model) {
        if (ix.net) {
            cudaStreamSynchronize(c.stream);
            ix.net->release();
            delete ix.net;
            ix.net = nullptr;
        }
        return NNM_OK;
    }
    if (!entry_ok(ctx, model, ix.d)) return NNM_ERR_INVALID;
    if (model->n_classes > ix.n) return fail(ctx, NNM_ERR_INVALID, "more classes than rows");
    if (probes == 0 || probes > (uint32_t)nnm::ENTRY_MAX_PROBES || probes > model->n_classes)
        return fail(ctx, NNM_ERR_INVALID, "probes must be in [1, min(8, n_classes)]");
    if (!ix.net) ix.net = new nnm::DevEntry();
    int rc = nnm::entry_upload(c, *ix.net, *model);
    if (rc) return rc;
    // the descent starts on the first layer that holds every class row
    uint32_t g0 = ix.L - 1;
    for (uint32_t g = 0; g < ix.L; g++)
        if (ix.nrows[g] >= model->n_classes) {
            g0 = g;
            break;
        }
    ix.entry_layer = g0;
    ix.n_classes = model->n_classes;
    ix.nprobe = probes;
    return NNM_OK;
}

}  // extern "C"
