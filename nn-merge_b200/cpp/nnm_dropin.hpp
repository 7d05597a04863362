// Drop-in replacements for the reference's hot-path classes, implemented
// over the C ABI of include/nnm.h.  Include this header instead of the
// reference's kgraph.h, smerge.h, jmerge.h, lynndescent.h, lysearch.h and
// space_lp.h; link with -lnnm.  Names, constructors and the virtual
// interface follow the reference:
//   AbstractGraph    abstractgraph.h:21-45
//   KGraph           kgraph.h:126-150   (buildKGraph returns new unsigned[n*k])
//   AbstractMerge    abstractmerge.h:16-40 (InitSGraph, InitialGraph,
//                    nnDescent, localJoin, merge2one, cutMat, EvaluateDelta)
//   Smerge, Jmerge   smerge.h:8-23, jmerge.h:7-22 (buildKGraph returns 0)
//   LyNNDescent      lynndescent.h:19-86 (buildhgraph(src, dst, grd, K, M))
//   LySearch         lysearch.h:23-91   (knnSearch is public here)
//   L2space, L1space, Ksquare  space_lp.h:9-53
// The reference seeds every phase from time(NULL); so do these classes,
// unless the environment variable NNM_SEED fixes the seed.  Errors print
// the library's message and exit, as the reference exits on failures.
#ifndef NNM_DROPIN_HPP
#define NNM_DROPIN_HPP

#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <fstream>
#include <iostream>
#include <map>
#include <string>
#include <vector>

#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include "../../include/nnm.h"

template <typename MTYPE>
using DISTFUNC = MTYPE (*)(const float *, const unsigned long s1, const float *, const unsigned long s2,
                           const unsigned int d0);

template <typename MTYPE>
class SpaceInterface {
public:
    virtual DISTFUNC<MTYPE> get_dist_func() = 0;
    // Which device metric this space is; spaces the engine does not
    // implement return -1 and are rejected with NNM_ERR_UNSUPPORTED_METRIC.
    virtual int nnm_metric() const { return -1; }
    virtual ~SpaceInterface() {}
};

namespace nnm_dropin {

inline float l2norm(const float *v1, const unsigned long s1, const float *v2, const unsigned long s2,
                    const unsigned int d0) {
    float res = 0.f;
    for (unsigned i = 0; i < d0; i++) {
        float diff = v1[s1 * d0 + i] - v2[s2 * d0 + i];
        res += diff * diff;
    }
    return res;
}
inline float l1norm(const float *v1, const unsigned long s1, const float *v2, const unsigned long s2,
                    const unsigned int d0) {
    float res = 0.f;
    for (unsigned i = 0; i < d0; i++) res += std::fabs(v1[s1 * d0 + i] - v2[s2 * d0 + i]);
    return res;
}
inline float ksquare(const float *v1, const unsigned long s1, const float *v2, const unsigned long s2,
                     const unsigned int d0) {
    float w2 = 0.f;
    for (unsigned i = 0; i < d0; i++) {
        float a = v1[s1 * d0 + i], b = v2[s2 * d0 + i], w1 = a - b;
        if (a != 0 || b != 0) w2 += w1 * w1 / (a + b);
    }
    return w2;
}

inline nnm_ctx *context() {
    static nnm_ctx *ctx = nullptr;
    if (!ctx) {
        int rc = nnm_ctx_create(0, &ctx);
        if (rc != NNM_OK) {
            std::cout << "nnm: " << nnm_status_string(rc) << std::endl;
            std::exit(0);
        }
    }
    return ctx;
}

inline void check(int rc) {
    if (rc != NNM_OK) {
        std::cout << "nnm: " << nnm_status_string(rc) << ": " << nnm_last_error(context()) << std::endl;
        std::exit(0);
    }
}

inline nnm_opts opts(int metric) {
    nnm_opts o;
    nnm_opts_default(&o);
    const char *env = std::getenv("NNM_SEED");
    o.seed = env ? (uint32_t)std::strtoul(env, nullptr, 10) : (uint32_t)time(NULL);
    if (metric < 0) check(NNM_ERR_UNSUPPORTED_METRIC);
    o.metric = (uint32_t)metric;
    return o;
}

inline bool ends_with(const char *fn, const char *e) {
    const size_t a = std::strlen(fn), l = std::strlen(e);
    return a >= l && std::strcmp(fn + a - l, e) == 0;
}

// A read-only memory map of a whole file (the fast path of the binary
// readers: no stream buffering, one copy out of the page cache).
struct MappedFile {
    const unsigned char *p = nullptr;
    size_t size = 0;
    explicit MappedFile(const char *fn) {
        const int fd = ::open(fn, O_RDONLY);
        if (fd < 0) return;
        struct stat st;
        if (::fstat(fd, &st) == 0 && st.st_size > 0) {
            void *m = ::mmap(nullptr, (size_t)st.st_size, PROT_READ, MAP_PRIVATE, fd, 0);
            if (m != MAP_FAILED) {
                p = static_cast<const unsigned char *>(m);
                size = (size_t)st.st_size;
                ::madvise(m, size, MADV_SEQUENTIAL);
            }
        }
        ::close(fd);
    }
    ~MappedFile() {
        if (p) ::munmap(const_cast<unsigned char *>(p), size);
    }
    MappedFile(const MappedFile &) = delete;
    MappedFile &operator=(const MappedFile &) = delete;
};

// IODelegator::load_refSet (iodelegator.cpp:159-182): .fvecs
// (load_fvecs, :222-265), .bvecs (loadBvec10m, :319-385: at most 10^7
// rows, bytes to floats) and .txt ("rows cols" then the values, loadMatrix
// :186-220).  The binary formats are read through a memory map.
inline float *load_refSet(const char *fn, unsigned &d, unsigned &r) {
    if (ends_with(fn, ".txt")) {
        std::ifstream in(fn);
        if (!in) { std::cout << "Fail to read " << fn << std::endl; std::exit(0); }
        float a, b;
        in >> a >> b;
        r = (unsigned)std::lround(a);
        d = (unsigned)std::lround(b);
        float *m = new float[(size_t)r * d];
        for (size_t i = 0; i < (size_t)r * d; i++) in >> m[i];
        return m;
    }
    const bool bytes = ends_with(fn, ".bvecs");
    if (!bytes && !ends_with(fn, ".fvecs")) { std::cout << "unknown format " << fn << std::endl; std::exit(0); }
    MappedFile f(fn);
    if (!f.p || f.size < 4) { std::cout << "File '" << fn << "' cannot open for read!" << std::endl; std::exit(0); }
    uint32_t dim = 0;
    std::memcpy(&dim, f.p, 4);
    const size_t rec = 4 + (size_t)dim * (bytes ? 1 : 4);
    size_t rows = f.size / rec;
    if (bytes && rows > 10000000) rows = 10000000;
    r = (unsigned)rows;
    d = dim;
    float *m = new float[(size_t)r * d];
    for (size_t i = 0; i < rows; i++) {
        const unsigned char *src = f.p + i * rec + 4;
        if (bytes)
            for (unsigned j = 0; j < d; j++) m[i * d + j] = (float)src[j];
        else
            std::memcpy(m + i * d, src, (size_t)d * 4);
    }
    return m;
}

// The k-NN graph text format (abstractmerge.cpp:278-291, kgraph.cpp:247-261),
// read back by the reference's IODelegator::loadKNNGraph
// (iodelegator.cpp:65-102).
inline void save_knn(const char *dst, const std::vector<uint32_t> &ids, unsigned n, unsigned k) {
    std::ofstream out(dst);
    out << n << " " << k << std::endl;
    for (unsigned i = 0; i < n; i++) {
        out << i << " " << k << " ";
        for (unsigned j = 0; j < k; j++) out << ids[(size_t)i * k + j] << " ";
        out << std::endl;
    }
}

// Binary k-NN graph (no counterpart in the reference; for graphs whose text
// form would dominate the build time): the bytes "NNMK", u32 version 1,
// u32 n, u32 k, then n x k u32 ids, row-major, little endian.
constexpr char KNN_MAGIC[4] = {'N', 'N', 'M', 'K'};

inline void save_knn_bin(const char *dst, const std::vector<uint32_t> &ids, unsigned n, unsigned k) {
    FILE *f = std::fopen(dst, "wb");
    if (!f) { std::cout << "File '" << dst << "' cannot open for write!" << std::endl; std::exit(0); }
    const uint32_t hdr[3] = {1u, n, k};
    std::fwrite(KNN_MAGIC, 1, 4, f);
    std::fwrite(hdr, 4, 3, f);
    std::fwrite(ids.data(), 4, (size_t)n * k, f);
    std::fclose(f);
}

// Either form, told apart by the magic: returns new unsigned[n * k] as
// IODelegator::loadKNNGraph returns its array (topk = k).
inline unsigned *load_knn(const char *fn, unsigned &n, unsigned &k) {
    {
        MappedFile f(fn);
        if (f.p && f.size >= 16 && std::memcmp(f.p, KNN_MAGIC, 4) == 0) {
            uint32_t hdr[3];
            std::memcpy(hdr, f.p + 4, 12);
            n = hdr[1];
            k = hdr[2];
            if (hdr[0] != 1 || f.size < 16 + (size_t)n * k * 4) {
                std::cout << "File '" << fn << "' is not a version-1 graph" << std::endl;
                std::exit(0);
            }
            unsigned *g = new unsigned[(size_t)n * k];
            std::memcpy(g, f.p + 16, (size_t)n * k * 4);
            return g;
        }
    }
    std::ifstream in(fn);
    if (!in) { std::cout << "File '" << fn << "' cannot open for read!" << std::endl; std::exit(0); }
    in >> n >> k;
    unsigned *g = new unsigned[(size_t)n * k]();
    for (unsigned i = 0; i < n && in; i++) {
        unsigned idx, num, v;
        in >> idx >> num;
        for (unsigned j = 0; j < num; j++) {
            in >> v;
            if (j < k) g[(size_t)i * k + j] = v;
        }
    }
    return g;
}

}  // namespace nnm_dropin

class L2space : public SpaceInterface<float> {
public:
    DISTFUNC<float> get_dist_func() override { return nnm_dropin::l2norm; }
    int nnm_metric() const override { return NNM_METRIC_L2; }
};
class L1space : public SpaceInterface<float> {
public:
    DISTFUNC<float> get_dist_func() override { return nnm_dropin::l1norm; }
    int nnm_metric() const override { return NNM_METRIC_L1; }
};
class Ksquare : public SpaceInterface<float> {
public:
    DISTFUNC<float> get_dist_func() override { return nnm_dropin::ksquare; }
    int nnm_metric() const override { return NNM_METRIC_CHI2; }
};

class AbstractGraph {
protected:
    unsigned K0 = 0, row = 0, col = 0;
    float *mat = nullptr;
    int metric = NNM_METRIC_L2;
    std::vector<uint32_t> ids_;

public:
    unsigned long nCmps = 0;
    AbstractGraph() {}
    explicit AbstractGraph(SpaceInterface<float> *func) { metric = func->nnm_metric(); }
    virtual ~AbstractGraph() {
        delete[] mat;  // the reference frees the caller's matrix too (abstractgraph.cpp:43-47)
        mat = nullptr;
    }
    virtual unsigned InitialMemory(float *mata, const unsigned k, const unsigned n, const unsigned d) {
        mat = mata;
        K0 = k;
        row = n;
        col = d;
        nCmps = 0;
        return 0;
    }
    virtual unsigned InitialGraph() { return 0; }  // part of the device build
    virtual unsigned *buildKGraph(float *mata, const unsigned K, const unsigned N, const unsigned D) = 0;
    // The reference's text format; a name ending in ".knng" gets the
    // binary form instead.
    virtual void saveKGraph(const char *dst) {
        if (nnm_dropin::ends_with(dst, ".knng")) nnm_dropin::save_knn_bin(dst, ids_, row, K0);
        else nnm_dropin::save_knn(dst, ids_, row, K0);
    }
    virtual void setdisfunc(SpaceInterface<float> *func) { metric = func->nnm_metric(); }
};

class KGraph : public AbstractGraph {
public:
    KGraph() {}
    explicit KGraph(SpaceInterface<float> *func) : AbstractGraph(func) {}
    unsigned *buildKGraph(float *mata, const unsigned k, const unsigned n, const unsigned d) override {
        InitialMemory(mata, k, n, d);
        nnm_opts o = nnm_dropin::opts(metric);
        nnm_stats st;
        ids_.resize((size_t)n * k);
        auto t0 = std::chrono::steady_clock::now();
        nnm_dropin::check(nnm_kgraph_build(nnm_dropin::context(), mata, n, d, k, &o, ids_.data(), nullptr, nullptr, &st));
        std::cout << "Construction time ..............................times = "
                  << std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() << std::endl;
        nCmps = st.ncmps;
        unsigned *out = new unsigned[(size_t)n * k];
        std::memcpy(out, ids_.data(), sizeof(unsigned) * (size_t)n * k);
        return out;
    }
};

// One entry of a pool as the reference's merges keep it (pvetex.h:18-30).
struct Neighbor {
    unsigned id = 0;
    float dist = 0.f;
    bool flag = false;
    unsigned gd = 0;
};
typedef std::vector<Neighbor> Neighbors;

// AbstractMerge (abstractmerge.h:16-40) over a device session (nnm_merge_*):
// the pools and compensation lists -- the reference's egraph -- live on the
// device from InitialMemory on, and every step below is one call of the
// session, in the reference's order giving the reference's graph.
//
// The local join runs inside nnDescent() on the device with the filter that
// join_filter() names: Smerge's and Jmerge's (groups differ; or either
// group is 1).  A subclass whose localJoin() is its own host code cannot
// run on the device: its nnDescent() ends with NNM_ERR_INVALID unless it
// also overrides join_filter() to pick one of the device filters.
class AbstractMerge : public AbstractGraph {
protected:
    nnm_merge *egraph = nullptr;
    unsigned preSize = 0;

    // NNM_MERGE_SMERGE / NNM_MERGE_JMERGE, or -1: no device filter
    virtual int join_filter() const { return -1; }

    nnm_opts session_opts() const { return nnm_dropin::opts(metric); }

public:
    AbstractMerge() {}
    explicit AbstractMerge(SpaceInterface<float> *func) : AbstractGraph(func) {}
    ~AbstractMerge() override {
        if (egraph) nnm_merge_free(egraph);
    }
    // AbstractMerge::InitialMemory (abstractmerge.cpp:25-35): the matrix to
    // the device, empty pools.
    unsigned InitialMemory(float *mata, const unsigned k, const unsigned n, const unsigned d) override {
        AbstractGraph::InitialMemory(mata, k, n, d);
        if (egraph) nnm_merge_free(egraph);
        egraph = nullptr;
        nnm_opts o = session_opts();
        nnm_dropin::check(nnm_merge_create(nnm_dropin::context(), mata, n, d, k, &o, &egraph));
        return 0;
    }
    unsigned InitialGraph() override = 0;
    unsigned *buildKGraph(float *mata, const unsigned K, const unsigned N, const unsigned D) override = 0;
    // abstractmerge.cpp:278-291, from the device pools
    void saveKGraph(const char *dst) override {
        if (egraph) {
            ids_.resize((size_t)row * K0);
            nnm_dropin::check(nnm_merge_read(egraph, ids_.data(), nullptr, nullptr));
        }
        AbstractGraph::saveKGraph(dst);
    }
    // AbstractMerge::nnDescent (abstractmerge.cpp:78-192): sampling,
    // shuffles, this class's local join and the convergence test, repeated
    // on the device until the reference's test passes.
    virtual unsigned nnDescent() {
        const int f = join_filter();
        if (f < 0) {
            std::cout << "nnm: this class's localJoin() has no device form (override join_filter())" << std::endl;
            nnm_dropin::check(NNM_ERR_INVALID);
        }
        nnm_stats st;
        nnm_dropin::check(nnm_merge_nndescent(egraph, (uint32_t)f, preSize, &st));
        nCmps += st.ncmps;
        return 0;
    }
    // The local join of one iteration runs inside nnDescent() (the only
    // place the reference calls it, abstractmerge.cpp:168); called on its
    // own there are no sample lists to join and it returns 0.
    virtual unsigned localJoin() = 0;
    void setdisfunc(SpaceInterface<float> *func) override = 0;
    // AbstractMerge::EvaluateDelta (abstractmerge.cpp:194-202): the share
    // of new entries among the first K of a pool.
    float EvaluateDelta(Neighbors &pool, unsigned K) {
        unsigned c = 0, N = K;
        if (pool.size() < N) N = (unsigned)pool.size();
        for (unsigned i = 0; i < N; ++i)
            if (pool[i].flag) ++c;
        return float(c) / K;
    }
    // AbstractMerge::InitSGraph (abstractmerge.cpp:55-76): rows [b_idx,
    // b_idx + size_data) take `graph` (local ids) with group id Gid.
    void InitSGraph(const unsigned b_idx, unsigned *graph, unsigned Gid, unsigned size_data) {
        nnm_dropin::check(nnm_merge_init_sgraph(egraph, b_idx, graph, Gid, size_data));
    }
    // KGraph::buildKGraph on rows [b_idx, l_idx) inside this merge (the
    // reference builds a KGraph on cutMat(mata, b_idx, l_idx)): the same
    // graph, with the merge's std::rand() stream continuing through it as
    // the reference's process-wide stream does.  Returns new unsigned[]
    // of local ids, as KGraph::buildKGraph.
    unsigned *subGraph(const unsigned b_idx, const unsigned l_idx) {
        unsigned *g = new unsigned[(size_t)(l_idx - b_idx) * K0];
        uint64_t c = 0;
        nnm_dropin::check(nnm_merge_subgraph(egraph, b_idx, l_idx, g, &c));
        nCmps += c;
        return g;
    }
    // AbstractMerge::merge2one (abstractmerge.cpp:232-277)
    unsigned merge2one(const unsigned sz) {
        nnm_dropin::check(nnm_merge_merge2one(egraph, sz));
        return 1;
    }
    // AbstractMerge::cutMat (abstractmerge.cpp:37-53): rows [b_idx, l_idx)
    // copied into new float[].
    float *cutMat(float *mata, const unsigned b_idx, const unsigned l_idx) {
        const size_t n = (size_t)(l_idx - b_idx) * col;
        float *c = new float[n];
        std::memcpy(c, mata + (size_t)b_idx * col, n * sizeof(float));
        return c;
    }
    // The pools as Neighbors (the reference's egraph->knnGraph[i].pool).
    Neighbors pool(const unsigned i) {
        std::vector<uint32_t> ids((size_t)row * K0);
        std::vector<float> ds((size_t)row * K0);
        std::vector<uint8_t> fl((size_t)row * K0);
        nnm_dropin::check(nnm_merge_read(egraph, ids.data(), ds.data(), fl.data()));
        Neighbors p(K0);
        for (unsigned j = 0; j < K0; j++) {
            p[j].id = ids[(size_t)i * K0 + j];
            p[j].dist = ds[(size_t)i * K0 + j];
            p[j].flag = fl[(size_t)i * K0 + j] != 0;
        }
        return p;
    }
};

// Smerge (smerge.h:8-23): Smerge::buildKGraph (smerge.cpp:46-91) step by step.
class Smerge : public AbstractMerge {
protected:
    int join_filter() const override { return NNM_MERGE_SMERGE; }

public:
    Smerge() {}
    explicit Smerge(SpaceInterface<float> *func) : AbstractMerge(func) {}
    unsigned *buildKGraph(float *mata, const unsigned K, const unsigned N, const unsigned D) override {
        std::cout << "1. Two Sub graphs are prepared..................k = " << K << std::endl;
        InitialMemory(mata, K, N, D);
        preSize = row * 5 / 10;
        unsigned *one = subGraph(0, preSize);
        unsigned *two = subGraph(preSize, row);
        nCmps = 0;
        std::cout << "2. Symmetric Merge process.....................:" << std::endl;
        auto t0 = std::chrono::steady_clock::now();
        InitSGraph(0, one, 0, preSize);
        InitSGraph(preSize, two, 1, row - preSize);
        delete[] one;
        delete[] two;
        InitialGraph();
        nnDescent();
        merge2one(row);
        std::cout << "Merge time .....................................times = "
                  << std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() << std::endl;
        std::cout << "Merge-Scanning rate:............................rate  = "
                  << nCmps / ((row / 2.0) * (row - 1.0)) << std::endl;
        return 0;
    }
    // Smerge::InitialGraph (smerge.cpp:94-209): cross samples of the other half.
    unsigned InitialGraph() override {
        nnm_dropin::check(nnm_merge_initial_graph(egraph, NNM_MERGE_SMERGE, preSize));
        nCmps += (unsigned long)row * (K0 * 1 / 2);
        return 1;
    }
    unsigned localJoin() override { return 0; }
    void setdisfunc(SpaceInterface<float> *func) override { metric = func->nnm_metric(); }
};

// Jmerge (jmerge.h:7-22): Jmerge::buildKGraph (jmerge.cpp:43-80) step by step.
class Jmerge : public AbstractMerge {
protected:
    int join_filter() const override { return NNM_MERGE_JMERGE; }

public:
    Jmerge() {}
    explicit Jmerge(SpaceInterface<float> *func) : AbstractMerge(func) {}
    unsigned *buildKGraph(float *mata, const unsigned K, const unsigned N, const unsigned D) override {
        std::cout << "1. One Sub graph are prepared...................k = " << K << std::endl;
        InitialMemory(mata, K, N, D);
        preSize = row * 5 / 10;
        unsigned *one = subGraph(0, preSize);
        std::cout << "2. Joint Merge process.........................:" << std::endl;
        nCmps = 0;
        auto t0 = std::chrono::steady_clock::now();
        InitSGraph(0, one, 0, preSize);
        delete[] one;
        InitialGraph();
        nnDescent();
        merge2one(preSize);
        std::cout << "Merge time .....................................times = "
                  << std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() << std::endl;
        std::cout << "Merge-Scanning rate:............................rate  = "
                  << nCmps / ((row / 2.0) * (row - 1.0)) << std::endl;
        return 0;
    }
    // Jmerge::InitialGraph (jmerge.cpp:83-176): cross samples of the raw
    // rows for the built ones, random pools for the raw ones.
    unsigned InitialGraph() override {
        nnm_dropin::check(nnm_merge_initial_graph(egraph, NNM_MERGE_JMERGE, preSize));
        nCmps += (unsigned long)preSize * (K0 * 3 / 6) + (unsigned long)(row - preSize) * K0;
        return 1;
    }
    unsigned localJoin() override { return 0; }
    void setdisfunc(SpaceInterface<float> *func) override { metric = func->nnm_metric(); }
};

class LyNNDescent {
protected:
    int metric = NNM_METRIC_L2;
    unsigned row = 0, col = 0;
    float *mat = nullptr;
    unsigned long nCmps = 0;

public:
    LyNNDescent() {}
    explicit LyNNDescent(SpaceInterface<float> *func) : metric(func->nnm_metric()) {}
    virtual ~LyNNDescent() { delete[] mat; }
    // Writes <dstFn>.txt (the layers, lynndescent.cpp:625-638) and
    // <dstFn>_baselayer.txt (the k-NN graph, :847-872).
    unsigned buildhgraph(const char *srcFn, const char *dstFn, const char *grd, const unsigned topk, const unsigned M) {
        (void)grd;
        mat = nnm_dropin::load_refSet(srcFn, col, row);
        std::cout << "Matrix size .............................. " << row << "x" << col << std::endl;
        nnm_opts o = nnm_dropin::opts(metric);
        nnm_stats st;
        nnm_layers lay;
        std::vector<uint32_t> ids((size_t)row * topk);
        auto t0 = std::chrono::steady_clock::now();
        nnm_dropin::check(nnm_hmerge_build(nnm_dropin::context(), mat, row, col, topk, M, &o, ids.data(), nullptr,
                                           nullptr, &lay, &st));
        std::cout << "Construction time ........................ times = "
                  << std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() << std::endl;
        nCmps = st.ncmps;
        std::ofstream out(std::string(dstFn) + ".txt");
        for (uint32_t g = 0; g < lay.nlayers; g++) {
            out << lay.nrows[g] << std::endl;
            for (uint32_t i = 0; i < lay.nrows[g]; i++) {
                out << i << " " << (lay.off[g][i + 1] - lay.off[g][i]) << " ";
                for (uint64_t t = lay.off[g][i]; t < lay.off[g][i + 1]; t++) out << lay.adj[g][t] << " ";
                out << std::endl;
            }
        }
        nnm_layers_free(&lay);
        std::ofstream base(std::string(dstFn) + "_baselayer.txt");
        base << row << " " << topk << std::endl;
        for (unsigned i = 0; i < row; i++) {
            base << i << " " << topk;
            for (unsigned j = 0; j < topk; j++) base << " " << ids[(size_t)i * topk + j];
            base << std::endl;
        }
        return 0;
    }
};

class LySearch {
protected:
    int metric = NNM_METRIC_L2;
    unsigned row = 0, col = 0;
    float *mat = nullptr;
    nnm_layers layers{};
    std::vector<std::vector<uint64_t>> off_;
    std::vector<std::vector<uint32_t>> adj_;

    // LySearch::loadGraphs (lysearch.cpp:112-186): consecutive layers of
    // "rows" followed by "i n ids..." lines.
    void loadGraphs(const char *fn) {
        std::ifstream in(fn);
        if (!in) {
            std::cout << "Open file '" << fn << "' failed!" << std::endl;
            std::exit(0);
        }
        unsigned rows;
        while (layers.nlayers < 16 && (in >> rows)) {
            std::vector<uint64_t> off(rows + 1, 0);
            std::vector<uint32_t> adj;
            for (unsigned i = 0; i < rows; i++) {
                unsigned idx, num, v;
                in >> idx >> num;
                for (unsigned j = 0; j < num; j++) {
                    in >> v;
                    adj.push_back(v);
                }
                off[i + 1] = off[i] + num;
            }
            off_.push_back(std::move(off));
            adj_.push_back(std::move(adj));
            layers.nrows[layers.nlayers++] = rows;
        }
        for (uint32_t g = 0; g < layers.nlayers; g++) {
            layers.off[g] = off_[g].data();
            layers.adj[g] = adj_[g].data();
        }
    }

    nnm_index *ix_ = nullptr;

    // The data set and hierarchy go to the device once (nnm_index_create);
    // the clock value seeds the entry point, as knnSearch's rand() does.
    nnm_index *index() {
        if (!ix_) {
            nnm_opts o = nnm_dropin::opts(metric);
            nnm_dropin::check(nnm_index_create(nnm_dropin::context(), mat, row, col, &layers, o.seed, o.metric, &ix_));
        }
        return ix_;
    }

    // The sweep both searches share (lysearch.cpp:380-436, :530-561): beam
    // widths 60 .. 2; "query id dist" of each query's nearest result to
    // dstFn, "beam recall time distances/query" lines to record; recall@1
    // against grdFn ("query id" pairs) when it can be read.
    int sweep(const char *qryFn, const char *dstFn, const char *grdFn, const char *record, uint32_t entry) {
        unsigned qd = 0, nq = 0;
        float *q = nnm_dropin::load_refSet(qryFn, qd, nq);
        if (qd != col) {
            std::cout << "query dimension " << qd << " != " << col << std::endl;
            std::exit(0);
        }
        std::map<unsigned, unsigned> grd;
        {
            std::ifstream g(grdFn);
            unsigned a, b;
            while (g >> a >> b) grd[a] = b;
        }
        std::ofstream rec(record);
        static const unsigned beams[17] = {60, 50, 40, 36, 32, 28, 24, 20, 18, 15, 14, 12, 10, 8, 6, 4, 2};
        for (unsigned t = 0; t < 17; t++) {
            const unsigned topk = beams[t];
            std::vector<uint32_t> ids((size_t)nq * topk);
            std::vector<float> ds((size_t)nq * topk);
            nnm_search_stats st;
            auto t0 = std::chrono::steady_clock::now();
            nnm_dropin::check(nnm_index_search(index(), q, nq, nullptr, topk, topk, NNM_SERVE_EXACT, entry,
                                               ids.data(), ds.data(), &st));
            double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
            std::ofstream out(dstFn);
            unsigned hits = 0;
            for (unsigned i = 0; i < nq; i++) {
                out << i << "\t" << ids[(size_t)i * topk] << "\t" << ds[(size_t)i * topk] << std::endl;
                auto it = grd.find(i);
                if (it != grd.end() && it->second == ids[(size_t)i * topk]) hits++;
            }
            float r = grd.empty() ? 0.f : (float)hits / (float)grd.size();
            const uint64_t per_q = nq ? st.ncmps / nq : 0;
            std::cout << "Top-1 : " << r << "\t" << per_q << "\t" << secs << std::endl;
            rec << topk << "\t" << r << "\t" << secs << "\t" << per_q << std::endl;
            if (r == 1) break;
        }
        delete[] q;
        return 0;
    }

public:
    LySearch(const char *Rsrc, const char *Gsrc, SpaceInterface<float> *func) : metric(func->nnm_metric()) {
        mat = nnm_dropin::load_refSet(Rsrc, col, row);
        loadGraphs(Gsrc);
    }
    virtual ~LySearch() {
        if (ix_) nnm_index_free(ix_);
        delete[] mat;
    }
    // knnSearch (lysearch.cpp:363-437): one global entry, greedy descent
    // through the upper layers, best-first beam on the last.
    int knnSearch(const char *qryFn, const char *dstFn, const char *grdFn, const char *record) {
        return sweep(qryFn, dstFn, grdFn, record, NNM_ENTRY_DEFAULT);
    }
    // singleknnSearch (lysearch.cpp:522-561) with nndFlatSrch (:439-520):
    // the beam starts from `beam` random rows of the last layer.
    int singleknnSearch(const char *qryFn, const char *dstFn, const char *grdFn, const char *record) {
        return sweep(qryFn, dstFn, grdFn, record, NNM_ENTRY_FLAT);
    }
};

#endif  // NNM_DROPIN_HPP
