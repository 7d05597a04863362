/* Test infrastructure: a command-line driver around the UNMODIFIED
 * reference classes (compiled from the reference sources in place by
 * oracle/Makefile).  It is the ground truth that the C restatement in
 * oracle/nnm_oracle.c is checked against and that tests/golden/ fixtures are
 * generated from.  Nothing in the product links or runs it.
 *
 * Determinism: the reference seeds every phase with mt19937(time(NULL)); the
 * force-included nnm_refseed.h routes time() to nnm_refshim_time(), which
 * returns the seed given on the command line, and main() calls srand(seed)
 * once for the std::rand() stream behind std::random_shuffle.
 *
 * Binary formats (little endian):
 *   matrix in : u32 n, u32 d, n*d f32 (row-major)
 *   graph out : u32 n, u32 k, n*k u32 ids, n*k f32 dists, n*k u8 flags,
 *               u64 distance evaluations (nCmps),
 *               u32 t, t f32 (one convergence mean per NN-Descent iteration,
 *               in call order)
 *   search out: u32 nq, u32 topk, u32 entry point, u64 nCmps,
 *               nq*topk u32 ids, nq*topk f32 dists  (ascending)
 *   loadknn   : the reference's own reader of the k-NN graph text
 *               (IODelegator::loadKNNGraph) -> u32 n, u32 k, n*k u32 ids
 *   loadvecs  : the reference's own reader of .fvecs/.bvecs/.txt vectors
 *               (IODelegator::load_refSet) -> matrix format above
 */
#include "kgraph.h"
#include "smerge.h"
#include "jmerge.h"
#include "lynndescent.h"
#include "lysearch.h"
#include "space_lp.h"
#include "iodelegator.h"

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

static time_t g_seed = 0;
extern "C" time_t nnm_refshim_time(time_t *t) {
    if (t) *t = g_seed;
    return g_seed;
}
std::vector<float> &nnm_refshim_mean_trace() {
    static std::vector<float> trace;
    return trace;
}

namespace {

float *read_matrix(const char *path, unsigned &n, unsigned &d) {
    FILE *f = std::fopen(path, "rb");
    if (!f) { std::perror(path); std::exit(2); }
    uint32_t hdr[2];
    if (std::fread(hdr, 4, 2, f) != 2) { std::fprintf(stderr, "bad matrix\n"); std::exit(2); }
    n = hdr[0]; d = hdr[1];
    float *m = new float[(size_t)n * d];
    if (std::fread(m, 4, (size_t)n * d, f) != (size_t)n * d) { std::fprintf(stderr, "short matrix\n"); std::exit(2); }
    std::fclose(f);
    return m;
}

struct Pool { uint32_t id; float dist; uint8_t flag; };

void write_graph(const char *path, unsigned n, unsigned k, const std::vector<Pool> &pools,
                 unsigned long ncmps) {
    FILE *f = std::fopen(path, "wb");
    if (!f) { std::perror(path); std::exit(2); }
    uint32_t hdr[2] = {n, k};
    std::fwrite(hdr, 4, 2, f);
    for (auto &p : pools) std::fwrite(&p.id, 4, 1, f);
    for (auto &p : pools) std::fwrite(&p.dist, 4, 1, f);
    for (auto &p : pools) std::fwrite(&p.flag, 1, 1, f);
    uint64_t c = ncmps;
    std::fwrite(&c, 8, 1, f);
    auto &tr = nnm_refshim_mean_trace();
    uint32_t t = (uint32_t)tr.size();
    std::fwrite(&t, 4, 1, f);
    if (t) std::fwrite(tr.data(), 4, t, f);
    std::fclose(f);
}

SpaceInterface<float> *make_space(const char *name) {
    if (!std::strcmp(name, "l2")) return new L2space();
    if (!std::strcmp(name, "l1")) return new L1space();
    if (!std::strcmp(name, "chi2")) return new Ksquare();
    std::fprintf(stderr, "unknown metric %s\n", name);
    std::exit(2);
}

/* Probe subclasses: the reference keeps its neighbour pools in protected
 * members; these only read them. */
struct KGraphProbe : public kgraph::KGraph {
    explicit KGraphProbe(SpaceInterface<float> *s) : kgraph::KGraph(s) {}
    void dump(std::vector<Pool> &out) {
        for (auto &row : knnGraph)
            for (auto &nb : row.pool) out.push_back({nb.id, nb.dist, (uint8_t)nb.flag});
    }
};
template <class Base> struct MergeProbe : public Base {
    explicit MergeProbe(SpaceInterface<float> *s) : Base(s) {}
    void dump(std::vector<Pool> &out) {
        for (auto &row : this->egraph->knnGraph)
            for (auto &nb : row.pool) out.push_back({nb.id, nb.dist, (uint8_t)nb.flag});
    }
};
struct HMergeProbe : public LyNNDescent {
    explicit HMergeProbe(SpaceInterface<float> *s) : LyNNDescent(s) {}
    unsigned long cmps() const { return nCmps; }
    void dump(std::vector<Pool> &out) {
        for (auto &row : hgraph->knnGraph)
            for (auto &nb : row.pool) out.push_back({nb.id, nb.dist, (uint8_t)nb.flag});
    }
};
/* LySearch::knnSearch (lysearch.cpp:363-437) sweeps 17 beam widths and keeps
 * only the top-1 id of each query.  For parity at one beam width this probe
 * runs the same per-query steps -- one global entry point drawn with rand()
 * (lysearch.cpp:382), greedy 1-NN descent over layers 0..3
 * (lysearch.cpp:393-420), then the reference's own nndHNSWSrch on layer 4
 * (lysearch.cpp:421) -- and keeps all topk results. */
struct SearchProbe : public LySearch {
    SearchProbe(const char *r, const char *g, SpaceInterface<float> *s) : LySearch(r, g, s) {}
    void run(const float *q, unsigned nq, unsigned dim, unsigned topk, const char *outp) {
        flags = new unsigned short int[row];
        std::memset(flags, 0, sizeof(unsigned short int) * row);
        nCmps = 0;
        unsigned enter = rand() % layers[0].szGraph;
        std::vector<uint32_t> ids((size_t)nq * topk, 0xffffffffu);
        std::vector<float> ds((size_t)nq * topk, 0.f);
        std::vector<RTPair> res;
        for (unsigned i = 0; i < nq; i++) {
            crntQry = const_cast<float *>(q) + (size_t)i * dim;
            unsigned cur = enter;
            float cur_d = distfunc(crntQry, 0, mat, cur, col);
            ++nCmps;
            for (unsigned ir = 0; ir < 4; ir++) {
                crntAugKnnGraph = layers[ir].augKnnGraph;
                crntKnnLocs = layers[ir].knnLocs;
                bool moved = true;
                while (moved) {
                    unsigned loc = crntKnnLocs[cur];
                    unsigned deg = crntAugKnnGraph[loc];
                    moved = false;
                    for (unsigned l = 1; l <= deg; l++) {
                        unsigned nn = crntAugKnnGraph[loc + l];
                        float dd = distfunc(crntQry, 0, mat, nn, col);
                        ++nCmps;
                        if (dd < cur_d) { cur_d = dd; cur = nn; moved = true; }
                    }
                }
            }
            res.clear();
            nndHNSWSrch(cur, cur_d, 5, res, topk);
            for (size_t r = 0; r < res.size() && r < topk; r++) {
                ids[(size_t)i * topk + r] = res[r].id;
                ds[(size_t)i * topk + r] = res[r].dst;
            }
        }
        write(outp, nq, topk, enter, ids, ds);
    }
    /* LySearch::singleknnSearch's per-query step (lysearch.cpp:522-561): the
     * reference's own nndFlatSrch on the last layer, which seeds each query
     * with getRndSds(mt19937(time(NULL)), topk) (lysearch.cpp:455-460). */
    void run_flat(const float *q, unsigned nq, unsigned dim, unsigned topk, const char *outp) {
        flags = new unsigned short int[row];
        std::memset(flags, 0, sizeof(unsigned short int) * row);
        nCmps = 0;
        std::vector<uint32_t> ids((size_t)nq * topk, 0xffffffffu);
        std::vector<float> ds((size_t)nq * topk, 0.f);
        std::vector<RTPair> res;
        for (unsigned i = 0; i < nq; i++) {
            crntQry = const_cast<float *>(q) + (size_t)i * dim;
            res.clear();
            nndFlatSrch(5, res, topk);
            for (size_t r = 0; r < res.size() && r < topk; r++) {
                ids[(size_t)i * topk + r] = res[r].id;
                ds[(size_t)i * topk + r] = res[r].dst;
            }
        }
        write(outp, nq, topk, 0, ids, ds);
    }
    void write(const char *outp, unsigned nq, unsigned topk, unsigned enter, const std::vector<uint32_t> &ids,
               const std::vector<float> &ds) {
        FILE *f = std::fopen(outp, "wb");
        uint32_t hdr[3] = {nq, topk, enter};
        std::fwrite(hdr, 4, 3, f);
        uint64_t c = nCmps;
        std::fwrite(&c, 8, 1, f);
        std::fwrite(ids.data(), 4, ids.size(), f);
        std::fwrite(ds.data(), 4, ds.size(), f);
        std::fclose(f);
    }
};

void write_fvecs(const std::string &path, const float *m, unsigned n, unsigned d) {
    FILE *f = std::fopen(path.c_str(), "wb");
    for (unsigned i = 0; i < n; i++) {
        std::fwrite(&d, 4, 1, f);
        std::fwrite(m + (size_t)i * d, 4, d, f);
    }
    std::fclose(f);
}

int usage() {
    std::fprintf(stderr,
        "usage: nnm_ref kgraph|smerge|jmerge <metric> <in.mat> <K> <seed> <out.graph>\n"
        "       nnm_ref hmerge <metric> <in.mat> <K> <M> <seed> <out.graph> <out_prefix>\n"
        "       nnm_ref search|flatsearch <metric> <in.mat> <layers.txt> <queries.mat> <topk> <seed> <out.res>\n"
        "       nnm_ref loadknn <graph.txt> <K> <out.ids>\n"
        "       nnm_ref loadvecs <in.fvecs|.bvecs|.txt> <out.mat>\n");
    return 2;
}

}  // namespace

int main(int argc, char **argv) {
    if (argc < 2) return usage();
    std::string cmd = argv[1];
    if (cmd == "kgraph" || cmd == "smerge" || cmd == "jmerge") {
        if (argc != 7) return usage();
        SpaceInterface<float> *space = make_space(argv[2]);
        unsigned n, d;
        float *m = read_matrix(argv[3], n, d);
        unsigned k = std::atoi(argv[4]);
        g_seed = (time_t)std::strtoll(argv[5], nullptr, 10);
        srand((unsigned)g_seed);
        std::vector<Pool> pools;
        unsigned long c = 0;
        if (cmd == "kgraph") {
            auto *g = new KGraphProbe(space);
            g->buildKGraph(m, k, n, d);
            g->dump(pools);
            c = g->nCmps;
        } else if (cmd == "smerge") {
            auto *g = new MergeProbe<Smerge>(space);
            g->buildKGraph(m, k, n, d);
            g->dump(pools);
            c = g->nCmps;
        } else {
            auto *g = new MergeProbe<Jmerge>(space);
            g->buildKGraph(m, k, n, d);
            g->dump(pools);
            c = g->nCmps;
        }
        write_graph(argv[6], n, k, pools, c);
        return 0;
    }
    if (cmd == "hmerge") {
        if (argc != 9) return usage();
        SpaceInterface<float> *space = make_space(argv[2]);
        unsigned n, d;
        float *m = read_matrix(argv[3], n, d);
        unsigned k = std::atoi(argv[4]);
        unsigned mm = std::atoi(argv[5]);
        g_seed = (time_t)std::strtoll(argv[6], nullptr, 10);
        srand((unsigned)g_seed);
        std::string prefix = argv[8];
        std::string src = prefix + "_input.fvecs";
        std::string grd = prefix + "_nogt.txt";
        write_fvecs(src, m, n, d);
        delete[] m;
        { std::ofstream g(grd); g << "0 0\n"; }
        auto *h = new HMergeProbe(space);
        h->buildhgraph(src.c_str(), prefix.c_str(), grd.c_str(), k, mm);
        std::vector<Pool> pools;
        h->dump(pools);
        write_graph(argv[7], n, k, pools, h->cmps());
        std::remove(src.c_str());
        std::remove(grd.c_str());
        return 0;
    }
    if (cmd == "loadknn") {
        if (argc != 5) return usage();
        unsigned n = 0, k = 0;
        unsigned *g = IODelegator::loadKNNGraph(argv[2], n, k, (unsigned)std::atoi(argv[3]));
        FILE *f = std::fopen(argv[4], "wb");
        std::fwrite(&n, 4, 1, f);
        std::fwrite(&k, 4, 1, f);
        std::fwrite(g, 4, (size_t)n * k, f);
        std::fclose(f);
        std::free(g);
        return 0;
    }
    if (cmd == "loadvecs") {
        if (argc != 4) return usage();
        unsigned n = 0, d = 0;
        float *m = IODelegator::load_refSet(argv[2], d, n);
        FILE *f = std::fopen(argv[3], "wb");
        std::fwrite(&n, 4, 1, f);
        std::fwrite(&d, 4, 1, f);
        std::fwrite(m, 4, (size_t)n * d, f);
        std::fclose(f);
        delete[] m;
        return 0;
    }
    if (cmd == "search" || cmd == "flatsearch") {
        if (argc != 9) return usage();
        SpaceInterface<float> *space = make_space(argv[2]);
        unsigned n, d, nq, qd;
        float *m = read_matrix(argv[3], n, d);
        std::string src = std::string(argv[8]) + "_base.fvecs";
        write_fvecs(src, m, n, d);
        delete[] m;
        float *q = read_matrix(argv[5], nq, qd);
        unsigned topk = std::atoi(argv[6]);
        g_seed = (time_t)std::strtoll(argv[7], nullptr, 10);
        srand((unsigned)g_seed);
        auto *s = new SearchProbe(src.c_str(), argv[4], space);
        if (cmd == "search") s->run(q, nq, qd, topk, argv[8]);
        else s->run_flat(q, nq, qd, topk, argv[8]);
        std::remove(src.c_str());
        return 0;
    }
    return usage();
}
