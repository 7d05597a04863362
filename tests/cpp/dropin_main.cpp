// Reference-style caller of the drop-in classes (as smerge.cpp:238-261 and
// kgraph.cpp:263-285 call the reference's): builds a graph from an .fvecs
// file and saves it in the reference's text format.
//   dropin_main kgraph|smerge|jmerge <in.fvecs> <K> <out.txt>
//   dropin_main hmerge <in.fvecs> <K> <M> <out_prefix>
//   dropin_main search|flatsearch <in.fvecs> <hierarchy.txt> <queries.fvecs> <out.txt> <record.txt>
#include <cstdlib>
#include <cstring>
#include <iostream>

#include "nnm_dropin.hpp"

int main(int argc, char **argv) {
    L2space l2;
    if (argc == 6 && !std::strcmp(argv[1], "hmerge")) {
        LyNNDescent h(&l2);  // lynndescent.cpp:873-896
        h.buildhgraph(argv[2], argv[5], nullptr, (unsigned)std::atoi(argv[3]), (unsigned)std::atoi(argv[4]));
        return 0;
    }
    if (argc == 7 && (!std::strcmp(argv[1], "search") || !std::strcmp(argv[1], "flatsearch"))) {
        LySearch s(argv[2], argv[3], &l2);  // lysearch.cpp:600-640
        if (!std::strcmp(argv[1], "search")) s.knnSearch(argv[4], argv[5], "", argv[6]);
        else s.singleknnSearch(argv[4], argv[5], "", argv[6]);
        return 0;
    }
    if (argc != 5) {
        std::cerr << "usage: dropin_main kgraph|smerge|jmerge <in.fvecs> <K> <out.txt>\n";
        return 2;
    }
    unsigned d = 0, n = 0, k = (unsigned)std::atoi(argv[3]);
    float *mat = nnm_dropin::load_refSet(argv[2], d, n);
    AbstractGraph *g = nullptr;
    if (!std::strcmp(argv[1], "kgraph")) g = new KGraph(&l2);
    else if (!std::strcmp(argv[1], "smerge")) g = new Smerge(&l2);
    else g = new Jmerge(&l2);
    unsigned *ids = g->buildKGraph(mat, k, n, d);
    g->saveKGraph(argv[4]);
    delete[] ids;
    delete g;
    return 0;
}
