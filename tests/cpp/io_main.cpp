// The drop-in's file readers and writers on their own (no device work):
//   io_main vecs <in.fvecs|.bvecs|.txt> <out.mat>   load_refSet -> u32 n, u32 d, n*d f32
//   io_main knn <in (text or binary)> <out>         load_knn -> saved as text, or binary
//                                                   when out ends in .knng
#include <cstdio>
#include <cstring>
#include <iostream>
#include <vector>

#include "nnm_dropin.hpp"

int main(int argc, char **argv) {
    if (argc == 4 && !std::strcmp(argv[1], "vecs")) {
        unsigned d = 0, n = 0;
        float *m = nnm_dropin::load_refSet(argv[2], d, n);
        FILE *f = std::fopen(argv[3], "wb");
        std::fwrite(&n, 4, 1, f);
        std::fwrite(&d, 4, 1, f);
        std::fwrite(m, 4, (size_t)n * d, f);
        std::fclose(f);
        delete[] m;
        return 0;
    }
    if (argc == 4 && !std::strcmp(argv[1], "knn")) {
        unsigned n = 0, k = 0;
        unsigned *g = nnm_dropin::load_knn(argv[2], n, k);
        std::vector<uint32_t> ids(g, g + (size_t)n * k);
        delete[] g;
        if (nnm_dropin::ends_with(argv[3], ".knng")) nnm_dropin::save_knn_bin(argv[3], ids, n, k);
        else nnm_dropin::save_knn(argv[3], ids, n, k);
        return 0;
    }
    std::cerr << "usage: io_main vecs <in> <out.mat> | knn <in> <out>\n";
    return 2;
}
