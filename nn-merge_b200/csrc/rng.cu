// Reference-exact random streams.
//
// 1. std::rand() (glibc, the generator behind std::random_shuffle in
//    kgraph.cpp:139-162 and friends).  glibc's TYPE_3 generator is the
//    additive lagged-Fibonacci sequence
//        r[i] = r[i-31] + r[i-3]  (mod 2^32),   rand() #k = r[k+344] >> 1,
//    with r[0..30] from srand's Park-Miller fill and r[31..33] = r[0..2].
//    The recurrence is linear, so s[n] = r[34+n] equals sum_j c_j s[j] where
//    c = x^n mod P(x), P(x) = x^31 - x^28 - 1, coefficients mod 2^32.  Each
//    GPU thread jumps to its own chunk with a product of precomputed
//    x^(2^b) mod P and then runs the recurrence: the whole stream for an
//    NN-Descent iteration is produced in parallel, with no host work.
// 2. std::mt19937 draws for the initial graphs are generated on the host
//    (gen_mt19937) and copied to the device; their count per row is fixed.
#include <cstdint>
#include <cstring>
#include <random>
#include <vector>

#include "nnm_rng.h"
#include "nnm_launch.h"

namespace nnm {

namespace {
constexpr int DEG = 31;
constexpr int CHUNK = 2048;  // outputs generated by one thread

__constant__ uint32_t c_pow2[64][DEG];  // x^(2^b) mod P (independent of the seed)

// c = a * b mod P(x), all coefficients mod 2^32.
__device__ __forceinline__ void poly_mulmod(const uint32_t* a, const uint32_t* b, uint32_t* c) {
    uint32_t t[2 * DEG - 1];
#pragma unroll
    for (int i = 0; i < 2 * DEG - 1; i++) t[i] = 0;
#pragma unroll
    for (int i = 0; i < DEG; i++)
#pragma unroll
        for (int j = 0; j < DEG; j++) t[i + j] += a[i] * b[j];
#pragma unroll
    for (int i = 2 * DEG - 2; i >= DEG; i--) {  // x^31 = x^28 + 1
        t[i - 3] += t[i];
        t[i - DEG] += t[i];
    }
#pragma unroll
    for (int i = 0; i < DEG; i++) c[i] = t[i];
}

__global__ void k_glibc_stream(int32_t* __restrict__ out, GlibcBase base, uint64_t first_output,
                               const uint64_t* __restrict__ count_ptr, uint64_t count_cap) {
    uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    uint64_t count = count_ptr ? *count_ptr : count_cap;
    if (count > count_cap) count = count_cap;
    uint64_t k0 = g * CHUNK;
    if (k0 >= count) return;
    uint64_t n = first_output + k0 + 310;  // s-index of the first output of this chunk
    uint32_t c[DEG];
#pragma unroll
    for (int i = 0; i < DEG; i++) c[i] = (i == 0);
    for (int b = 0; b < 64; b++) {
        if ((n >> b) & 1ull) {
            uint32_t tmp[DEG];
            poly_mulmod(c, c_pow2[b], tmp);
#pragma unroll
            for (int i = 0; i < DEG; i++) c[i] = tmp[i];
        }
    }
    uint32_t w[DEG];
#pragma unroll
    for (int m = 0; m < DEG; m++) {
        uint32_t acc = 0;
#pragma unroll
        for (int j = 0; j < DEG; j++) acc += c[j] * base.s[j + m];
        w[m] = acc;
    }
    uint64_t end = k0 + CHUNK < count ? k0 + CHUNK : count;
    uint64_t pos = k0;
    while (pos < end) {
#pragma unroll
        for (int m = 0; m < DEG; m++)
            if (pos + m < end) out[pos + m] = (int32_t)(w[m] >> 1);
        pos += DEG;
#pragma unroll
        for (int m = 0; m < DEG; m++) w[m] = (m < 3 ? w[28 + m] : w[m - 3]) + w[m];
    }
}

void host_mulmod(const uint32_t* a, const uint32_t* b, uint32_t* c) {
    uint32_t t[2 * DEG - 1] = {0};
    for (int i = 0; i < DEG; i++)
        for (int j = 0; j < DEG; j++) t[i + j] += a[i] * b[j];
    for (int i = 2 * DEG - 2; i >= DEG; i--) {
        t[i - 3] += t[i];
        t[i - DEG] += t[i];
    }
    std::memcpy(c, t, sizeof(uint32_t) * DEG);
}
}  // namespace

GlibcBase glibc_base(uint32_t seed) {
    // r[0..30]: srandom_r's fill; r[31..33] = r[0..2]; s[n] = r[34+n].
    if (seed == 0) seed = 1;
    std::vector<uint32_t> r(34 + 2 * DEG);
    int32_t word = (int32_t)seed;
    r[0] = (uint32_t)word;
    for (int i = 1; i < 31; i++) {
        long hi = word / 127773, lo = word % 127773;
        word = (int32_t)(16807 * lo - 2836 * hi);
        if (word < 0) word += 2147483647;
        r[i] = (uint32_t)word;
    }
    for (int i = 31; i < 34; i++) r[i] = r[i - 31];
    for (size_t i = 34; i < r.size(); i++) r[i] = r[i - 3] + r[i - 31];
    GlibcBase b;
    for (int i = 0; i < 2 * DEG; i++) b.s[i] = r[34 + i];
    return b;
}

cudaError_t glibc_tables_init() {
    uint32_t pw[64][DEG];
    std::memset(pw, 0, sizeof(pw));
    pw[0][1] = 1;  // x
    for (int b = 1; b < 64; b++) host_mulmod(pw[b - 1], pw[b - 1], pw[b]);
    return cudaMemcpyToSymbol(c_pow2, pw, sizeof(pw));
}

cudaError_t glibc_stream_generate(int32_t* out, const GlibcBase& base, uint64_t first_output,
                                  const uint64_t* d_count, uint64_t count_cap, cudaStream_t st) {
    if (count_cap == 0) return cudaSuccess;
    uint64_t threads = (count_cap + CHUNK - 1) / CHUNK;
    unsigned blocks = (unsigned)((threads + 127) / 128);
    k_glibc_stream<<<blocks, 128, 0, st>>>(out, base, first_output, d_count, count_cap); count_launch();
    return cudaGetLastError();
}

void gen_mt19937(uint32_t seed, uint64_t count, uint32_t* out) {
    std::mt19937 g(seed);
    for (uint64_t i = 0; i < count; i++) out[i] = (uint32_t)g();
}

}  // namespace nnm
