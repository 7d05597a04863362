// Shared device-side definitions for the nn-merge B200 kernels.
//
// HBM layout (all row-major, SoA):
//   vectors  : n x dp float32, dp = d rounded up to a multiple of 4 (zero
//              padded; a zero tail adds exact zeros to every metric, so the
//              sequential sums below are unchanged), 16-byte aligned rows.
//   pools    : n x K packed u32 ids (bits 0..29 id, bit 30 group id "gd",
//              bit 31 "new" flag) + n x K float32 distances, each row sorted
//              as the reference keeps it (pvetex.h:18-30, kgraph.h:24-36).
//   sample lists: fixed-capacity rows of packed u32 (bit 31 = group id).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace nnm {

constexpr uint32_t ID_MASK = 0x3fffffffu;
constexpr uint32_t GD_BIT = 1u << 30;
constexpr uint32_t FLAG_BIT = 1u << 31;
constexpr uint32_t LGID_BIT = 1u << 31;   // group id bit of a sample-list entry
constexpr uint32_t LID_MASK = 0x7fffffffu;
constexpr int MAXK = 32;                  // pool size limit (one warp lane per entry)

enum Metric : int { L2 = 0, L1 = 1, CHI2 = 2 };

// One term of the reference distances, rounded exactly as the reference's
// scalar float code rounds it (no FMA contraction):
//   L2   VMath::l2norm   (vmath.cpp:56-88)   res += (a-b)*(a-b)
//   L1   DistOpt::l1norm (distopt.cpp:82-114) res += |a-b|
//   CHI2 DistOpt::KSquare (distopt.cpp:165-184) res += (a-b)^2/(a+b) unless a==b==0
template <int M>
__device__ __forceinline__ float dist_step(float acc, float a, float b) {
    float diff = __fsub_rn(a, b);
    if (M == L2) return __fadd_rn(acc, __fmul_rn(diff, diff));
    if (M == L1) return __fadd_rn(acc, fabsf(diff));
    if (a != 0.f || b != 0.f) return __fadd_rn(acc, __fdiv_rn(__fmul_rn(diff, diff), __fadd_rn(a, b)));
    return acc;
}

// Exact sequential distance between two rows (one thread).
template <int M>
__device__ __forceinline__ float dist_seq(const float* __restrict__ a, const float* __restrict__ b, int dp) {
    float acc = 0.f;
    for (int t = 0; t < dp; t += 4) {
        float4 va = *reinterpret_cast<const float4*>(a + t);
        float4 vb = *reinterpret_cast<const float4*>(b + t);
        acc = dist_step<M>(acc, va.x, vb.x);
        acc = dist_step<M>(acc, va.y, vb.y);
        acc = dist_step<M>(acc, va.z, vb.z);
        acc = dist_step<M>(acc, va.w, vb.w);
    }
    return acc;
}

__device__ __forceinline__ float dist_seq_rt(int metric, const float* a, const float* b, int dp) {
    if (metric == L2) return dist_seq<L2>(a, b, dp);
    if (metric == L1) return dist_seq<L1>(a, b, dp);
    return dist_seq<CHI2>(a, b, dp);
}

// ---------------------------------------------------------------------
// Device port of libstdc++'s std::sort as the reference calls it on a pool
// (kgraph.cpp:90, smerge.cpp:150 ...): comparator "a.dist < b.dist",
// introsort (median-of-three pivot, heapsort past 2*floor(log2 n) levels)
// followed by insertion sort with threshold 16.  The sort is not stable, so
// equal distances end up in the order these exact steps produce.  Runs on
// one thread over a small array.
struct SortEnt {
    float dist;
    uint32_t id;  // packed pool word
};

__device__ __forceinline__ bool sless(const SortEnt& a, const SortEnt& b) { return a.dist < b.dist; }
__device__ __forceinline__ void sswap(SortEnt* a, SortEnt* b) { SortEnt t = *a; *a = *b; *b = t; }

__device__ inline void s_heap_push(SortEnt* f, int hole, int top, SortEnt v) {
    int parent = (hole - 1) / 2;
    while (hole > top && sless(f[parent], v)) {
        f[hole] = f[parent];
        hole = parent;
        parent = (hole - 1) / 2;
    }
    f[hole] = v;
}
__device__ inline void s_heap_adjust(SortEnt* f, int hole, int len, SortEnt v) {
    int top = hole, second = hole;
    while (second < (len - 1) / 2) {
        second = 2 * (second + 1);
        if (sless(f[second], f[second - 1])) second--;
        f[hole] = f[second];
        hole = second;
    }
    if ((len & 1) == 0 && second == (len - 2) / 2) {
        second = 2 * (second + 1);
        f[hole] = f[second - 1];
        hole = second - 1;
    }
    s_heap_push(f, hole, top, v);
}
__device__ inline void s_heapsort(SortEnt* first, SortEnt* last) {
    int len = (int)(last - first);
    if (len >= 2)
        for (int parent = (len - 2) / 2;; parent--) {
            s_heap_adjust(first, parent, len, first[parent]);
            if (parent == 0) break;
        }
    while (last - first > 1) {
        --last;
        SortEnt v = *last;
        *last = *first;
        s_heap_adjust(first, 0, (int)(last - first), v);
    }
}
__device__ inline void s_median_to_first(SortEnt* r, SortEnt* a, SortEnt* b, SortEnt* c) {
    if (sless(*a, *b)) {
        if (sless(*b, *c)) sswap(r, b);
        else if (sless(*a, *c)) sswap(r, c);
        else sswap(r, a);
    } else if (sless(*a, *c)) sswap(r, a);
    else if (sless(*b, *c)) sswap(r, c);
    else sswap(r, b);
}
__device__ inline SortEnt* s_partition(SortEnt* first, SortEnt* last, SortEnt* pivot) {
    for (;;) {
        while (sless(*first, *pivot)) ++first;
        --last;
        while (sless(*pivot, *last)) --last;
        if (!(first < last)) return first;
        sswap(first, last);
        ++first;
    }
}
__device__ inline void s_linear_insert(SortEnt* last) {
    SortEnt v = *last;
    SortEnt* next = last - 1;
    while (sless(v, *next)) {
        *last = *next;
        last = next;
        --next;
    }
    *last = v;
}
__device__ inline void s_insertion(SortEnt* first, SortEnt* last) {
    if (first == last) return;
    for (SortEnt* i = first + 1; i != last; ++i) {
        if (sless(*i, *first)) {
            SortEnt v = *i;
            for (SortEnt* p = i; p != first; --p) *p = *(p - 1);
            *first = v;
        } else {
            s_linear_insert(i);
        }
    }
}
// Introsort loop without recursion: the right part is pushed on a small
// explicit stack, which visits ranges in the same order as the recursive
// libstdc++ code (right part fully first, then the left part).
__device__ inline void std_sort_dev(SortEnt* first, int len) {
    if (len <= 0) return;
    SortEnt* last = first + len;
    int lg = 31 - __clz(len);
    struct Frame { SortEnt* f; SortEnt* l; int depth; int stage; };
    Frame st[40];
    int sp = 0;
    st[sp++] = Frame{first, last, 2 * lg, 0};
    while (sp > 0) {
        Frame& fr = st[sp - 1];
        if (fr.l - fr.f > 16) {
            if (fr.depth == 0) {
                s_heapsort(fr.f, fr.l);
                --sp;
                continue;
            }
            --fr.depth;
            SortEnt* mid = fr.f + (fr.l - fr.f) / 2;
            s_median_to_first(fr.f, fr.f + 1, mid, fr.l - 1);
            SortEnt* cut = s_partition(fr.f + 1, fr.l, fr.f);
            SortEnt* rl = fr.l;
            fr.l = cut;                          // this frame continues on [f, cut)
            st[sp++] = Frame{cut, rl, fr.depth, 0};  // recurse into [cut, l) first
        } else {
            --sp;
        }
    }
    if (len > 16) {
        s_insertion(first, first + 16);
        for (SortEnt* i = first + 16; i != last; ++i) s_linear_insert(i);
    } else {
        s_insertion(first, last);
    }
}

// getRndSds (abstractgraph.cpp:7-35): k distinct ids in [0, N) from k
// mt19937 draws (rng() % (N - k)), a sort, a strictly-increasing fix-up and
// one more draw for a rotation.  `draws` holds the k+1 raw generator outputs
// for this call (none when N == k).
__device__ inline void rnd_seeds_dev(const uint32_t* draws, uint32_t k, uint32_t N, uint32_t* addr) {
    if (N == k) {
        for (uint32_t i = 0; i < k; i++) addr[i] = i;
        return;
    }
    for (uint32_t i = 0; i < k; i++) addr[i] = draws[i] % (uint32_t)(N - k);
    for (uint32_t i = 1; i < k; i++) {  // insertion sort of unsigned values
        uint32_t v = addr[i];
        uint32_t j = i;
        while (j > 0 && addr[j - 1] > v) {
            addr[j] = addr[j - 1];
            --j;
        }
        addr[j] = v;
    }
    for (uint32_t i = 1; i < k; i++)
        if (addr[i] <= addr[i - 1]) addr[i] = addr[i - 1] + 1;
    uint32_t off = draws[k] % N;
    for (uint32_t i = 0; i < k; i++) addr[i] = (addr[i] + off) % N;
}

__device__ __forceinline__ uint32_t warp_prefix_count(unsigned mask_bits, int lane) {
    return __popc(mask_bits & ((1u << lane) - 1u));
}

}  // namespace nnm

namespace nnm {
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as
// easy as 1, 2, 3", SC'11): a counter-based generator, so every (row, phase,
// draw) pair gets its own independent value with no shared state.  Used by
// the fast tier in place of the reference's sequential streams.
struct Philox {
    uint32_t k0, k1;
    __device__ __forceinline__ uint4 operator()(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3) const {
        uint32_t a0 = k0, a1 = k1;
        uint4 c = make_uint4(c0, c1, c2, c3);
#pragma unroll
        for (int r = 0; r < 10; r++) {
            const uint32_t hi0 = __umulhi(0xD2511F53u, c.x), lo0 = 0xD2511F53u * c.x;
            const uint32_t hi1 = __umulhi(0xCD9E8D57u, c.z), lo1 = 0xCD9E8D57u * c.z;
            c = make_uint4(hi1 ^ c.y ^ a0, lo1, hi0 ^ c.w ^ a1, lo0);
            a0 += 0x9E3779B9u;
            a1 += 0xBB67AE85u;
        }
        return c;
    }
};

// Uniform integer in [0, m) from a 32-bit draw (multiply-shift).
__device__ __forceinline__ uint32_t bounded(uint32_t r, uint32_t m) {
    return (uint32_t)(((unsigned long long)r * m) >> 32);
}
}  // namespace nnm
