// Local-join definitions shared by the FP32 pair kernels (nndescent.cu) and
// the tensor-core join (join_tc.cu).
#pragma once
#include <cstdint>

#include "nnm_nnd.h"

namespace nnm {

// Joined rows are binned by list size S = |new| + |old| into tiers: S <= 16,
// 32, 64, 128 and the rest.  The FP32 kernels stage a tier's vectors in
// shared memory sized for it (the last tier reads from L2); the tensor-core
// join packs 8, 4, 2 or 1 rows of the first four tiers into one 128-slot tile.
constexpr int NTIER = 5;
constexpr uint32_t TIER_CAP[4] = {16, 32, 64, 128};
constexpr int TIER_THREADS[NTIER] = {64, 64, 64, 128, 128};
constexpr uint32_t TC_MAX_S = 128;  // rows the tensor-core join takes

__host__ __device__ __forceinline__ int tier_of(uint32_t S) {
    return S <= 16 ? 0 : S <= 32 ? 1 : S <= 64 ? 2 : S <= 128 ? 3 : 4;  // TIER_CAP
}

struct JoinArgs {
    const float* x;
    uint32_t dp, K, n;
    const float* pdist;
    const uint32_t *newL, *oldL, *newlen, *oldlen;
    uint32_t capn, capo, caps;
    uint32_t mode, verse;
    const uint32_t* leaf_off;
    uint32_t nleaf;
    const uint32_t* tier_rows;  // NTIER lists of n rows
    const uint64_t* poff;       // first pair slot of each row
    float* pd;                  // pair distances
    uint16_t* cntpos;
    uint32_t *bcnt, *bcur;
    const uint64_t* boff;
    void* bucket;               // Prop (exact tier) or Prop8 (fast tier) entries
    IterCounters* ctr;
    // tensor-core join: the operand copy of the vectors (kq bytes a row,
    // zero padded; u8 or BF16 by tc_kind) and their squared norms (u32
    // integers for u8, float bits for BF16); tc != 0 when it takes tiers 0-3
    const uint8_t* xq;
    const uint32_t* nrm;
    uint32_t kq, tc;
    unsigned* tc_err;
    uint32_t* emit_rows;  // 4 lists of n rows: rows of tiers 0-3 that have proposals
    uint32_t fast_key;    // tie-break keys from ids instead of list positions (fast tier)
    uint32_t tc_kind;     // 0: u8 (exact), 1: BF16 hi + lo, 2: FP8 hi + mid + lo (join_tc.cu)
    float err_c;          // reduced precision: |d~ - reference distance| <= err_c * (|a|^2 + |b|^2)
    const float* scl;     // FP8: per-row inverse scales
    uint32_t audit;       // reduced precision: check every pair's d~ against its exact distance
    const float* kthv;    // every row's K-th distance at the iteration's start (compact copy of pdist's)
};

// Tie-break key of the exact tier's proposal "target gets the other entry"
// from the join of `row`: the reference's sequential insert order (the
// row, the pair's index in join order, then the side: 0 = into the outer
// element's pool).  The fast tier's key (fast_key, nnm_nnd.h) is the other
// entry's id and group bit alone, so that the graphs do not depend on the
// order of the sample lists nor on which row proposed a pair: copies of a
// proposal are equal in (distance, key) and the merge keeps one; when a
// row's lists hold an id twice with different group bits, the copies order
// by the group bit rather than by their arrival in the bucket.
__device__ __forceinline__ unsigned long long prop_key(uint32_t row, uint32_t pair_idx, uint32_t side) {
    return (1ull << 63) | ((unsigned long long)row << 32) | ((unsigned long long)pair_idx << 1) | side;
}

// Writes proposal number `slot` of the bucket array in the tier's format.
template <bool FAST>
__device__ __forceinline__ void put_prop(void* bucket, unsigned long long slot, float dist, uint32_t idg,
                                         uint32_t row, uint32_t pair_idx, uint32_t side) {
    if (FAST)
        reinterpret_cast<uint2*>(bucket)[slot] = make_uint2(__float_as_uint(dist), idg);
    else
        reinterpret_cast<Prop*>(bucket)[slot] = Prop{dist, idg, prop_key(row, pair_idx, side)};
}

__device__ __forceinline__ uint32_t leaf_of(uint32_t id, const uint32_t* off, uint32_t nleaf) {
    uint32_t lo = 0, hi = nleaf;  // off[0] = 0 <= id < off[nleaf]
    while (hi - lo > 1) {
        uint32_t mid = (lo + hi) >> 1;
        if (id >= off[mid]) lo = mid;
        else hi = mid;
    }
    return lo;
}

// Slot of pair (a, b), a < b, a in the new list: row-major over the upper
// triangle of new x new, then new x old.
__device__ __forceinline__ uint32_t pair_slot(uint32_t a, uint32_t b, uint32_t nn, uint32_t no) {
    return b < nn ? a * nn - a * (a + 1) / 2 + (b - a - 1) : nn * (nn - 1) / 2 + a * no + (b - nn);
}

// The reference's join filter and visiting order for pair (a, b), a < b:
// returns false if the pair is skipped, else the outer (first-inserted
// target) and inner positions.
__device__ __forceinline__ bool pair_order(uint32_t mode, uint32_t verse, uint32_t av, uint32_t bv, uint32_t nn,
                                           uint32_t ea, uint32_t eb, uint32_t ga, uint32_t gb, uint32_t& outer,
                                           uint32_t& inner) {
    const uint32_t ida = ea & LID_MASK, idb = eb & LID_MASK;
    if (ida == idb) return false;
    outer = av;
    inner = bv;
    if (mode == MODE_KGRAPH) {
        if (bv < nn && idb < ida) {  // kgraph.h:112-116 visits it from the smaller id
            outer = bv;
            inner = av;
        }
        return true;
    }
    if (mode == MODE_SMERGE) return ga != gb;
    return ga != gb || ga == 1 || gb == 1 || verse;
}

// Tensor-core join (join_tc.cu).
struct Ctx;
struct GraphStore;
struct GraphDev;
// Decides whether the tensor-core join applies to g's vectors (L2 metric,
// every component an integer in [0, 255], every distance below 2^24) and,
// if so, builds the u8 copy and the norms.  Returns an engine status.
int tc_prepare(Ctx& ctx, GraphStore& s, GraphDev& g);
cudaError_t tc_set_attributes(uint32_t kq, uint32_t kind);
// pass 0: per-slot proposal counts; pass 1: proposals into the buckets.
// ntier: rows per tier as the host read them, or null (grid of every SM's
// CTAs, the kernel reads the counts on the device).
cudaError_t launch_join_tc(int pass, const JoinArgs& ja, const unsigned* ntier, int nsm, cudaStream_t st);
// Rows of the last tier (lists longer than a tile's) of the u8 join on the
// tensor cores, count pass: their stored pair distances, per-slot counts and
// bucket totals, as k_pairs_u8 computes them (k_emit_rows then writes the
// proposals).  R: the longest list (new + old caps); applies when
// pairs_tc_smem(R, kq) fits a CTA's shared memory.
size_t pairs_tc_smem(uint32_t R, uint32_t kq);
cudaError_t pairs_tc_set_attributes(uint32_t R, uint32_t kq);
cudaError_t launch_pairs_tc(const JoinArgs& ja, uint32_t R, const unsigned* ntier, int nsm, cudaStream_t st);

}  // namespace nnm
