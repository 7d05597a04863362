// NN-Descent iteration kernels and the device graph they operate on.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "nnm_common.cuh"
#include "nnm_rng.h"

namespace nnm {

// Join filters of the reference local joins.
enum JoinMode : uint32_t {
    MODE_KGRAPH = 0,  // KGraph::join (kgraph.cpp:191-210): all pairs, new x new by id order
    MODE_SMERGE = 1,  // Smerge::localJoin (smerge.cpp:212-235): groups differ
    MODE_JMERGE = 2,  // Jmerge::localJoin (jmerge.cpp:178-203): groups differ or either is 1
    MODE_LY = 3,      // LyNNDescent::localJoin (lynndescent.cpp:313-342): as J-Merge, or verse
};

// A proposal "insert id into target's pool with distance dist", ordered by
// (dist, key); key = 2^63 | row << 32 | pair index << 1 | side reproduces the
// reference's sequential insert order (row ascending, pairs in join order,
// first insert into the outer element's pool, then the inner's).  Exact tier.
struct __align__(16) Prop {
    float dist;
    uint32_t idg;  // id | group bit << 31
    unsigned long long key;
};

// The fast tier's proposal, 8 bytes: its tie-break key depends only on the
// proposed entry (fast_key below), so the bucket holds (dist, idg) and the
// merge derives the key -- half the bytes written by the join and read by
// the merge.
struct __align__(8) Prop8 {
    float dist;
    uint32_t idg;
};

// Bit 30 of a proposal's idg (ids stay below 2^30): its distance is the
// reduced-precision join's approximation d~, within err_c * (|t|^2 + |u|^2)
// of the exact FP32 distance; the merge computes the exact value of those
// proposals that can still reach the top K.
constexpr uint32_t APPROX_BIT = 1u << 30;

// Key of a fast-tier proposal of list entry `idg`: the entry's id, then its
// group bit with group 1 first; bit 63 set so that the start pool's entries
// (keys 0..K-1) precede every proposal of equal distance.
__host__ __device__ __forceinline__ unsigned long long fast_key(uint32_t idg) {
    return (1ull << 63) | ((unsigned long long)(idg & 0x3fffffffu) << 1) | ((idg >> 31) ^ 1u);
}

// Per-iteration statistics read back by the host.
struct IterCounters {
    unsigned long long flags;      // pool entries inserted this iteration
    unsigned long long ncmps;      // distance evaluations in the join
    unsigned long long proposals;  // bucketed proposals
    unsigned long long rand_draws; // std::rand() calls of the shuffles
    unsigned int error;            // nonzero: a capacity or input check failed
    unsigned int nbig_rev;         // reverse lists longer than one warp
    unsigned int overflow;         // a buffer sized ahead of the counts was too small (OVF_*): the
                                   // join and merge kernels did nothing, the host grows it and reruns
    unsigned int audit_max;        // audit: largest |d~ - d| / (|a|^2 + |b|^2) seen (float bits)
    unsigned long long sum_s;      // sum over joined rows of |new| + |old|
    unsigned long long pairs;      // pair-distance slots of this iteration
    unsigned int ntier[5];         // rows per join tier (by list size)
    unsigned int pad2;
    unsigned long long sum_s_tc;   // the part of sum_s joined on the tensor cores
    unsigned int nemit[4];         // rows of tiers 0-3 with at least one proposal (tensor-core emit pass)
    // reduced-precision joins, counted while profiling: proposals that carry
    // d~, and those of them whose exact distance the merge computed
    unsigned long long approx_props;
    unsigned long long rechecks;
    unsigned int tc_next[2];       // tiles claimed by the tensor-core join's CTAs, per pass
};

// IterCounters::overflow bits (the whole-iteration graph sizes its buffers
// from earlier iterations and checks them on the device).
constexpr unsigned int OVF_PAIRS = 1;      // stored pair distances beyond the pair buffer
constexpr unsigned int OVF_PROPOSALS = 2;  // proposals beyond the bucket array

enum DevError : unsigned int {
    DERR_NONE = 0,
    DERR_LIST_CAP = 1,      // a sample list overflowed its row capacity
    DERR_CROSS_SAMPLE = 2,  // a merge found fewer new ids than it needs
    DERR_TC_WAIT = 4,       // a tensor-core join wait ran out (the kernel gave up)
    DERR_TC_RANGE = 8,      // a reduced-precision emit pass filled a reserved bucket range differently
    DERR_BOUND = 16,        // audit: a pair's reduced-precision distance lay outside its stated bound
};

}  // namespace nnm
