// NN-Descent iterations on the device, reproducing the reference loop
// (kgraph.cpp:98-189, abstractmerge.cpp:78-192, lynndescent.cpp:201-310)
// bit for bit under a fixed seed.
//
// One iteration:
//   1. sampling pass   k_sample_count / k_sample_fill   (kgraph.cpp:105-136)
//      forward new/old lists from each pool, reverse entries to neighbours
//      whose K-th distance is below the entry's distance, flags cleared.
//   2. reverse lists   k_rev_sort_*                    (ascending source row,
//      the order the reference's sequential pass pushes them in)
//   3. shuffle         k_shuffle_append                 (kgraph.cpp:139-162)
//      std::random_shuffle with the std::rand() stream (rng.cu), truncation
//      to smplNum, appended to the sample lists.
//   4. local join      k_join<COUNT>, k_join<FILL>      (pvetex.h:111-125 ...)
//      all valid pairs of a row's lists, exact FP32 distances in the
//      reference's operation order, proposals filtered by the target's K-th
//      distance at the start of the iteration and bucketed per target.
//   5. top-K merge     k_merge                          (pvetex.h:40-85)
//      Within one iteration the reference's sequential UpdateKnnList calls
//      leave in each pool the K smallest (dist, first-insert time) entries of
//      start pool + proposals, with one entry per id (equal ids always have
//      equal distances because the distances are bitwise symmetric).  The
//      merge computes exactly that, so the order of the parallel inserts does
//      not matter.
//   6. convergence     flags counted on the device, mean decided on the host
//      with the reference's float arithmetic.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "nnm_engine.h"
#include "nnm_join.h"
#include "nnm_launch.h"
#include "nnm_scan.h"

namespace nnm {
namespace {

constexpr unsigned FULL = 0xffffffffu;
constexpr int MERGE_WARPS = 8;
constexpr int SHUF_SMEM = 512;  // reverse-list entries a shuffling warp stages in shared memory
constexpr int BIGSORT_CH = 4096;

// ---------------------------------------------------------------------------
// 1. Sampling pass.
struct SampleArgs {
    uint32_t* pid;
    const float* pdist;
    uint32_t n, K, mode, split;
    uint32_t *rcnt_new, *rcnt_old;           // reverse-entry counts (start at the carried length)
    uint32_t *rcur_new, *rcur_old;           // fill cursors (start at the carried length)
    const uint64_t *roff_new, *roff_old;     // reverse segments
    uint32_t *rseg_new, *rseg_old;
    uint32_t *newL, *oldL, *newlen, *oldlen; // sample lists
    uint32_t capn, capo;
    const uint32_t *rnewT, *roldT, *rnewTlen, *roldTlen;  // carried reverse lists (or null)
    uint32_t smpl;
    IterCounters* ctr;
    const float* kth;  // every row's K-th distance (k_kth_gather)
};

// Every row's K-th distance, gathered once per iteration: the sampling and
// the join read it for random rows, and the 4-byte array stays in L2 where
// the pools' last entries (a sector per row) do not.
__global__ void k_kth_gather(const float* pdist, uint32_t K, uint32_t n, float* kth) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) kth[t] = pdist[(size_t)t * K + K - 1];
}

__global__ void k_sample_count(SampleArgs a) {
    uint32_t row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    if (row >= a.n || lane >= (int)a.K) return;
    size_t o = (size_t)row * a.K + lane;
    uint32_t e = a.pid[o];
    float d = a.pdist[o];
    uint32_t id = e & ID_MASK;
    float kth = a.kth[id];
    if (kth < d) atomicAdd((e & FLAG_BIT) ? &a.rcnt_new[id] : &a.rcnt_old[id], 1u);
}

__global__ void k_sample_fill(SampleArgs a) {
    uint32_t row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    if (row >= a.n) return;
    const bool act = lane < (int)a.K;
    size_t o = (size_t)row * a.K + lane;
    uint32_t e = act ? a.pid[o] : 0;
    float d = act ? a.pdist[o] : 0.f;
    uint32_t id = e & ID_MASK;
    bool isnew = act && (e & FLAG_BIT);
    unsigned bal = __ballot_sync(FULL, isnew);
    unsigned actmask = a.K >= 32 ? FULL : ((1u << a.K) - 1u);
    uint32_t nnf = __popc(bal);
    uint32_t base_n = a.newlen[row], base_o = a.oldlen[row];
    if (base_n + nnf > a.capn || base_o + (a.K - nnf) > a.capo) {
        if (lane == 0) atomicOr(&a.ctr->error, (unsigned)DERR_LIST_CAP);
        return;
    }
    uint32_t entry = id | (((e >> 30) & 1u) << 31);
    if (act) {
        unsigned lt = (1u << lane) - 1u;
        if (isnew) a.newL[(size_t)row * a.capn + base_n + __popc(bal & lt)] = entry;
        else a.oldL[(size_t)row * a.capo + base_o + __popc(~bal & actmask & lt)] = entry;
        float kth = a.kth[id];
        if (kth < d) {
            uint32_t rg = (a.mode == MODE_KGRAPH) ? 0u : (row >= a.split ? 1u : 0u);
            uint32_t v = row | (rg << 31);
            if (isnew) a.rseg_new[a.roff_new[id] + atomicAdd(&a.rcur_new[id], 1u)] = v;
            else a.rseg_old[a.roff_old[id] + atomicAdd(&a.rcur_old[id], 1u)] = v;
        }
        if (isnew) a.pid[o] = e & ~FLAG_BIT;
    }
    if (lane == 0) {
        a.newlen[row] = base_n + nnf;
        a.oldlen[row] = base_o + (a.K - nnf);
    }
    if (a.rnewTlen) {  // carried reverse lists go first in this row's segments
        uint32_t cn = a.rnewTlen[row], co = a.roldTlen[row];
        for (uint32_t j = lane; j < cn; j += 32) a.rseg_new[a.roff_new[row] + j] = a.rnewT[(size_t)row * a.smpl + j];
        for (uint32_t j = lane; j < co; j += 32) a.rseg_old[a.roff_old[row] + j] = a.roldT[(size_t)row * a.smpl + j];
    }
}

// ---------------------------------------------------------------------------
// 2. Reverse lists in ascending source-row order.
struct RevSortArgs {
    const uint64_t* roff[2];
    uint32_t* rseg[2];
    uint32_t* rscr[2];
    const uint32_t* carry[2];  // carried prefix length per row (or null)
    uint32_t n;
    uint32_t* big;             // (row | list << 31) of segments longer than 32
    IterCounters* ctr;
};

__device__ __forceinline__ uint32_t rkey(uint32_t v) { return v == 0xffffffffu ? 0xffffffffu : (v & LID_MASK); }

__global__ void k_rev_sort_small(RevSortArgs a) {
    uint32_t t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    int l = blockIdx.y;
    if (t >= a.n) return;
    uint64_t lo = a.roff[l][t] + (a.carry[l] ? a.carry[l][t] : 0), hi = a.roff[l][t + 1];
    uint32_t len = (uint32_t)(hi - lo);
    if (len <= 1) return;
    if (len > 32) {
        if (lane == 0) a.big[atomicAdd(&a.ctr->nbig_rev, 1u)] = t | ((uint32_t)l << 31);
        return;
    }
    uint32_t* seg = a.rseg[l] + lo;
    uint32_t v = lane < (int)len ? seg[lane] : 0xffffffffu;
    for (int k = 2; k <= 32; k <<= 1)
        for (int j = k >> 1; j > 0; j >>= 1) {
            uint32_t o = __shfl_xor_sync(FULL, v, j);
            bool take_min = ((lane & j) == 0) == ((lane & k) == 0);
            uint32_t kv = rkey(v), ko = rkey(o);
            if (take_min ? (ko < kv) : (ko > kv)) v = o;
        }
    if (lane < (int)len) seg[lane] = v;
}

__global__ void k_rev_sort_big(RevSortArgs a) {
    __shared__ uint32_t sh[BIGSORT_CH];
    uint32_t nbig = a.ctr->nbig_rev;
    for (uint32_t bi = blockIdx.x; bi < nbig; bi += gridDim.x) {
        uint32_t code = a.big[bi];
        uint32_t t = code & LID_MASK;
        int l = code >> 31;
        uint64_t lo = a.roff[l][t] + (a.carry[l] ? a.carry[l][t] : 0);
        uint32_t len = (uint32_t)(a.roff[l][t + 1] - lo);
        uint32_t* seg = a.rseg[l] + lo;
        uint32_t* scr = a.rscr[l] + lo;
        // phase 1: bitonic sort of chunks in shared memory
        for (uint32_t cs = 0; cs < len; cs += BIGSORT_CH) {
            uint32_t m = min((uint32_t)BIGSORT_CH, len - cs);
            uint32_t P = 1;
            while (P < m) P <<= 1;
            for (uint32_t i = threadIdx.x; i < P; i += blockDim.x) sh[i] = i < m ? seg[cs + i] : 0xffffffffu;
            __syncthreads();
            for (uint32_t k = 2; k <= P; k <<= 1)
                for (uint32_t j = k >> 1; j > 0; j >>= 1) {
                    for (uint32_t i = threadIdx.x; i < P; i += blockDim.x) {
                        uint32_t ix = i ^ j;
                        if (ix > i) {
                            uint32_t x = sh[i], y = sh[ix];
                            bool asc = (i & k) == 0;
                            if (asc ? rkey(x) > rkey(y) : rkey(x) < rkey(y)) {
                                sh[i] = y;
                                sh[ix] = x;
                            }
                        }
                    }
                    __syncthreads();
                }
            for (uint32_t i = threadIdx.x; i < m; i += blockDim.x) seg[cs + i] = sh[i];
            __syncthreads();
        }
        // phase 2: merge sorted runs pairwise (keys are distinct source rows)
        uint32_t* src = seg;
        uint32_t* dst = scr;
        for (uint32_t w = BIGSORT_CH; w < len; w <<= 1) {
            for (uint32_t i = threadIdx.x; i < len; i += blockDim.x) {
                uint32_t run = i / w;
                uint32_t rs = run * w;
                uint32_t pb = (run & ~1u) * w;
                uint32_t os = (run & 1u) ? rs - w : rs + w;
                uint32_t oe = min(os + w, len);
                if (os > len) os = len;
                uint32_t key = rkey(src[i]);
                uint32_t lo2 = os, hi2 = oe;  // lower bound of key in the other run
                while (lo2 < hi2) {
                    uint32_t mid = (lo2 + hi2) >> 1;
                    if (rkey(src[mid]) < key) lo2 = mid + 1;
                    else hi2 = mid;
                }
                dst[pb + (i - rs) + (lo2 - os)] = src[i];
            }
            __syncthreads();
            uint32_t* tmp = src;
            src = dst;
            dst = tmp;
        }
        if (src != seg)
            for (uint32_t i = threadIdx.x; i < len; i += blockDim.x) seg[i] = src[i];
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// 3. Shuffle, truncate and append.
struct ShufArgs {
    const uint64_t *roff_new, *roff_old;
    uint32_t *rseg_new, *rseg_old;
    const uint64_t* rofs;       // first draw of each row, relative to the generated buffer
    const int32_t* rbuf;
    uint32_t *newL, *oldL, *newlen, *oldlen;
    uint32_t capn, capo, n, smpl;
    uint32_t *rnewT, *roldT, *rnewTlen, *roldTlen;
    uint32_t* npairs;     // pair-distance slots per row
    IterCounters* ctr;
    uint32_t fast, seed, phase;  // fast tier: Philox sample instead of std::random_shuffle
    uint32_t tc_max_s;    // rows with S up to this go to the tensor-core join (no stored pairs)
    int max_staged;       // highest FP32 tier whose vectors fit in shared memory (-1: none); larger lists go unstaged
    uint32_t *rscr_new, *rscr_old;  // scratch of the reverse lists' sizes (fast tier: duplicate removal)
    uint32_t dedupe;      // fast tier, first iteration of an H-Merge level: carried + new lists may repeat ids
    const uint32_t* phase_dev;  // non-null: the draw phase is read here (an iteration graph's replays)
    uint8_t* rtier;       // each row's join tier (0xff: no new entries, not joined); k_tier_lists bins them
};

__global__ void k_rand_count(const uint64_t* roff_new, const uint64_t* roff_old, uint32_t n, uint32_t* out) {
    uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    uint32_t ln = (uint32_t)(roff_new[t + 1] - roff_new[t]);
    uint32_t lo = (uint32_t)(roff_old[t + 1] - roff_old[t]);
    out[t] = (ln ? ln - 1 : 0) + (lo ? lo - 1 : 0);
}

// std::random_shuffle over seg[0..len) with draws[0..len-1), one thread.
__device__ __forceinline__ void shuffle_seg(uint32_t* seg, uint32_t len, const int32_t* draws) {
    for (uint32_t i = 1; i < len; i++) {
        uint32_t j = (uint32_t)(draws[i - 1] % (int32_t)(i + 1));
        if (j != i) {
            uint32_t t = seg[i];
            seg[i] = seg[j];
            seg[j] = t;
        }
    }
}

// Fast tier: keeps, in place at seg[0, keep), the `keep` entries of
// seg[0, len) with the smallest (hash(id), id), the hash a Philox draw keyed
// by (row, phase, list, id) -- a uniform random subset that depends only on
// the ids, not on their order.  The keep-th smallest hash is found by an
// 8-bit radix select (4 rounds over a 256-bin histogram), ties on it by the
// smallest ids.  Warp-wide; hist is this warp's 256-entry shared scratch.
// hc (len entries of shared memory, or null): the hashes, computed once --
// a Philox draw is 10 rounds, and the select reads every hash five times.
__device__ void hash_sample(uint32_t* seg, uint32_t len, uint32_t keep, const Philox& ph, uint32_t t,
                            uint32_t phase, uint32_t l, uint32_t* hist, uint32_t* hc) {
    const int lane = threadIdx.x & 31;
    uint32_t prefix = 0, need = keep;
    if (hc) {
        for (uint32_t j = lane; j < len; j += 32) hc[j] = ph(t, phase, l, seg[j] & LID_MASK).x;
        __syncwarp();
    }
    auto hash = [&](uint32_t j) { return hc ? hc[j] : ph(t, phase, l, seg[j] & LID_MASK).x; };
    for (int byte = 3; byte >= 0; byte--) {
        for (uint32_t i = lane; i < 256; i += 32) hist[i] = 0;
        __syncwarp();
        const uint32_t hi_mask = byte == 3 ? 0u : (0xffffffffu << (8 * (byte + 1)));
        for (uint32_t j = lane; j < len; j += 32) {
            const uint32_t h = hash(j);
            if ((h & hi_mask) == prefix) atomicAdd(&hist[(h >> (8 * byte)) & 255u], 1u);
        }
        __syncwarp();
        // the bin holding the need-th entry: 8 bins per lane, scan over lanes
        uint32_t c[8], sum = 0;
#pragma unroll
        for (int q = 0; q < 8; q++) {
            c[q] = hist[lane * 8 + q];
            sum += c[q];
        }
        uint32_t incl = sum;
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(FULL, incl, o);
            if (lane >= o) incl += y;
        }
        const uint32_t excl = incl - sum;
        const int src = __ffs(__ballot_sync(FULL, excl < need && need <= incl)) - 1;
        uint32_t bin = 0, before = 0;
        if (lane == src) {
            uint32_t run = excl;
#pragma unroll
            for (int q = 0; q < 8; q++) {
                if (run + c[q] >= need) {
                    bin = lane * 8 + q;
                    before = run;
                    break;
                }
                run += c[q];
            }
        }
        bin = __shfl_sync(FULL, bin, src);
        before = __shfl_sync(FULL, before, src);
        need -= before;
        prefix |= bin << (8 * byte);
        __syncwarp();
    }
    // all hashes below the threshold T, and the `need` smallest ids at T
    const uint32_t T = prefix;
    uint32_t idT = 0;
    for (uint32_t r = 0; r < need; r++) {
        uint32_t mn = 0xffffffffu;
        for (uint32_t j = lane; j < len; j += 32) {
            const uint32_t id = seg[j] & LID_MASK;
            if ((r == 0 || id > idT) && id < mn && hash(j) == T) mn = id;
        }
        idT = __reduce_min_sync(FULL, mn);
    }
    uint32_t out = 0;
    for (uint32_t j0 = 0; j0 < len; j0 += 32) {  // stable compaction in place
        const uint32_t j = j0 + lane;
        uint32_t v = 0;
        bool sel = false;
        if (j < len) {
            v = seg[j];
            const uint32_t id = v & LID_MASK, h = hash(j);
            sel = h < T || (h == T && id <= idT);
        }
        __syncwarp();
        const unsigned m = __ballot_sync(FULL, sel);
        const uint32_t pos = out + __popc(m & ((1u << lane) - 1u));
        if (sel && pos < keep) seg[pos] = v;
        out += __popc(m);
        __syncwarp();
    }
}

// Removes repeated ids from seg[0, len): an id's copies keep the larger word
// (a set group bit wins), identical copies the first; the kept entries go to
// scr in list order and back to seg.  The kept set does not depend on the
// order of the list (which, in the fast tier, is the order of atomics), so
// the hash sample after it is deterministic.  Returns the new length.
__device__ uint32_t dedupe_ids(uint32_t* seg, uint32_t len, uint32_t* scr) {
    const int lane = threadIdx.x & 31;
    uint32_t out = 0;
    for (uint32_t j0 = 0; j0 < len; j0 += 32) {
        const uint32_t j = j0 + lane;
        bool keep = false;
        uint32_t v = 0;
        if (j < len) {
            v = seg[j];
            keep = true;
            for (uint32_t i = 0; i < len && keep; i++) {
                const uint32_t u = seg[i];
                if (i != j && (u & LID_MASK) == (v & LID_MASK) && (u > v || (u == v && i < j))) keep = false;
            }
        }
        const unsigned m = __ballot_sync(FULL, keep);
        if (keep) scr[out + __popc(m & ((1u << lane) - 1u))] = v;
        out += __popc(m);
    }
    __syncwarp();
    for (uint32_t j = lane; j < out; j += 32) seg[j] = scr[j];
    __syncwarp();
    return out;
}

// One warp per row: lane 0 shuffles in shared memory, the warp appends.
__global__ void k_shuffle_append(ShufArgs a) {
    __shared__ uint32_t stage[8][SHUF_SMEM];
    __shared__ uint32_t hist[8][256];
    int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    uint32_t t = blockIdx.x * 8 + w;
    if (t >= a.n) return;
    const int32_t* draws = a.fast ? nullptr : a.rbuf + a.rofs[t];
    uint32_t nl = a.newlen[t], ol = a.oldlen[t];
    // both lists' segments read up front (independent loads in flight together)
    const uint64_t lo_n = a.roff_new[t], hi_n = a.roff_new[t + 1], lo_o = a.roff_old[t], hi_o = a.roff_old[t + 1];
    // Fast tier, the common row: both reverse lists of at most 32 entries
    // and within the sample cap -- kept whole, in list order -- copied with
    // one load of each list, in flight together.
    if (a.fast && !a.dedupe && hi_n - lo_n <= min(32u, a.smpl) && hi_o - lo_o <= min(32u, a.smpl)) {
        const uint32_t ln = (uint32_t)(hi_n - lo_n), lk = (uint32_t)(hi_o - lo_o);
        const uint32_t vn = lane < (int)ln ? a.rseg_new[lo_n + lane] : 0u;
        const uint32_t vo = lane < (int)lk ? a.rseg_old[lo_o + lane] : 0u;
        if (nl + ln > a.capn || ol + lk > a.capo) {
            if (lane == 0) {
                atomicOr(&a.ctr->error, (unsigned)DERR_LIST_CAP);
                a.rtier[t] = 0xff;
            }
            return;
        }
        if (lane < (int)ln) {
            a.newL[(size_t)t * a.capn + nl + lane] = vn;
            if (a.rnewT) a.rnewT[(size_t)t * a.smpl + lane] = vn;
        }
        if (lane < (int)lk) {
            a.oldL[(size_t)t * a.capo + ol + lane] = vo;
            if (a.roldT) a.roldT[(size_t)t * a.smpl + lane] = vo;
        }
        if (lane == 0 && a.rnewT) {
            a.rnewTlen[t] = ln;
            a.roldTlen[t] = lk;
        }
        nl += ln;
        ol += lk;
    } else
    for (int l = 0; l < 2; l++) {
        uint64_t lo = l ? lo_o : lo_n;
        uint32_t len = (uint32_t)((l ? hi_o : hi_n) - lo);
        uint32_t* seg = (l ? a.rseg_old : a.rseg_new) + lo;
        if (a.dedupe && len > 1) len = dedupe_ids(seg, len, (l ? a.rscr_old : a.rscr_new) + lo);
        uint32_t keep = min(len, a.smpl);
        uint32_t* sh = stage[w];
        bool staged = len <= SHUF_SMEM;
        if (a.fast) {
            // a uniform random subset of smplNum entries, chosen by id
            if (len > a.smpl)
                hash_sample(seg, len, keep, Philox{a.seed, 0x6e6e6d01u}, t, a.phase_dev ? *a.phase_dev : a.phase,
                            (uint32_t)l, hist[w], staged ? stage[w] : nullptr);
            __syncwarp();
            sh = seg;
        } else if (staged) {
            for (uint32_t j = lane; j < len; j += 32) sh[j] = seg[j];
            __syncwarp();
            if (lane == 0) shuffle_seg(sh, len, draws);
            __syncwarp();
        } else {
            if (lane == 0) shuffle_seg(seg, len, draws);
            __syncwarp();
            sh = seg;
        }
        draws += len ? len - 1 : 0;
        uint32_t* L = l ? a.oldL + (size_t)t * a.capo : a.newL + (size_t)t * a.capn;
        uint32_t base = l ? ol : nl;
        uint32_t cap = l ? a.capo : a.capn;
        uint32_t* T = l ? a.roldT : a.rnewT;
        if (base + keep > cap) {
            if (lane == 0) {
                atomicOr(&a.ctr->error, (unsigned)DERR_LIST_CAP);
                a.rtier[t] = 0xff;
            }
            return;
        }
        for (uint32_t j = lane; j < keep; j += 32) {
            uint32_t v = sh[j];
            L[base + j] = v;
            if (T) T[(size_t)t * a.smpl + j] = v;
        }
        if (l) ol += keep;
        else nl += keep;
        if (lane == 0 && T) (l ? a.roldTlen : a.rnewTlen)[t] = keep;
        __syncwarp();
    }
    if (lane == 0) {
        a.newlen[t] = nl;
        a.oldlen[t] = ol;
        // stored pairs of the local join: new x new above the diagonal, new x old
        const uint32_t S = nl + ol;
        a.npairs[t] = nl && S > a.tc_max_s ? nl * (nl - 1) / 2 + nl * ol : 0u;
        int tier = 0xff;
        if (nl) {
            tier = tier_of(S);
            // next to the tensor-core join (tc_max_s != 0) longer lists take the
            // pair kernel; without it, tiers whose staged vectors do not fit
            if (tier < NTIER - 1 && S > a.tc_max_s && (a.tc_max_s != 0 || tier > a.max_staged)) tier = NTIER - 1;
        }
        a.rtier[t] = (uint8_t)tier;
    }
}

// The tier lists from the rows' tiers: a block per chunk of rows counts its
// rows per tier in shared memory, reserves each tier's range with one
// global atomic, then places its rows.  (An atomic per row on the five tier
// counters serialised the shuffle kernel.)  The order within a tier is free:
// the joins and the merge do not depend on it.
constexpr uint32_t TIER_CHUNK = 2048;
__global__ void __launch_bounds__(256) k_tier_lists(const uint8_t* rtier, uint32_t n, uint32_t* tier_rows,
                                                    IterCounters* ctr) {
    __shared__ uint32_t cnt[NTIER], base[NTIER];
    const uint32_t c0 = blockIdx.x * TIER_CHUNK, c1 = min(n, c0 + TIER_CHUNK);
    if (threadIdx.x < NTIER) cnt[threadIdx.x] = 0;
    __syncthreads();
    for (uint32_t r = c0 + threadIdx.x; r < c1; r += blockDim.x) {
        const uint32_t t = rtier[r];
        if (t < NTIER) atomicAdd(&cnt[t], 1u);
    }
    __syncthreads();
    if (threadIdx.x < NTIER) {
        base[threadIdx.x] = cnt[threadIdx.x] ? atomicAdd(&ctr->ntier[threadIdx.x], cnt[threadIdx.x]) : 0u;
        cnt[threadIdx.x] = 0;
    }
    __syncthreads();
    for (uint32_t r = c0 + threadIdx.x; r < c1; r += blockDim.x) {
        const uint32_t t = rtier[r];
        if (t < NTIER) tier_rows[(size_t)t * n + base[t] + atomicAdd(&cnt[t], 1u)] = r;
    }
}

// ---------------------------------------------------------------------------
// 4. Local join, in two kernels.
//   k_pairs: every pair of a row's lists once -- new x new above the
//     diagonal and new x old -- with the exact sequential distance, stored
//     in the row's slice of the pair buffer; per list position, the number
//     of proposals that pass the K-th-distance filter (for bucket sizes).
//   k_emit: reads the stored distances and writes the proposals into the
//     per-target buckets.
// Vectors of a row's lists in shared memory: row q starts at 16-byte unit
// q * vstride + q / 4 with vstride = 1 mod 8, so that the rows of 4x4 tiles
// of neighbouring threads (q = 4t + i for consecutive t) fall in different
// bank groups.
__device__ __forceinline__ uint32_t vrow(uint32_t q, uint32_t vstride) { return q * vstride + (q >> 2); }
__host__ __device__ __forceinline__ uint32_t vec_stride(uint32_t units) { return ((units + 7) & ~7u) + 1; }

// Where pairs_row reads a row's vectors: FP32 from global memory (L2), FP32
// staged in shared memory, or the u8 operand copy of the tensor-core join
// staged in shared memory.  The u8 form is used only when every component
// is an integer in [0, 255]: d(a, b) = |a|^2 + |b|^2 - 2 a.b is then an
// exact integer below 2^24, the value of the reference's sequential float
// sum of the same terms, so all three give the same distances.
constexpr int VEC_GLOBAL = 0, VEC_F32 = 1, VEC_U8 = 2;

template <int M, int VEC>
__device__ void pairs_row(const JoinArgs& a, uint32_t row, unsigned char* smem, uint32_t R) {
    const uint32_t nn = a.newlen[row], no = a.oldlen[row], S = nn + no;
    uint32_t* s_ids = reinterpret_cast<uint32_t*>(smem);
    float* s_kth = reinterpret_cast<float*>(s_ids + R);
    uint32_t* s_cnt = reinterpret_cast<uint32_t*>(s_kth + R);
    uint32_t* s_grp = s_cnt + R;
    uint32_t* s_nrm = s_grp + R;  // VEC_U8 only
    float4* s_vec = reinterpret_cast<float4*>(VEC == VEC_U8 ? s_nrm + ((R + 3) & ~3u) : s_grp + R);
    const uint32_t dq = VEC == VEC_U8 ? a.kq >> 4 : a.dp >> 2, vstride = vec_stride(dq);
    const float4* x4 = reinterpret_cast<const float4*>(VEC == VEC_U8 ? (const void*)a.xq : (const void*)a.x);

    for (uint32_t q = threadIdx.x; q < S; q += blockDim.x) {
        uint32_t e = q < nn ? a.newL[(size_t)row * a.capn + q] : a.oldL[(size_t)row * a.capo + q - nn];
        uint32_t id = e & LID_MASK;
        s_ids[q] = e;
        s_kth[q] = a.kthv[id];
        s_cnt[q] = 0;
        s_grp[q] = a.mode == MODE_SMERGE ? leaf_of(id, a.leaf_off, a.nleaf) : (e >> 31);
        if (VEC == VEC_U8) s_nrm[q] = a.nrm[id];
    }
    __syncthreads();
    if (VEC != VEC_GLOBAL) {
        for (uint32_t i = threadIdx.x; i < S * dq; i += blockDim.x) {
            uint32_t q = i / dq, c = i - q * dq;
            s_vec[vrow(q, vstride) + c] = x4[(size_t)(s_ids[q] & LID_MASK) * dq + c];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) atomicAdd(&a.ctr->sum_s, (unsigned long long)S);
    const uint32_t ntA = (nn + 3) >> 2, ntB = (S + 3) >> 2;
    const uint32_t ntiles = ntA * ntB - ntA * (ntA - 1) / 2;
    float* pd = a.pd + a.poff[row];
    uint32_t cmps = 0;
    for (uint32_t t = threadIdx.x; t < ntiles; t += blockDim.x) {
        uint32_t ta = 0, rem = t;
        while (rem >= ntB - ta) {
            rem -= ntB - ta;
            ta++;
        }
        const uint32_t tb = ta + rem;
        const float4* pa[4];
        const float4* pb[4];
#pragma unroll
        for (int i = 0; i < 4; i++) {
            uint32_t ai = min(ta * 4 + i, nn - 1), bj = min(tb * 4 + i, S - 1);
            pa[i] = VEC != VEC_GLOBAL ? s_vec + vrow(ai, vstride) : x4 + (size_t)(s_ids[ai] & LID_MASK) * dq;
            pb[i] = VEC != VEC_GLOBAL ? s_vec + vrow(bj, vstride) : x4 + (size_t)(s_ids[bj] & LID_MASK) * dq;
        }
        float acc[4][4];
        if (VEC == VEC_U8) {
            uint32_t dot[4][4];
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) dot[i][j] = 0u;
            for (uint32_t c = 0; c < dq; c++) {  // 16 components per step
                uint4 A[4], B[4];
#pragma unroll
                for (int i = 0; i < 4; i++) {
                    A[i] = reinterpret_cast<const uint4*>(pa[i])[c];
                    B[i] = reinterpret_cast<const uint4*>(pb[i])[c];
                }
#pragma unroll
                for (int i = 0; i < 4; i++)
#pragma unroll
                    for (int j = 0; j < 4; j++) {
                        dot[i][j] = __dp4a(A[i].x, B[j].x, dot[i][j]);
                        dot[i][j] = __dp4a(A[i].y, B[j].y, dot[i][j]);
                        dot[i][j] = __dp4a(A[i].z, B[j].z, dot[i][j]);
                        dot[i][j] = __dp4a(A[i].w, B[j].w, dot[i][j]);
                    }
            }
#pragma unroll
            for (int i = 0; i < 4; i++) {
                const uint32_t na = s_nrm[min(ta * 4 + i, nn - 1)];
#pragma unroll
                for (int j = 0; j < 4; j++)
                    acc[i][j] = (float)((int)(na + s_nrm[min(tb * 4 + j, S - 1)]) - 2 * (int)dot[i][j]);
            }
        } else {
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) acc[i][j] = 0.f;
            for (uint32_t c = 0; c < dq; c++) {
                float4 A[4], B[4];
#pragma unroll
                for (int i = 0; i < 4; i++) {
                    A[i] = pa[i][c];
                    B[i] = pb[i][c];
                }
#pragma unroll
                for (int i = 0; i < 4; i++)
#pragma unroll
                    for (int j = 0; j < 4; j++) {
                        acc[i][j] = dist_step<M>(acc[i][j], A[i].x, B[j].x);
                        acc[i][j] = dist_step<M>(acc[i][j], A[i].y, B[j].y);
                        acc[i][j] = dist_step<M>(acc[i][j], A[i].z, B[j].z);
                        acc[i][j] = dist_step<M>(acc[i][j], A[i].w, B[j].w);
                    }
            }
        }
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const uint32_t av = ta * 4 + i;
            if (av >= nn) continue;
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const uint32_t bv = tb * 4 + j;
                if (bv >= S || (bv < nn && bv <= av)) continue;
                const float dd = acc[i][j];
                pd[pair_slot(av, bv, nn, no)] = dd;
                uint32_t outer, inner;
                if (!pair_order(a.mode, a.verse, av, bv, nn, s_ids[av], s_ids[bv], s_grp[av], s_grp[bv], outer, inner))
                    continue;
                cmps++;
                if (dd < s_kth[outer]) atomicAdd(&s_cnt[outer], 1u);
                if (dd < s_kth[inner]) atomicAdd(&s_cnt[inner], 1u);
            }
        }
    }
    for (int o = 16; o > 0; o >>= 1) cmps += __shfl_xor_sync(FULL, cmps, o);
    if ((threadIdx.x & 31) == 0 && cmps) atomicAdd(&a.ctr->ncmps, (unsigned long long)cmps);
    __syncthreads();
    for (uint32_t q = threadIdx.x; q < S; q += blockDim.x) {
        uint32_t c = s_cnt[q];
        a.cntpos[(size_t)row * a.caps + q] = (uint16_t)c;
        if (c) atomicAdd(&a.bcnt[s_ids[q] & LID_MASK], c);
    }
    __syncthreads();
}

template <int M, int TIER>
__global__ void __launch_bounds__(TIER_THREADS[TIER]) k_pairs(JoinArgs a, uint32_t R) {
    extern __shared__ __align__(16) unsigned char smem[];
    if (a.ctr->overflow) return;
    const uint32_t cnt = a.ctr->ntier[TIER];
    const uint32_t* rows = a.tier_rows + (size_t)TIER * a.n;
    for (uint32_t b = blockIdx.x; b < cnt; b += gridDim.x)
        pairs_row<M, (TIER < NTIER - 1 ? VEC_F32 : VEC_GLOBAL)>(a, rows[b], smem, R);
}

// Rows of the last tier (S > 128) next to the u8 tensor-core join: the u8
// vectors staged in shared memory, integer dot products (dp4a).
__global__ void __launch_bounds__(TIER_THREADS[NTIER - 1]) k_pairs_u8(JoinArgs a, uint32_t R) {
    extern __shared__ __align__(16) unsigned char smem[];
    if (a.ctr->overflow) return;
    const uint32_t cnt = a.ctr->ntier[NTIER - 1];
    const uint32_t* rows = a.tier_rows + (size_t)(NTIER - 1) * a.n;
    for (uint32_t b = blockIdx.x; b < cnt; b += gridDim.x) pairs_row<L2, VEC_U8>(a, rows[b], smem, R);
}

// One warp per row: proposals from the stored pair distances.  With the
// tensor-core join active, only the rows of the last tier have stored pairs.
constexpr int EMIT_WARPS = 4;

// Members of one row (bucket bases, ids, K-th distances, cursors, groups)
// in shared memory, 24 bytes a list slot.
struct EmitRow {
    unsigned long long* base;
    uint32_t *ids, *cur, *grp;
    float* kth;
};

__device__ __forceinline__ EmitRow emit_row_smem(unsigned char* p, uint32_t R) {
    EmitRow m;
    m.base = reinterpret_cast<unsigned long long*>(p);
    m.ids = reinterpret_cast<uint32_t*>(m.base + R);
    m.kth = reinterpret_cast<float*>(m.ids + R);
    m.cur = reinterpret_cast<uint32_t*>(m.kth + R);
    m.grp = m.cur + R;
    return m;
}

// Loads the members of list slots first, first + step, ... and reserves
// their bucket ranges; false when no pair of the row passed the filter.
__device__ __forceinline__ bool emit_load_row(const JoinArgs& a, uint32_t row, uint32_t nn, uint32_t S,
                                              EmitRow m, uint32_t first, uint32_t step) {
    bool any_c = false;
    for (uint32_t q = first; q < S; q += step) {
        uint32_t e = q < nn ? a.newL[(size_t)row * a.capn + q] : a.oldL[(size_t)row * a.capo + q - nn];
        uint32_t id = e & LID_MASK;
        m.ids[q] = e;
        m.kth[q] = a.kthv[id];
        m.cur[q] = 0;
        m.grp[q] = a.mode == MODE_SMERGE ? leaf_of(id, a.leaf_off, a.nleaf) : (e >> 31);
        uint32_t c = a.cntpos[(size_t)row * a.caps + q];
        if (c) m.base[q] = a.boff[id] + atomicAdd(&a.bcur[id], c);
        any_c |= c != 0;
    }
    return any_c;
}

// Proposals of the pairs (av, bv) of a row with av = av0, av0 + av_step, ...
// (a warp's share), lanes over bv; FAST: the fast tier's 8-byte form.
template <bool FAST>
__device__ __forceinline__ void emit_pairs(const JoinArgs& a, uint32_t row, uint32_t nn, uint32_t no,
                                           EmitRow m, uint32_t av0, uint32_t av_step) {
    const int lane = threadIdx.x & 31;
    const uint32_t S = nn + no;
    const unsigned long long* s_base = m.base;
    const uint32_t* s_ids = m.ids;
    const float* s_kth = m.kth;
    uint32_t* s_cur = m.cur;
    const uint32_t* s_grp = m.grp;
    const float* pd = a.pd + a.poff[row];
    for (uint32_t av = av0; av < nn; av += av_step) {
        for (uint32_t bv = av + 1 + lane; bv < S; bv += 32) {
            uint32_t outer, inner;
            if (!pair_order(a.mode, a.verse, av, bv, nn, s_ids[av], s_ids[bv], s_grp[av], s_grp[bv], outer, inner))
                continue;
            const float dd = pd[pair_slot(av, bv, nn, no)];
            const uint32_t pidx = outer * S + inner;
            if (dd < s_kth[outer]) {
                unsigned long long slot = s_base[outer] + atomicAdd(&s_cur[outer], 1u);
                put_prop<FAST>(a.bucket, slot, dd, s_ids[inner], row, pidx, 0);
            }
            if (dd < s_kth[inner]) {
                unsigned long long slot = s_base[inner] + atomicAdd(&s_cur[inner], 1u);
                put_prop<FAST>(a.bucket, slot, dd, s_ids[outer], row, pidx, 1);
            }
        }
    }
}

// FP32 join: a warp per row.
__global__ void __launch_bounds__(EMIT_WARPS * 32) k_emit(JoinArgs a) {
    extern __shared__ __align__(16) unsigned char smem[];
    if (a.ctr->overflow) return;
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t row = blockIdx.x * EMIT_WARPS + w;
    if (row >= a.n) return;
    const uint32_t nn = a.newlen[row], no = a.oldlen[row];
    if (nn == 0) return;
    const EmitRow m = emit_row_smem(smem + (size_t)w * a.caps * 24, a.caps);
    if (!__any_sync(FULL, emit_load_row(a, row, nn, nn + no, m, lane, 32))) return;
    __syncwarp();
    if (a.fast_key) emit_pairs<true>(a, row, nn, no, m, 0, 1);
    else emit_pairs<false>(a, row, nn, no, m, 0, 1);
}

// Rows of the last tier next to the tensor-core join (lists of more than
// 128 entries, up to caps^2 / 2 pairs each, a few thousand rows): a block
// per row, its warps taking the outer entries in turn, so that no row is a
// single warp's long chain of loads.
constexpr int EMIT_ROW_WARPS = 8;

__global__ void __launch_bounds__(EMIT_ROW_WARPS * 32) k_emit_rows(JoinArgs a) {
    extern __shared__ __align__(16) unsigned char smem[];
    if (a.ctr->overflow) return;
    const uint32_t cnt = a.ctr->ntier[NTIER - 1];
    for (uint32_t b = blockIdx.x; b < cnt; b += gridDim.x) {  // a block per row
        const uint32_t row = a.tier_rows[(size_t)(NTIER - 1) * a.n + b];
        const uint32_t nn = a.newlen[row], no = a.oldlen[row];
        if (nn == 0) continue;
        const EmitRow m = emit_row_smem(smem, a.caps);
        const bool any = __syncthreads_or(emit_load_row(a, row, nn, nn + no, m, threadIdx.x, blockDim.x));
        if (any) {
            if (a.fast_key) emit_pairs<true>(a, row, nn, no, m, threadIdx.x >> 5, EMIT_ROW_WARPS);
            else emit_pairs<false>(a, row, nn, no, m, threadIdx.x >> 5, EMIT_ROW_WARPS);
        }
        __syncthreads();  // the row's members in shared memory are read before the next row's load
    }
}

// ---------------------------------------------------------------------------
// 5. Top-K merge per target.
struct MergeArgs {
    uint32_t* pid;
    float* pdist;
    uint32_t n, K;
    const uint32_t* bcnt;
    const uint64_t* boff;
    const void* bucket;  // Prop (exact tier) or Prop8 (fast tier) entries
    uint8_t* nflag;
    IterCounters* ctr;
    // reduced-precision joins: proposals flagged APPROX_BIT carry d~; the
    // exact distance is the sequential FP32 sum of the rows of x, and
    // |d~ - d| <= err_c * (nrm[t] + nrm[u]) (float norms)
    const float* x;
    uint32_t dp;
    const uint32_t* nrm;
    float err_c;
    uint32_t count_approx;  // count the approximate proposals and their exact rechecks (profiling)
};

// Proposal number i of the bucket array: distance bits and list entry (and,
// exact tier, the key).
template <bool FAST>
__device__ __forceinline__ void load_prop(const void* bucket, unsigned long long i, uint32_t& dbits, uint32_t& idg,
                                          unsigned long long& key) {
    if (FAST) {
        const uint2 p = reinterpret_cast<const uint2*>(bucket)[i];
        dbits = p.x;
        idg = p.y;
        key = fast_key(idg);
    } else {
        const Prop p = reinterpret_cast<const Prop*>(bucket)[i];
        dbits = __float_as_uint(p.dist);
        idg = p.idg;
        key = p.key;
    }
}

// The reference's FP32 distance of rows t and u (the reduced-precision
// joins' exact value), one non-inlined copy.
__device__ __noinline__ float merge_exact_l2(const float* x, uint32_t dp, uint32_t t, uint32_t u) {
    return dist_seq<L2>(x + (size_t)t * dp, x + (size_t)u * dp, (int)dp);
}

struct MEnt {
    uint32_t d;
    uint32_t e;
    unsigned long long k;
};

__device__ __forceinline__ bool mless(uint32_t d1, unsigned long long k1, uint32_t d2, unsigned long long k2) {
    return d1 < d2 || (d1 == d2 && k1 < k2);
}

// Number of entries of a sorted per-lane list (first `cnt` lanes) that are
// smaller than (d, k) -- or, with `or_equal`, not greater.  Pool entries
// count the smaller proposals and proposals count the pool entries that
// are not greater, so that an entry present on both sides (the same
// proposal made twice, possible with the fast tier's keys) gets two
// distinct merged positions, pool first; the duplicate is dropped below.
__device__ __forceinline__ uint32_t count_less(uint32_t ld, unsigned long long lk, uint32_t cnt, uint32_t d,
                                               unsigned long long k, bool or_equal = false) {
    uint32_t lo = 0, hi = cnt;
#pragma unroll
    for (int s = 0; s < 6; s++) {
        uint32_t mid = (lo + hi) >> 1;
        uint32_t md = __shfl_sync(FULL, ld, mid & 31);
        unsigned long long mk = __shfl_sync(FULL, lk, mid & 31);
        if (lo < hi) {
            const bool below = mless(md, mk, d, k) || (or_equal && md == d && mk == k);
            if (below) lo = mid + 1;
            else hi = mid;
        }
    }
    return lo;
}

// One round of the merge: the sorted chunk (pd, pk, pe; m valid entries in
// the first lanes) merged with the pool (cd, ce, ck in lanes < K), equal
// ids dropped (first in (dist, key) order kept), K smallest kept.
__device__ __forceinline__ void merge_round(uint32_t pd, unsigned long long pk, uint32_t pe, uint32_t m, uint32_t K,
                                            uint32_t& cd, uint32_t& ce, unsigned long long& ck, MEnt* sm,
                                            MEnt* kept) {
    const int lane = threadIdx.x & 31;
    {
        const uint32_t pos = lane + count_less(pd, pk, m, cd, ck);  // every lane takes part in the shuffles
        if (lane < (int)K) sm[pos] = MEnt{cd, ce, ck};
    }
    {
        uint32_t pos = lane + count_less(cd, ck, K, pd, pk, true);
        if (lane < (int)m) sm[pos] = MEnt{pd, pe, pk};
    }
    __syncwarp();
    const uint32_t tot = K + m;
    bool keep0 = false, keep1 = false;
    for (int h = 0; h < 2; h++) {
        uint32_t s = lane + 32 * h;
        bool keep = false;
        if (s < tot) {
            keep = true;
            MEnt me = sm[s];
            for (int q = (int)s - 1; q >= 0 && sm[q].d == me.d; q--)
                if ((sm[q].e & ID_MASK) == (me.e & ID_MASK)) {
                    keep = false;
                    break;
                }
        }
        if (h == 0) keep0 = keep;
        else keep1 = keep;
    }
    unsigned b0m = __ballot_sync(FULL, keep0), b1m = __ballot_sync(FULL, keep1);
    unsigned lt = (1u << lane) - 1u;
    uint32_t r0 = __popc(b0m & lt), r1 = __popc(b0m) + __popc(b1m & lt);
    if (keep0 && r0 < K) kept[r0] = sm[lane];
    if (keep1 && r1 < K) kept[r1] = sm[lane + 32];
    __syncwarp();
    if (lane < (int)K) {
        MEnt me = kept[lane];
        cd = me.d;
        ce = me.e;
        ck = me.k;
    }
    __syncwarp();
}

// Bitonic sort of one entry per lane by (dist, key).
__device__ __forceinline__ void warp_sort_ment(uint32_t& pd, unsigned long long& pk, uint32_t& pe) {
    const int lane = threadIdx.x & 31;
    for (int k = 2; k <= 32; k <<= 1)
        for (int j = k >> 1; j > 0; j >>= 1) {
            uint32_t od = __shfl_xor_sync(FULL, pd, j);
            unsigned long long ok = __shfl_xor_sync(FULL, pk, j);
            uint32_t oe = __shfl_xor_sync(FULL, pe, j);
            bool take_min = ((lane & j) == 0) == ((lane & k) == 0);
            bool swap = take_min ? mless(od, ok, pd, pk) : mless(pd, pk, od, ok);
            if (swap) {
                pd = od;
                pk = ok;
                pe = oe;
            }
        }
}

// Fast-tier merge.  A fast-tier key is a function of the entry (fast_key),
// so an entry and its order fit one 64-bit word:
//   dist bits (63..32) | id (31..2) | new flag (1) | group bit ^ 1 (0)
// and the words order as (distance, id, ...) (distances are non-negative,
// so their bits order as the floats).  Copies of an entry -- the same id at
// the same distance -- are adjacent in sorted order, one already in the pool
// (flag 0) before a proposal, proposals of group 1 before group 0 (as
// fast_key orders them); the first copy is kept.  The start pool is keyed
// the same way: entries of equal distance order by id, not by their
// previous position, and a proposal equal in distance to a pool entry of a
// larger id precedes it -- deterministic, as the tier requires.
__device__ __forceinline__ unsigned long long fm_word(uint32_t dist_bits, uint32_t pool_word) {
    return ((unsigned long long)dist_bits << 32) | ((pool_word & ID_MASK) << 2) | ((pool_word >> 31) << 1) |
           (((pool_word >> 30) & 1u) ^ 1u);
}

__device__ __forceinline__ uint32_t fm_pool_word(unsigned long long v) {
    const uint32_t lo = (uint32_t)v;
    return ((lo >> 2) & ID_MASK) | (((lo & 1u) ^ 1u) << 30) | (((lo >> 1) & 1u) << 31);
}

// Ascending bitonic sort of one word per lane.
__device__ __forceinline__ unsigned long long fm_sort32(unsigned long long v) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int k = 2; k <= 32; k <<= 1)
#pragma unroll
        for (int j = k >> 1; j > 0; j >>= 1) {
            const unsigned long long o = __shfl_xor_sync(FULL, v, j);
            const bool take_min = ((lane & j) == 0) == ((lane & k) == 0);
            v = take_min ? min(v, o) : max(v, o);
        }
    return v;
}

// Ascending order of a bitonic sequence of one word per lane.
__device__ __forceinline__ unsigned long long fm_bitonic_merge32(unsigned long long v) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int j = 16; j > 0; j >>= 1) {
        const unsigned long long o = __shfl_xor_sync(FULL, v, j);
        v = (lane & j) ? max(v, o) : min(v, o);
    }
    return v;
}

constexpr unsigned long long FM_EMPTY = ~0ull;

// Reduced-precision joins: an upper bound (float bits) of the K-th exact
// distance the merge will leave -- the K-th smallest of the start pool's
// exact distances and, for each id proposed and not in the pool, one upper
// bound of its distance (d~ + err_c (|t|^2 + |u|^2), or the exact value).
// Any set of K distinct ids bounds the final K-th entry from above, so a
// proposal whose lower bound exceeds it cannot enter the pool.  The 32
// smallest upper bounds are kept by a buffered warp sort, then ids already
// in the pool or repeated among them are dropped.  pool_d / pool_id: the
// start pool in lanes < K, ascending distances; scratch: 32 words.
template <bool FAST>
__device__ uint32_t approx_bound(const MergeArgs& a, unsigned long long b_first, uint32_t c, uint32_t K,
                                 uint32_t pool_d, uint32_t pool_id, float nt, unsigned long long* scratch) {
    const int lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;
    constexpr unsigned long long EMPTY = ~0ull;
    unsigned long long kept = EMPTY, klast = EMPTY;
    uint32_t nb = 0;
    for (uint32_t b0 = 0;; b0 += 32) {
        const bool last = b0 >= c;
        unsigned long long v = EMPTY;
        bool rest = false;
        if (last) {
            if (nb == 0) break;
        } else {
            bool valid = false;
            if (b0 + lane < c) {
                uint32_t dbits, idg;
                unsigned long long key;
                load_prop<FAST>(a.bucket, b_first + b0 + lane, dbits, idg, key);
                const uint32_t id = idg & ID_MASK;
                float ub = __uint_as_float(dbits);
                if (idg & APPROX_BIT) ub += a.err_c * (nt + __uint_as_float(a.nrm[id]));
                v = ((unsigned long long)__float_as_uint(ub) << 32) | id;
                valid = v < klast;
            }
            const unsigned vb = __ballot_sync(FULL, valid);
            if (!vb) continue;
            const uint32_t take = min((uint32_t)__popc(vb), 32u - nb);
            const uint32_t rank = __popc(vb & lt);
            if (valid && rank < take) scratch[nb + rank] = v;
            __syncwarp();
            nb += take;
            if (nb < 32) continue;
            rest = valid && rank >= take;
        }
        unsigned long long bv = lane < (int)nb ? scratch[lane] : EMPTY;
        __syncwarp();
        // the 32 smallest of kept and the buffer
        bv = fm_sort32(bv);
        kept = fm_bitonic_merge32(min(kept, __shfl_sync(FULL, bv, 31 - lane)));
        klast = __shfl_sync(FULL, kept, 31);
        nb = 0;
        if (last) break;
        rest = rest && v < klast;
        const unsigned rb = __ballot_sync(FULL, rest);
        if (rest) scratch[__popc(rb & lt)] = v;
        __syncwarp();
        nb = __popc(rb);
    }
    // one value per id: drop ids of the pool and repeats (kept is sorted by
    // value, so the first copy of an id is its smallest bound)
    const uint32_t kid = (uint32_t)kept;
    bool drop = kept == EMPTY;
    for (uint32_t j = 0; j < K; j++) drop |= (__shfl_sync(FULL, pool_id, j) & ID_MASK) == kid;
    for (int j = 0; j < 31; j++) {
        const uint32_t o = __shfl_sync(FULL, kid, j);
        if (j < lane && o == kid) drop = true;
    }
    unsigned long long kv = drop ? EMPTY : (kept & 0xffffffff00000000ull) | 0xffffffffull;
    kv = fm_sort32(kv);
    const unsigned long long pw = lane < (int)K ? (((unsigned long long)pool_d << 32) | (uint32_t)lane) : EMPTY;
    const unsigned long long lo = fm_bitonic_merge32(min(pw, __shfl_sync(FULL, kv, 31 - lane)));
    return (uint32_t)(__shfl_sync(FULL, lo, K - 1) >> 32);
}

// One warp per target.  Proposals that pass the current K-th entry are
// collected in a 32-entry buffer; a full buffer (and the rest at the end)
// is sorted and merged into the pool, which lowers the K-th entry for the
// proposals still to come.
// Eight blocks (64 warps) per SM, registers capped at 32: the merge waits on
// scattered bucket and pool reads, and the added warps hide more of that
// latency -- the 1M build is 2.4 % faster than at the uncapped 48 registers.
// The kernel is bound by instruction fetch (the GPC instruction cache ran at
// 96 % of its request rate with the flush inlined twice), so the flush and
// the pool-side binary search each have a single inlined copy: 9 % off the
// 1M build.
// APPROX: proposals may carry the reduced-precision joins' d~ (APPROX_BIT);
// a first pass bounds the final K-th distance, the second buffers only the
// proposals whose lower bound d~ - err_c (|t|^2 + |u|^2) reaches it and
// computes their exact distances at the flush -- so the pool gets what the
// FP32 join's proposals would give it.
template <bool APPROX>
__global__ void __launch_bounds__(MERGE_WARPS * 32, 8) k_merge(MergeArgs a) {
    __shared__ MEnt sm[MERGE_WARPS][64];
    __shared__ MEnt kept[MERGE_WARPS][32];
    __shared__ MEnt buf[MERGE_WARPS][32];
    __shared__ uint8_t bufax[APPROX ? MERGE_WARPS : 1][32];
    if (a.ctr->overflow) return;
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t t = blockIdx.x * MERGE_WARPS + w;
    uint32_t nfl = 0;
    if (t < a.n) {
        const uint32_t K = a.K;
        const uint32_t c = a.bcnt[t];
        if (c) {
            uint32_t cd = 0xffffffffu, ce = 0;
            unsigned long long ck = ~0ull;
            if (lane < (int)K) {
                ce = a.pid[(size_t)t * K + lane];
                cd = __float_as_uint(a.pdist[(size_t)t * K + lane]);
                ck = (unsigned long long)lane;  // start entries precede every proposal of equal distance
            }
            uint32_t kd = __shfl_sync(FULL, cd, K - 1);
            unsigned long long kk = __shfl_sync(FULL, ck, K - 1);
            // the K-th distance the join filtered against: an approximate
            // proposal whose exact distance is not below it is one the FP32
            // join would not have made (a tie at the K-th distance)
            const uint32_t kd0 = kd;
            const unsigned long long b_first = a.boff[t];
            const unsigned lt = (1u << lane) - 1u;
            float nt = 0.f;
            uint32_t bound = 0xffffffffu;
            if (APPROX) {
                nt = __uint_as_float(a.nrm[t]);
                bound = approx_bound<false>(a, b_first, c, K, cd, ce, nt,
                                            reinterpret_cast<unsigned long long*>(&sm[w][0]));
            }
            uint32_t nb = 0;  // entries in buf
            uint32_t nrc = 0, nax = 0;  // rechecks, approximate proposals (count_approx)
            auto flush = [&]() {
                uint32_t pd = 0xffffffffu, pe = 0;
                unsigned long long pk = ~0ull;
                if (lane < (int)nb) {
                    const MEnt me = buf[w][lane];
                    pd = me.d;
                    pe = me.e;
                    pk = me.k;
                    if (APPROX && bufax[w][lane]) {
                        pd = __float_as_uint(merge_exact_l2(a.x, a.dp, t, pe & ID_MASK));
                        if (pd >= kd0) {
                            pd = 0xffffffffu;
                            pe = 0;
                            pk = ~0ull;
                        }
                    }
                }
                if (APPROX && a.count_approx) nrc += __popc(__ballot_sync(FULL, lane < (int)nb && bufax[w][lane]));
                __syncwarp();
                warp_sort_ment(pd, pk, pe);
                merge_round(pd, pk, pe, nb, K, cd, ce, ck, sm[w], kept[w]);
                kd = __shfl_sync(FULL, cd, K - 1);
                kk = __shfl_sync(FULL, ck, K - 1);
                nb = 0;
            };
            // One call site of flush (its sort and merge are long): a full
            // buffer flushes inside the loop, the last partial one after the
            // final chunk, at the same points of the proposal stream as
            // before.
            for (uint32_t b0 = 0;; b0 += 32) {
                uint32_t pd = 0xffffffffu, pe = 0;
                unsigned long long pk = ~0ull;
                bool rest = false, ax = false;
                float lb = 0.f;
                const bool last = b0 >= c;
                if (last) {
                    if (nb == 0) break;
                } else {
                    bool valid = false;
                    if (b0 + lane < c) {
                        const Prop p = reinterpret_cast<const Prop*>(a.bucket)[b_first + b0 + lane];
                        pd = __float_as_uint(p.dist);
                        pk = p.key;
                        pe = (p.idg & ID_MASK) | ((p.idg >> 31) << 30) | FLAG_BIT;
                        if (APPROX && (p.idg & APPROX_BIT)) {
                            ax = true;
                            lb = p.dist - a.err_c * (nt + __uint_as_float(a.nrm[p.idg & ID_MASK]));
                            valid = lb <= __uint_as_float(bound) && lb <= __uint_as_float(kd);
                        } else {
                            valid = mless(pd, pk, kd, kk);
                        }
                    }
                    if (APPROX && a.count_approx) nax += __popc(__ballot_sync(FULL, ax));
                    const unsigned vb = __ballot_sync(FULL, valid);
                    if (!vb) continue;
                    const uint32_t take = min((uint32_t)__popc(vb), 32u - nb);
                    const uint32_t rank = __popc(vb & lt);
                    if (valid && rank < take) {
                        buf[w][nb + rank] = MEnt{pd, pe, pk};
                        if (APPROX) bufax[w][nb + rank] = ax;
                    }
                    __syncwarp();
                    nb += take;
                    if (nb < 32) continue;
                    rest = valid && rank >= take;
                }
                flush();
                if (last) break;
                // the rest of this chunk, against the new K-th entry
                rest = rest && (ax ? lb <= __uint_as_float(kd) : mless(pd, pk, kd, kk));
                const unsigned rb = __ballot_sync(FULL, rest);
                if (rest) {
                    buf[w][__popc(rb & lt)] = MEnt{pd, pe, pk};
                    if (APPROX) bufax[w][__popc(rb & lt)] = ax;
                }
                __syncwarp();
                nb = __popc(rb);
            }
            if (lane < (int)K) {
                a.pid[(size_t)t * K + lane] = ce;
                a.pdist[(size_t)t * K + lane] = __uint_as_float(cd);
            }
            if (APPROX && a.count_approx && lane == 0 && nax) {
                atomicAdd(&a.ctr->approx_props, (unsigned long long)nax);
                atomicAdd(&a.ctr->rechecks, (unsigned long long)nrc);
            }
            nfl = __popc(__ballot_sync(FULL, lane < (int)K && (ce & FLAG_BIT)));
        }
        if (lane == 0) a.nflag[t] = (uint8_t)nfl;
    }
}

// The pool (sorted words in lanes < K, FM_EMPTY above) merged with a buffer
// of up to 32 proposal words (FM_EMPTY padded): the K smallest distinct
// entries of both.  `stage` is the warp's 64-word shared scratch.
__device__ __forceinline__ unsigned long long fm_flush(unsigned long long pool, unsigned long long buf, uint32_t K,
                                                       unsigned long long* stage) {
    const int lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;
    buf = fm_sort32(buf);
    const unsigned long long br = __shfl_sync(FULL, buf, 31 - lane);
    // lo: the 32 smallest words of both (a bitonic sequence), hi: the rest
    unsigned long long lo = min(pool, br), hi = max(pool, br);
    lo = fm_bitonic_merge32(lo);
    unsigned long long prev = __shfl_up_sync(FULL, lo, 1);
    const bool keep = lo != FM_EMPTY && (lane == 0 || (prev >> 2) != (lo >> 2));
    const unsigned m = __ballot_sync(FULL, keep);
    const uint32_t r = __popc(m & lt);
    if (keep && r < K) stage[r] = lo;
    uint32_t got = __popc(m);
    if (got < K) {  // copies among the 32 smallest: take entries of hi too
        hi = fm_bitonic_merge32(hi);
        const unsigned long long last_lo = __shfl_sync(FULL, lo, 31);
        prev = __shfl_up_sync(FULL, hi, 1);
        if (lane == 0) prev = last_lo;
        const bool keep2 = hi != FM_EMPTY && (prev >> 2) != (hi >> 2);
        const unsigned m2 = __ballot_sync(FULL, keep2);
        const uint32_t r2 = got + __popc(m2 & lt);
        if (keep2 && r2 < K) stage[r2] = hi;
        got += __popc(m2);
    }
    __syncwarp();
    const unsigned long long out = (lane < (int)K && (uint32_t)lane < got) ? stage[lane] : FM_EMPTY;
    __syncwarp();
    return out;
}

// One warp per target, as k_merge, on the fast tier's 8-byte proposals;
// APPROX as there.
template <bool APPROX>
__global__ void __launch_bounds__(MERGE_WARPS * 32, 8) k_merge_fast(MergeArgs a) {
    __shared__ unsigned long long buf[MERGE_WARPS][32];
    __shared__ unsigned long long stage[MERGE_WARPS][32];
    __shared__ uint8_t bufax[APPROX ? MERGE_WARPS : 1][32];
    if (a.ctr->overflow) return;
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t t = blockIdx.x * MERGE_WARPS + w;
    if (t >= a.n) return;
    const uint32_t K = a.K;
    const uint32_t c = a.bcnt[t];
    uint32_t nfl = 0;
    if (c) {
        unsigned long long pool = FM_EMPTY;
        if (lane < (int)K)
            pool = fm_word(__float_as_uint(a.pdist[(size_t)t * K + lane]), a.pid[(size_t)t * K + lane]);
        // the start pool in word order (entries of equal distance by id);
        // a pool the previous merge wrote is in that order already
        const unsigned long long pprev = __shfl_up_sync(FULL, pool, 1);
        if (!__all_sync(FULL, lane == 0 || pprev <= pool)) pool = fm_sort32(pool);
        unsigned long long kth = __shfl_sync(FULL, pool, K - 1);
        // the K-th distance the join filtered against (as in k_merge)
        const uint32_t kd0 = (uint32_t)(kth >> 32);
        const unsigned long long b_first = a.boff[t];
        const uint2* bp = reinterpret_cast<const uint2*>(a.bucket) + b_first;
        const unsigned lt = (1u << lane) - 1u;
        float nt = 0.f;
        uint32_t bound = 0xffffffffu;
        if (APPROX) {
            nt = __uint_as_float(a.nrm[t]);
            bound = approx_bound<true>(a, b_first, c, K, (uint32_t)(pool >> 32), (uint32_t)(pool >> 2), nt, stage[w]);
        }
        uint32_t nb = 0;
        uint32_t nrc = 0, nax = 0;  // rechecks, approximate proposals (count_approx)
        for (uint32_t b0 = 0;; b0 += 32) {
            unsigned long long v = FM_EMPTY;
            bool rest = false, ax = false;
            float lb = 0.f;
            const bool last = b0 >= c;
            if (last) {
                if (nb == 0) break;
            } else {
                bool valid = false;
                if (b0 + lane < c) {
                    const uint2 p = bp[b0 + lane];
                    // a new entry: flag 1, group bit from the list entry
                    v = ((unsigned long long)p.x << 32) | ((p.y & ID_MASK) << 2) | 2u | ((p.y >> 31) ^ 1u);
                    if (APPROX && (p.y & APPROX_BIT)) {
                        ax = true;
                        lb = __uint_as_float(p.x) - a.err_c * (nt + __uint_as_float(a.nrm[p.y & ID_MASK]));
                        valid = lb <= __uint_as_float(bound) && lb <= __uint_as_float((uint32_t)(kth >> 32));
                    } else {
                        valid = v < kth;
                    }
                }
                if (APPROX && a.count_approx) nax += __popc(__ballot_sync(FULL, ax));
                const unsigned vb = __ballot_sync(FULL, valid);
                if (!vb) continue;
                const uint32_t take = min((uint32_t)__popc(vb), 32u - nb);
                const uint32_t rank = __popc(vb & lt);
                if (valid && rank < take) {
                    buf[w][nb + rank] = v;
                    if (APPROX) bufax[w][nb + rank] = ax;
                }
                __syncwarp();
                nb += take;
                if (nb < 32) continue;
                rest = valid && rank >= take;
            }
            unsigned long long bv = FM_EMPTY;
            if (lane < (int)nb) {
                bv = buf[w][lane];
                if (APPROX && bufax[w][lane]) {  // the exact distance replaces d~
                    const uint32_t ex = __float_as_uint(merge_exact_l2(a.x, a.dp, t, (uint32_t)(bv >> 2) & ID_MASK));
                    bv = ex < kd0 ? ((unsigned long long)ex << 32) | (uint32_t)bv : FM_EMPTY;
                }
            }
            if (APPROX && a.count_approx) nrc += __popc(__ballot_sync(FULL, lane < (int)nb && bufax[w][lane]));
            __syncwarp();
            pool = fm_flush(pool, bv, K, stage[w]);
            kth = __shfl_sync(FULL, pool, K - 1);
            nb = 0;
            if (last) break;
            // the rest of this chunk, against the new K-th entry
            rest = rest && (ax ? lb <= __uint_as_float((uint32_t)(kth >> 32)) : v < kth);
            const unsigned rb = __ballot_sync(FULL, rest);
            if (rest) {
                buf[w][__popc(rb & lt)] = v;
                if (APPROX) bufax[w][__popc(rb & lt)] = ax;
            }
            __syncwarp();
            nb = __popc(rb);
        }
        if (lane < (int)K) {
            a.pid[(size_t)t * K + lane] = fm_pool_word(pool);
            a.pdist[(size_t)t * K + lane] = __uint_as_float((uint32_t)(pool >> 32));
        }
        if (APPROX && a.count_approx && lane == 0 && nax) {
            atomicAdd(&a.ctr->approx_props, (unsigned long long)nax);
            atomicAdd(&a.ctr->rechecks, (unsigned long long)nrc);
        }
        nfl = __popc(__ballot_sync(FULL, lane < (int)K && (pool & 2ull)));
    }
    if (lane == 0) a.nflag[t] = (uint8_t)nfl;
}

// Total of the per-row flag counts (the warps of k_merge finish unevenly, so
// they do not meet at a block barrier to add them up).
__global__ void k_sum_flags(const uint8_t* nflag, uint32_t n, IterCounters* ctr) {
    __shared__ unsigned int part[8];
    if (ctr->overflow) return;
    unsigned int s = 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) s += nflag[i];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(FULL, s, o);
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned int b = 0;
        for (int w = 0; w < 8; w++) b += part[w];
        if (b) atomicAdd(&ctr->flags, (unsigned long long)b);
    }
}

// ---------------------------------------------------------------------------
// Sets `bit` of the overflow word when *total exceeds cap.
__global__ void k_check_cap(IterCounters* ctr, const unsigned long long* total, unsigned long long cap,
                            unsigned int bit) {
    if (threadIdx.x == 0 && *total > cap) atomicOr(&ctr->overflow, bit);
}

__global__ void k_clear_lists(uint32_t* newlen, uint32_t* oldlen, uint32_t* tn, uint32_t* to, uint32_t n) {
    uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    newlen[t] = 0;
    oldlen[t] = 0;
    if (tn) {
        tn[t] = 0;
        to[t] = 0;
    }
}

__global__ void k_set_u32(uint32_t* dst, const uint32_t* src, uint32_t n) {
    uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) dst[t] = src ? src[t] : 0u;
}

template <typename T> T* P(DevBuf& b) { return b.as<T>(); }

}  // namespace

int graph_alloc(Ctx& ctx, GraphStore& s, GraphDev& g, bool with_carry) {
    const size_t nk = (size_t)g.n_cap * g.K;
    NNM_CUDA_TRY(s.pid.ensure(nk * 4));
    NNM_CUDA_TRY(s.pdist.ensure(nk * 4));
    NNM_CUDA_TRY(s.cpid.ensure(nk * 4));
    NNM_CUDA_TRY(s.cpdist.ensure(nk * 4));
    g.capn = g.capo = (g.K + g.smpl) * (with_carry ? 2 : 1);
    NNM_CUDA_TRY(s.newL.ensure((size_t)g.n_cap * g.capn * 4));
    NNM_CUDA_TRY(s.oldL.ensure((size_t)g.n_cap * g.capo * 4));
    NNM_CUDA_TRY(s.newlen.ensure((size_t)g.n_cap * 4));
    NNM_CUDA_TRY(s.oldlen.ensure((size_t)g.n_cap * 4));
    NNM_CUDA_TRY(cudaMemsetAsync(s.newlen.p, 0, (size_t)g.n_cap * 4, ctx.stream));
    NNM_CUDA_TRY(cudaMemsetAsync(s.oldlen.p, 0, (size_t)g.n_cap * 4, ctx.stream));
    g.pid = s.pid.as<uint32_t>();
    g.pdist = s.pdist.as<float>();
    g.cpid = s.cpid.as<uint32_t>();
    g.cpdist = s.cpdist.as<float>();
    g.newL = s.newL.as<uint32_t>();
    g.oldL = s.oldL.as<uint32_t>();
    g.newlen = s.newlen.as<uint32_t>();
    g.oldlen = s.oldlen.as<uint32_t>();
    g.rnewT = g.roldT = g.rnewTlen = g.roldTlen = nullptr;
    if (with_carry) {
        NNM_CUDA_TRY(s.rnewT.ensure((size_t)g.n_cap * g.smpl * 4));
        NNM_CUDA_TRY(s.roldT.ensure((size_t)g.n_cap * g.smpl * 4));
        NNM_CUDA_TRY(s.rnewTlen.ensure((size_t)g.n_cap * 4));
        NNM_CUDA_TRY(s.roldTlen.ensure((size_t)g.n_cap * 4));
        NNM_CUDA_TRY(cudaMemsetAsync(s.rnewTlen.p, 0, (size_t)g.n_cap * 4, ctx.stream));
        NNM_CUDA_TRY(cudaMemsetAsync(s.roldTlen.p, 0, (size_t)g.n_cap * 4, ctx.stream));
        g.rnewT = s.rnewT.as<uint32_t>();
        g.roldT = s.roldT.as<uint32_t>();
        g.rnewTlen = s.rnewTlen.as<uint32_t>();
        g.roldTlen = s.roldTlen.as<uint32_t>();
    }
    g.carry = false;
    return 0;
}

// Shared memory of a k_pairs block: member arrays (16 B per list slot) and,
// for the staged tiers, the swizzled vectors.
static size_t pairs_smem(uint32_t R, uint32_t dp, bool staged) {
    const uint32_t vstride = vec_stride(dp / 4);
    return (size_t)R * 16 + (staged ? ((size_t)R * vstride + R / 4 + 1) * 16 : 0) + 64;
}

// k_pairs_u8: the member arrays, the norms, then kq bytes a row.
static size_t pairs_smem_u8(uint32_t R, uint32_t kq) {
    const uint32_t vstride = vec_stride(kq / 16);
    return (size_t)R * 16 + (size_t)((R + 3) & ~3u) * 4 + ((size_t)R * vstride + R / 4 + 1) * 16 + 64;
}

// Highest list-size tier whose staged vectors fit in a CTA's shared memory
// at this dimension (3: all; lower at large d, -1 for none -- those rows
// take the unstaged kernel of the last tier, with the same sums).
static int max_staged_tier(uint32_t dp, int device) {
    int optin = 0;
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
    int t = 0;
    while (t < NTIER - 1 && pairs_smem(TIER_CAP[t], dp, true) <= (size_t)optin) t++;
    return t - 1;
}

template <int M>
static cudaError_t prep_pairs(uint32_t caps, uint32_t dp, size_t emit_smem, int max_staged) {
    cudaError_t e;
    if (max_staged >= 0 && (e = cudaFuncSetAttribute(k_pairs<M, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                     (int)pairs_smem(TIER_CAP[0], dp, true))) != cudaSuccess) return e;
    if (max_staged >= 1 && (e = cudaFuncSetAttribute(k_pairs<M, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                     (int)pairs_smem(TIER_CAP[1], dp, true))) != cudaSuccess) return e;
    if (max_staged >= 2 && (e = cudaFuncSetAttribute(k_pairs<M, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                     (int)pairs_smem(TIER_CAP[2], dp, true))) != cudaSuccess) return e;
    if (max_staged >= 3 && (e = cudaFuncSetAttribute(k_pairs<M, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                     (int)pairs_smem(TIER_CAP[3], dp, true))) != cudaSuccess) return e;
    if ((e = cudaFuncSetAttribute(k_pairs<M, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)pairs_smem(caps, dp, false))) != cudaSuccess) return e;
    if ((e = cudaFuncSetAttribute(k_emit_rows, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(caps * 24 + 64))) !=
        cudaSuccess)
        return e;
    return cudaFuncSetAttribute(k_emit, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)emit_smem);
}

// FP32 pair kernels: all tiers, or only the last one when the tensor-core
// join takes the others.
template <int M>
static void launch_pairs(const JoinArgs& ja, const unsigned* ntier, uint32_t caps, uint32_t dp, int nsm,
                         bool last_only, bool u8_last, bool u8_tc, cudaStream_t st) {
    if (!last_only && ntier) {
        if (ntier[0]) { k_pairs<M, 0><<<ntier[0], TIER_THREADS[0], pairs_smem(TIER_CAP[0], dp, true), st>>>(ja, TIER_CAP[0]); count_launch(); }
        if (ntier[1]) { k_pairs<M, 1><<<ntier[1], TIER_THREADS[1], pairs_smem(TIER_CAP[1], dp, true), st>>>(ja, TIER_CAP[1]); count_launch(); }
        if (ntier[2]) { k_pairs<M, 2><<<ntier[2], TIER_THREADS[2], pairs_smem(TIER_CAP[2], dp, true), st>>>(ja, TIER_CAP[2]); count_launch(); }
        if (ntier[3]) { k_pairs<M, 3><<<ntier[3], TIER_THREADS[3], pairs_smem(TIER_CAP[3], dp, true), st>>>(ja, TIER_CAP[3]); count_launch(); }
    }
    // ntier null (the tensor-core join takes tiers 0-3): the count of the
    // last tier is on the device only, the blocks loop over its rows; the
    // grid is every block that fits on the SMs at once
    if (u8_tc) {  // the last tier on the tensor cores
        launch_pairs_tc(ja, caps, ntier, nsm, st);
        return;
    }
    if (!ntier || ntier[4]) {
        const size_t smem = u8_last ? pairs_smem_u8(caps, ja.kq) : pairs_smem(caps, dp, false);
        int per_sm = 0;
        if (u8_last)
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pairs_u8, TIER_THREADS[4], smem);
        else
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pairs<M, 4>, TIER_THREADS[4], smem);
        const unsigned full = (unsigned)nsm * (unsigned)std::max(per_sm, 1);
        const unsigned g = ntier ? std::min<unsigned>(ntier[4], full) : full;
        if (u8_last) {
            k_pairs_u8<<<g, TIER_THREADS[4], smem, st>>>(ja, caps);
        } else {
            k_pairs<M, 4><<<g, TIER_THREADS[4], smem, st>>>(ja, caps);
        }
        count_launch();
    }
}

// Grid of k_emit_rows when the row count is on the device only: every
// block that fits on the SMs at once.
static unsigned emit_rows_grid(uint32_t caps, int nsm) {
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_emit_rows, EMIT_ROW_WARPS * 32, (size_t)caps * 24 + 64);
    return (unsigned)nsm * (unsigned)std::max(per_sm, 1);
}

// Sequential float mean of the per-row deltas, as the reference computes it
// with a Boost float accumulator (EvaluateDelta: float(c)/K per row).
static float host_mean(const std::vector<uint8_t>& nflag, uint32_t n, uint32_t K) {
    volatile float sum = 0.f;
    for (uint32_t i = 0; i < n; i++) sum = sum + (float)nflag[i] / (float)K;
    return sum / (float)n;
}

int run_nndescent(Ctx& ctx, GraphDev& g, JoinMode mode, uint32_t split, uint32_t verse,
                  const uint32_t* d_leaf_off, uint32_t nleaf) {
    Workspace& ws = ctx.ws;
    cudaStream_t st = ctx.stream;
    const uint32_t n = g.n, K = g.K;
    const size_t n1 = (size_t)n + 1;
    const bool track = g.rnewT != nullptr;
    const size_t rev_cap = (size_t)n * K + (track ? (size_t)n * g.smpl : 0);
    const uint32_t caps = g.capn + g.capo;
    int nsm = 148;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, ctx.device);

    NNM_CUDA_TRY(ws.rcnt.ensure(n1 * 2 * 4));
    NNM_CUDA_TRY(ws.rcur.ensure(n1 * 2 * 4));
    NNM_CUDA_TRY(ws.roff.ensure(n1 * 2 * 8));
    NNM_CUDA_TRY(ws.rseg.ensure(rev_cap * 2 * 4));
    NNM_CUDA_TRY(ws.rscr.ensure(rev_cap * 2 * 4));
    NNM_CUDA_TRY(ws.rcount.ensure(n1 * 4));
    NNM_CUDA_TRY(ws.rofs.ensure(n1 * 8));
    NNM_CUDA_TRY(ws.rbuf.ensure(rev_cap * 2 * 4 + 64));
    NNM_CUDA_TRY(ws.cntpos.ensure((size_t)n * caps * 2));
    NNM_CUDA_TRY(ws.bcnt.ensure(n1 * 4));
    NNM_CUDA_TRY(ws.bcur.ensure(n1 * 4));
    NNM_CUDA_TRY(ws.boff.ensure(n1 * 8));
    NNM_CUDA_TRY(ws.bigrev.ensure(n1 * 2 * 4));
    NNM_CUDA_TRY(ws.nflag.ensure(n1));
    NNM_CUDA_TRY(ws.kth.ensure(n1 * 4));
    NNM_CUDA_TRY(ws.rtier.ensure(n1));
    NNM_CUDA_TRY(ws.scan_tmp.ensure((scan_temp_elems(n1) + 8) * 8));
    NNM_CUDA_TRY(ws.counters.ensure(sizeof(IterCounters) + 64));
    const size_t prop_bytes = g.fast ? sizeof(Prop8) : sizeof(Prop);  // the tier's proposal format
    if (ws.bucket.bytes < (size_t)n * K * 4 * prop_bytes) NNM_CUDA_TRY(ws.bucket.ensure((size_t)n * K * 4 * prop_bytes));

    uint32_t *rcnt_new = P<uint32_t>(ws.rcnt), *rcnt_old = rcnt_new + n1;
    uint32_t *rcur_new = P<uint32_t>(ws.rcur), *rcur_old = rcur_new + n1;
    uint64_t *roff_new = P<uint64_t>(ws.roff), *roff_old = roff_new + n1;
    uint32_t *rseg_new = P<uint32_t>(ws.rseg), *rseg_old = rseg_new + rev_cap;
    uint32_t *rscr_new = P<uint32_t>(ws.rscr), *rscr_old = rscr_new + rev_cap;
    uint64_t* scan_tmp = P<uint64_t>(ws.scan_tmp);
    uint64_t* d_tot = P<uint64_t>(ws.scan_tmp) + scan_temp_elems(n1) + 4;  // past the scan scratch
    IterCounters* ctr = P<IterCounters>(ws.counters);

    const size_t emit_smem = (size_t)EMIT_WARPS * caps * 24 + 64;
    const int max_staged = max_staged_tier(g.dp, ctx.device);
    cudaError_t ae = g.metric == L2 ? prep_pairs<L2>(caps, g.dp, emit_smem, max_staged)
                     : g.metric == L1 ? prep_pairs<L1>(caps, g.dp, emit_smem, max_staged)
                                      : prep_pairs<CHI2>(caps, g.dp, emit_smem, max_staged);
    NNM_CUDA_TRY(ae);
    NNM_CUDA_TRY(ws.npairs.ensure(n1 * 4));
    NNM_CUDA_TRY(ws.poff.ensure(n1 * 8));
    NNM_CUDA_TRY(ws.tiers.ensure((size_t)n * NTIER * 4 + 16));
    const bool tc = g.xq != nullptr;
    // reduced-precision joins (BF16, FP8) emit approximate distances
    const bool approx = tc && g.tc_kind != 0;
    bool u8_last = false;  // rows of S > 128 on the u8 vectors (staged vectors fit)
    bool u8_tc = false;    // ... on the tensor cores (k_pairs_tc), else k_pairs_u8
    if (tc) {
        NNM_CUDA_TRY(tc_set_attributes(g.kq, g.tc_kind));
        NNM_CUDA_TRY(ws.erows.ensure((size_t)n * 4 * 4 + 16));
        int optin = 0;
        NNM_CUDA_TRY(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, ctx.device));
        const size_t u8_smem = pairs_smem_u8(caps, g.kq);
        u8_last = g.tc_kind == 0 && g.metric == L2 && u8_smem <= (size_t)optin;
        if (u8_last)
            NNM_CUDA_TRY(cudaFuncSetAttribute(k_pairs_u8, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)u8_smem));
        u8_tc = u8_last && pairs_tc_smem(caps, g.kq) <= (size_t)optin;
        if (u8_tc) NNM_CUDA_TRY(pairs_tc_set_attributes(caps, g.kq));
    }

    const unsigned warp_blocks = (unsigned)((n + 7) / 8);
    const unsigned tblocks = (unsigned)((n + 255) / 256);
    std::vector<uint8_t> h_nflag;

    // Fast tier: an iteration's sampling segment -- list clears through the
    // pair-count scan and the counter read-back -- launches the same kernels
    // with the same arguments in every iteration but the first of a carried
    // H-Merge level, except the draw phase of k_shuffle_append.  It is
    // captured once per call as a CUDA graph and replayed, the phase set on
    // the instantiated graph's node before each replay.  (The join and the
    // merge follow host reads of tile, pair and proposal counts.)
    struct SegGraph {
        cudaGraph_t graph = nullptr;  // kept while exec lives: its node handle names the node to update
        cudaGraphExec_t exec = nullptr;
        cudaGraphNode_t shuf = nullptr;
        cudaKernelNodeParams kp{};
        uint64_t launches = 0;
        bool disabled = false;
        ~SegGraph() {
            if (exec) cudaGraphExecDestroy(exec);
            if (graph) cudaGraphDestroy(graph);
        }
    } seg;
    // The whole-iteration graph of the fast tier on the tensor cores: the
    // context's executable graph of this join mode, once it holds this
    // call's iteration (owned by the context).
    struct {
        cudaGraphExec_t exec = nullptr;
        bool disabled = false;
    } whole_g;
    // the draw phase of the replays: a device word past the counters and its
    // pinned host source past the host counters
    uint32_t* phase_dev = reinterpret_cast<uint32_t*>(ctr + 1);
    uint32_t* h_phase = reinterpret_cast<uint32_t*>(ctx.h_counters + 1);
    // the node of kernel `fn` in a captured graph, and its parameters
    auto find_kernel_node = [](cudaGraph_t graph, void* fn, cudaKernelNodeParams& out) -> cudaGraphNode_t {
        size_t nn = 0;
        cudaGraphGetNodes(graph, nullptr, &nn);
        std::vector<cudaGraphNode_t> nodes(nn);
        cudaGraphGetNodes(graph, nodes.data(), &nn);
        for (cudaGraphNode_t nd : nodes) {
            cudaGraphNodeType ty;
            cudaKernelNodeParams kp{};
            if (cudaGraphNodeGetType(nd, &ty) == cudaSuccess && ty == cudaGraphNodeTypeKernel &&
                cudaGraphKernelNodeGetParams(nd, &kp) == cudaSuccess && kp.func == fn) {
                out = kp;
                return nd;
            }
        }
        return nullptr;
    };
    for (uint32_t it = 0;; it++) {
        const bool carry_now = (it == 0) && g.carry && track;
        const uint32_t phase = g.phase++;
        auto shuf_args = [&]() {
            return ShufArgs{roff_new, roff_old, rseg_new, rseg_old, P<uint64_t>(ws.rofs), P<int32_t>(ws.rbuf),
                            g.newL, g.oldL, g.newlen, g.oldlen,
                            g.capn, g.capo, n, g.smpl,
                            track ? g.rnewT : nullptr, track ? g.roldT : nullptr,
                            track ? g.rnewTlen : nullptr, track ? g.roldTlen : nullptr,
                            P<uint32_t>(ws.npairs), ctr, g.fast ? 1u : 0u, g.seed, phase,
                            tc ? (g.tc_kind == 0 ? g.tile_rows : TC_MAX_S) : 0u, max_staged, rscr_new, rscr_old,
                            (g.fast && carry_now) ? 1u : 0u, nullptr, P<uint8_t>(ws.rtier)};
        };
        // the segment; its first failing call's error is returned.  copy:
        // read the counters back at its end (the whole-iteration graph reads
        // them once, after the merge)
        auto seg_a = [&](bool copy = true, const uint32_t* phase_dev = nullptr) -> cudaError_t {
            cudaError_t e = cudaSuccess;
            auto chk = [&](cudaError_t x) {
                if (e == cudaSuccess) e = x;
            };
            if (!carry_now) {
                k_clear_lists<<<tblocks, 256, 0, st>>>(g.newlen, g.oldlen,
                                                       track ? g.rnewTlen : nullptr,
                                                       track ? g.roldTlen : nullptr, n); count_launch();
            }
            chk(cudaMemsetAsync(ctr, 0, sizeof(IterCounters), st));
            // reverse counts and cursors start at the carried lengths
            k_set_u32<<<tblocks, 256, 0, st>>>(rcnt_new, track ? g.rnewTlen : nullptr, n); count_launch();
            k_set_u32<<<tblocks, 256, 0, st>>>(rcnt_old, track ? g.roldTlen : nullptr, n); count_launch();
            k_set_u32<<<tblocks, 256, 0, st>>>(rcur_new, track ? g.rnewTlen : nullptr, n); count_launch();
            k_set_u32<<<tblocks, 256, 0, st>>>(rcur_old, track ? g.roldTlen : nullptr, n); count_launch();
            SampleArgs sa{g.pid, g.pdist, n, K, (uint32_t)mode, split,
                          rcnt_new, rcnt_old, rcur_new, rcur_old, roff_new, roff_old, rseg_new, rseg_old,
                          g.newL, g.oldL, g.newlen, g.oldlen,
                          g.capn, g.capo,
                          carry_now ? g.rnewT : nullptr, carry_now ? g.roldT : nullptr,
                          carry_now ? g.rnewTlen : nullptr, carry_now ? g.roldTlen : nullptr,
                          g.smpl, ctr, P<float>(ws.kth)};
            k_kth_gather<<<tblocks, 256, 0, st>>>(g.pdist, K, n, P<float>(ws.kth)); count_launch();
            k_sample_count<<<warp_blocks, 256, 0, st>>>(sa); count_launch();
            chk(exclusive_scan(rcnt_new, roff_new, n, scan_tmp, nullptr, st));
            chk(exclusive_scan(rcnt_old, roff_old, n, scan_tmp, nullptr, st));
            k_sample_fill<<<warp_blocks, 256, 0, st>>>(sa); count_launch();
            RevSortArgs ra{{roff_new, roff_old}, {rseg_new, rseg_old}, {rscr_new, rscr_old},
                           {carry_now ? g.rnewTlen : nullptr, carry_now ? g.roldTlen : nullptr},
                           n, P<uint32_t>(ws.bigrev), ctr};
            // reverse lists in ascending source order, as the reference pushes
            // them; the fast tier keeps them in the (arbitrary) order the atomics
            // left: its samples and tie-break keys do not depend on list order
            if (!g.fast) {
                k_rev_sort_small<<<dim3(warp_blocks, 2), 256, 0, st>>>(ra); count_launch();
                k_rev_sort_big<<<nsm * 2, 512, 0, st>>>(ra); count_launch();
                // std::rand() draws of this iteration's shuffles
                k_rand_count<<<tblocks, 256, 0, st>>>(roff_new, roff_old, n, P<uint32_t>(ws.rcount)); count_launch();
                chk(exclusive_scan(P<uint32_t>(ws.rcount), P<uint64_t>(ws.rofs), n, scan_tmp, d_tot, st));
                chk(glibc_stream_generate(P<int32_t>(ws.rbuf), g.gbase, g.gpos, d_tot, rev_cap * 2, st));
            } else {
                chk(cudaMemsetAsync(d_tot, 0, 8, st));
            }
            ShufArgs sh = shuf_args();
            sh.phase_dev = phase_dev;
            k_shuffle_append<<<warp_blocks, 256, 0, st>>>(sh); count_launch();
            k_tier_lists<<<(n + TIER_CHUNK - 1) / TIER_CHUNK, 256, 0, st>>>(P<uint8_t>(ws.rtier), n,
                                                                           P<uint32_t>(ws.tiers), ctr); count_launch();
            chk(exclusive_scan(P<uint32_t>(ws.npairs), P<uint64_t>(ws.poff), n, scan_tmp,
                               reinterpret_cast<uint64_t*>(&ctr->pairs), st));
            chk(cudaMemsetAsync(ws.bcnt.p, 0, n1 * 4, st));
            chk(cudaMemsetAsync(ws.bcur.p, 0, n1 * 4, st));
            if (copy) chk(cudaMemcpyAsync(ctx.h_counters, ctr, sizeof(IterCounters), cudaMemcpyDeviceToHost, st));
            chk(cudaGetLastError());
            return e;
        };
        // Event records inside a capture become graph nodes (external events)
        // so that the profile reads the replayed kernels' times.
        auto rec = [&](int i) {
            if (!ctx.prof) return;
            cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
            cudaStreamIsCapturing(st, &cs);
            if (cs == cudaStreamCaptureStatusActive) cudaEventRecordWithFlags(ctx.ev[i], st, cudaEventRecordExternal);
            else cudaEventRecord(ctx.ev[i], st);
        };
        auto make_ja = [&]() {
            return JoinArgs{g.x, g.dp, K, n, g.pdist, g.newL, g.oldL, g.newlen, g.oldlen, g.capn, g.capo, caps,
                            (uint32_t)mode, verse, d_leaf_off, nleaf, P<uint32_t>(ws.tiers), P<uint64_t>(ws.poff),
                            P<float>(ws.pd), P<uint16_t>(ws.cntpos), P<uint32_t>(ws.bcnt), P<uint32_t>(ws.bcur),
                            P<uint64_t>(ws.boff), ws.bucket.p, ctr,
                            g.xq, g.nrm, g.kq, tc ? 1u : 0u, &ctr->error, tc ? P<uint32_t>(ws.erows) : nullptr,
                            g.fast ? 1u : 0u, g.tc_kind, g.err_c, g.scl, g.audit ? 1u : 0u, P<float>(ws.kth)};
        };
        // local join, pass 1: per-target proposal counts (and, on the FP32
        // path, the stored pair distances), then the bucket offsets.  nt:
        // rows per tier read by the host, or null (grids of every SM; the
        // kernels read the counts on the device).
        auto part0 = [&](const JoinArgs& ja, const unsigned* nt) -> cudaError_t {
            cudaError_t e = cudaSuccess;
            rec(0);
            if (tc) e = launch_join_tc(0, ja, nt, nsm, st);
            if (e == cudaSuccess) {
                if (g.metric == L2) launch_pairs<L2>(ja, nt, caps, g.dp, nsm, tc, u8_last, u8_tc, st);
                else if (g.metric == L1) launch_pairs<L1>(ja, nt, caps, g.dp, nsm, tc, false, false, st);
                else launch_pairs<CHI2>(ja, nt, caps, g.dp, nsm, tc, false, false, st);
                rec(1);
                e = exclusive_scan(P<uint32_t>(ws.bcnt), P<uint64_t>(ws.boff), n, scan_tmp,
                                   reinterpret_cast<uint64_t*>(&ctr->proposals), st);
            }
            return e != cudaSuccess ? e : cudaGetLastError();
        };
        // pass 2: proposals, recomputed on the tensor cores or read from the
        // stored distances; the top-K merge and the flag total
        auto part1 = [&](const JoinArgs& ja, const unsigned* nt) -> cudaError_t {
            cudaError_t e = cudaSuccess;
            rec(2);
            if (tc) e = launch_join_tc(1, ja, nt, nsm, st);
            if (e != cudaSuccess) return e;
            if (tc) {
                const unsigned rows4 = nt ? nt[NTIER - 1] : emit_rows_grid(caps, nsm);
                if (rows4) {
                    k_emit_rows<<<rows4, EMIT_ROW_WARPS * 32, (size_t)caps * 24 + 64, st>>>(ja); count_launch();
                }
            } else if (n > 0) {
                k_emit<<<(n + EMIT_WARPS - 1) / EMIT_WARPS, EMIT_WARPS * 32, emit_smem, st>>>(ja); count_launch();
            }
            MergeArgs ma{g.pid, g.pdist, n, K, P<uint32_t>(ws.bcnt), P<uint64_t>(ws.boff),
                         ja.bucket, P<uint8_t>(ws.nflag), ctr, g.x, g.dp, g.nrm, g.err_c, ctx.prof ? 1u : 0u};
            rec(3);
            const unsigned mgrid = (n + MERGE_WARPS - 1) / MERGE_WARPS;
            if (g.fast) {
                if (approx) k_merge_fast<true><<<mgrid, MERGE_WARPS * 32, 0, st>>>(ma);
                else k_merge_fast<false><<<mgrid, MERGE_WARPS * 32, 0, st>>>(ma);
            } else {
                if (approx) k_merge<true><<<mgrid, MERGE_WARPS * 32, 0, st>>>(ma);
                else k_merge<false><<<mgrid, MERGE_WARPS * 32, 0, st>>>(ma);
            }
            count_launch();
            k_sum_flags<<<std::min<unsigned>((n + 255) / 256, (unsigned)nsm * 4), 256, 0, st>>>(P<uint8_t>(ws.nflag), n, ctr); count_launch();
            rec(4);
            return cudaGetLastError();
        };
        auto copy_back = [&]() -> cudaError_t {
            cudaError_t e = cudaMemcpyAsync(ctx.h_counters, ctr, sizeof(IterCounters), cudaMemcpyDeviceToHost, st);
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(&ctx.h_counters->rand_draws, d_tot, 8, cudaMemcpyDeviceToHost, st);
            return e;
        };
        // Fast tier on the tensor cores, after the first iteration of the
        // call has sized the pair and bucket buffers: the whole iteration --
        // sampling, both join passes, merge, counters -- is one CUDA graph,
        // replayed with the draw phase set on its shuffle node, and the host
        // reads the counters once.  The buffers are sized from earlier
        // iterations (with headroom) and checked on the device; on overflow
        // the join and merge kernels do nothing, and the host grows the
        // buffer and reruns the skipped part directly.
        const bool whole = g.fast && tc && !carry_now && !whole_g.disabled && !g.no_graph && it > 0;
        bool done = false;
        if (whole) {
            // The graph is captured at the call's first whole iteration and
            // applied to the context's executable graph of this join mode
            // (cudaGraphExecUpdate: no new instantiation while the shape of
            // the iteration is the same); the draw phase is read from a
            // device word, written before each replay.
            Ctx::IterGraph& ig = ctx.iter_graph[(int)mode & 3];
            if (!whole_g.exec) {
                const uint64_t c0 = launch_counter().load();
                cudaGraph_t graph = nullptr;
                cudaError_t e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
                if (e == cudaSuccess) {
                    const JoinArgs ja = make_ja();
                    cudaError_t e1 = seg_a(false, phase_dev);
                    if (e1 == cudaSuccess) {
                        k_check_cap<<<1, 32, 0, st>>>(ctr, reinterpret_cast<const unsigned long long*>(&ctr->pairs),
                                                      (unsigned long long)(ws.pd.bytes / 4), OVF_PAIRS); count_launch();
                        e1 = part0(ja, nullptr);
                    }
                    if (e1 == cudaSuccess) {
                        k_check_cap<<<1, 32, 0, st>>>(ctr, reinterpret_cast<const unsigned long long*>(&ctr->proposals),
                                                      (unsigned long long)(ws.bucket.bytes / prop_bytes),
                                                      OVF_PROPOSALS); count_launch();
                        e1 = part1(ja, nullptr);
                    }
                    if (e1 == cudaSuccess) e1 = copy_back();
                    const cudaError_t e2 = cudaStreamEndCapture(st, &graph);
                    e = e1 != cudaSuccess ? e1 : e2;
                }
                if (e == cudaSuccess && ig.exec) {
                    cudaGraphExecUpdateResultInfo info;
                    if (cudaGraphExecUpdate(ig.exec, graph, &info) != cudaSuccess) {
                        cudaGetLastError();
                        cudaGraphExecDestroy(ig.exec);
                        ig.exec = nullptr;
                    }
                }
                if (e == cudaSuccess && !ig.exec) e = cudaGraphInstantiate(&ig.exec, graph, 0);
                if (graph) cudaGraphDestroy(graph);
                ig.launches = launch_counter().load() - c0;
                if (e != cudaSuccess) {  // no graph: this call launches directly
                    cudaGetLastError();
                    if (ig.exec) cudaGraphExecDestroy(ig.exec);
                    ig.exec = nullptr;
                    whole_g.disabled = true;
                } else {
                    whole_g.exec = ig.exec;
                }
            } else {
                count_launch(ig.launches);
            }
            if (whole_g.exec) {
                *h_phase = phase;  // pinned; the copy is enqueued before the replay
                NNM_CUDA_TRY(cudaMemcpyAsync(phase_dev, h_phase, 4, cudaMemcpyHostToDevice, st));
                NNM_CUDA_TRY(cudaGraphLaunch(whole_g.exec, st));
                NNM_CUDA_TRY(cudaStreamSynchronize(st));
                IterCounters& h = *ctx.h_counters;
                if (h.error) {
                    ctx.last_error = "device capacity check failed (code " + std::to_string(h.error) + ")";
                    return 6;
                }
                if (h.overflow) {
                    // grow what was short (the graph names the old buffers:
                    // it is captured again next iteration) and rerun what the
                    // kernels skipped
                    whole_g.exec = nullptr;
                    unsigned nt[NTIER];
                    for (int t = 0; t < NTIER; t++) nt[t] = h.ntier[t];
                    const unsigned ovf = h.overflow;
                    NNM_CUDA_TRY(cudaMemsetAsync(&ctr->overflow, 0, 4, st));
                    if (ovf & OVF_PAIRS) {
                        NNM_CUDA_TRY(ws.pd.ensure((size_t)(std::max<uint64_t>(h.pairs, 1) * 1.5 + 1024) * 4));
                        NNM_CUDA_TRY(part0(make_ja(), nt));
                        NNM_CUDA_TRY(cudaMemcpyAsync(ctx.h_counters, ctr, sizeof(IterCounters), cudaMemcpyDeviceToHost, st));
                        NNM_CUDA_TRY(cudaStreamSynchronize(st));
                    }
                    const uint64_t nprop = ctx.h_counters->proposals;
                    if (nprop * prop_bytes > ws.bucket.bytes)
                        NNM_CUDA_TRY(ws.bucket.ensure((size_t)(nprop * 1.5 + 1024) * prop_bytes));
                    NNM_CUDA_TRY(part1(make_ja(), nt));
                    NNM_CUDA_TRY(copy_back());
                    NNM_CUDA_TRY(cudaStreamSynchronize(st));
                }
                done = true;
            }
        }
        if (!done) {
            const bool graphable = g.fast && !carry_now && !seg.disabled && !tc && !g.no_graph;
            if (graphable && seg.exec) {
                ShufArgs sh = shuf_args();
                void* kargs[] = {&sh};
                cudaKernelNodeParams kp = seg.kp;
                kp.kernelParams = kargs;
                kp.extra = nullptr;
                cudaError_t e = cudaGraphExecKernelNodeSetParams(seg.exec, seg.shuf, &kp);
                if (e == cudaSuccess) e = cudaGraphLaunch(seg.exec, st);
                NNM_CUDA_TRY(e);
                count_launch(seg.launches);
            } else if (graphable) {
                const uint64_t c0 = launch_counter().load();
                cudaGraph_t& graph = seg.graph;
                cudaError_t e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
                if (e == cudaSuccess) {
                    const cudaError_t e1 = seg_a();
                    const cudaError_t e2 = cudaStreamEndCapture(st, &graph);
                    e = e1 != cudaSuccess ? e1 : e2;
                }
                if (e == cudaSuccess) e = cudaGraphInstantiate(&seg.exec, graph, 0);
                if (e == cudaSuccess) seg.shuf = find_kernel_node(graph, reinterpret_cast<void*>(k_shuffle_append), seg.kp);
                seg.launches = launch_counter().load() - c0;
                if (e == cudaSuccess && seg.shuf) e = cudaGraphLaunch(seg.exec, st);  // capture counted its kernels
                if (e != cudaSuccess || !seg.shuf) {
                    // no graph: this call launches the segment directly
                    cudaGetLastError();
                    if (seg.exec) cudaGraphExecDestroy(seg.exec);
                    if (seg.graph) cudaGraphDestroy(seg.graph);
                    seg.exec = nullptr;
                    seg.graph = nullptr;
                    seg.disabled = true;
                    NNM_CUDA_TRY(seg_a());
                }
            } else {
                NNM_CUDA_TRY(seg_a());
            }
            NNM_CUDA_TRY(cudaStreamSynchronize(st));
            if (ctx.h_counters->error) {
                ctx.last_error = "device capacity check failed (code " + std::to_string(ctx.h_counters->error) + ")";
                return 6;
            }
            unsigned ntier[NTIER];
            for (int t = 0; t < NTIER; t++) ntier[t] = ctx.h_counters->ntier[t];
            // headroom for the iterations the whole-iteration graph runs
            const double room = (g.fast && tc) ? 1.5 : 1.0;
            const size_t pd_need = (size_t)(std::max<uint64_t>(ctx.h_counters->pairs, 1) * room) * 4;
            if (pd_need > ws.pd.bytes) NNM_CUDA_TRY(ws.pd.ensure(pd_need + 4096));
            JoinArgs ja = make_ja();
            NNM_CUDA_TRY(part0(ja, ntier));
            NNM_CUDA_TRY(cudaMemcpyAsync(ctx.h_counters, ctr, sizeof(IterCounters), cudaMemcpyDeviceToHost, st));
            NNM_CUDA_TRY(cudaStreamSynchronize(st));
            const uint64_t nprop = ctx.h_counters->proposals;
            if (nprop * prop_bytes > ws.bucket.bytes) {
                NNM_CUDA_TRY(ws.bucket.ensure((size_t)(nprop * (g.fast && tc ? 1.5 : 1.25) + 1024) * prop_bytes));
                ja.bucket = ws.bucket.p;
            }
            NNM_CUDA_TRY(part1(ja, ntier));
            NNM_CUDA_TRY(copy_back());
            NNM_CUDA_TRY(cudaStreamSynchronize(st));
        }
        NNM_CUDA_TRY(cudaGetLastError());
        const IterCounters hc = *ctx.h_counters;
        if (hc.error) {
            ctx.last_error = "device capacity check failed (code " + std::to_string(hc.error) + ")";
            return 6;
        }
        if (ctx.prof && g.audit) {
            float am;
            std::memcpy(&am, &hc.audit_max, 4);
            ctx.audit_max = std::max(ctx.audit_max, am);
            ctx.audit_err_c = g.err_c;
        }
        if (ctx.prof) {
            float t01 = 0.f, t23 = 0.f, t34 = 0.f;
            cudaEventElapsedTime(&t01, ctx.ev[0], ctx.ev[1]);
            cudaEventElapsedTime(&t23, ctx.ev[2], ctx.ev[3]);
            cudaEventElapsedTime(&t34, ctx.ev[3], ctx.ev[4]);
            // algorithmic traffic of the count pass: each joined row gathers
            // its list vectors (FP32, or u8 on the tensor cores, with their
            // norms), list ids and the K-th distances once and writes one
            // 2-byte count per list slot; the FP32 path also writes one
            // distance per pair.  The emit pass gathers the same members
            // again on the tensor cores (or reads the stored distances) and
            // writes every proposal (16 B in the exact tier, 8 B in the fast tier).
            for (int t = 0; t < NTIER; t++) ctx.join_rows[t] += hc.ntier[t];
            if (ctx.iter_log.size() < 4096) {
                Ctx::IterLog L{n, {hc.ntier[0], hc.ntier[1], hc.ntier[2], hc.ntier[3], hc.ntier[4]},
                               hc.pairs, hc.proposals, hc.flags, hc.ncmps, hc.sum_s, t01, t23, t34};
                ctx.iter_log.push_back(L);
            }
            if (tc) ctx.join_rows_tc += hc.ntier[0] + hc.ntier[1] + hc.ntier[2] + hc.ntier[3] + (u8_tc ? hc.ntier[4] : 0u);
            const double s_tc = (double)hc.sum_s_tc, s_f32 = (double)(hc.sum_s - hc.sum_s_tc);
            ctx.kjoin.launches += tc ? 1 + (hc.ntier[4] > 0)
                                     : (hc.ntier[0] > 0) + (hc.ntier[1] > 0) + (hc.ntier[2] > 0) +
                                           (hc.ntier[3] > 0) + (hc.ntier[4] > 0);
            ctx.kjoin.ms += t01;
            const double f32_slot = u8_last ? (double)g.kq + 14.0 : (double)g.dp * 4.0 + 10.0;
            ctx.kjoin.bytes += s_f32 * f32_slot + s_tc * ((double)g.kq + 14.0) + (double)hc.pairs * 4.0;
            ctx.kjoin.flops += (double)hc.pairs * (double)g.d * 3.0;
            ctx.kemit.launches += tc ? 1 + (hc.ntier[4] > 0) : 1;
            ctx.kemit.ms += t23;
            ctx.kemit.bytes += (double)hc.pairs * 4.0 + s_f32 * 18.0 + s_tc * ((double)g.kq + 22.0) +
                               (double)hc.proposals * (double)prop_bytes;
            if (tc) {
                // every MMA chain fills a 128 x 128 tile over the padded row:
                // kq K elements (u8), 3 products of kq/4 (BF16 hi + lo), 6 of
                // kq/3 (FP8 hi + mid + lo)
                const double kel = g.tc_kind == 0 ? (double)g.kq : g.tc_kind == 1 ? 3.0 * g.kq / 4.0 : 6.0 * g.kq / 3.0;
                const double per_tile = 2.0 * 128.0 * 128.0 * kel;
                double t0n = 0, t1n = 0;
                for (int t = 0; t < 4; t++) {
                    t0n += (double)((hc.ntier[t] + (8u >> t) - 1) >> (3 - t));
                    t1n += (double)(((approx ? hc.ntier[t] : hc.nemit[t]) + (8u >> t) - 1) >> (3 - t));
                }
                ctx.kjoin.tensor_ops += t0n * per_tile;
                ctx.kemit.tensor_ops += t1n * per_tile;
            }
            ctx.approx_props += hc.approx_props;
            ctx.rechecks += hc.rechecks;
            ctx.kmerge.launches += 1;
            ctx.kmerge.ms += t34;
            ctx.kmerge.bytes += (double)n * K * 16.0 + (double)hc.proposals * (double)prop_bytes + (double)n * 13.0;
        }
        g.gpos += hc.rand_draws;
        g.ncmps += hc.ncmps;
        g.iters++;
        // Convergence: the reference sums float(c_i)/K in float row by row and
        // divides by the row count.  The exact flag total decides unless it is
        // within the float rounding bound of the threshold; then the host
        // repeats the reference's float sum.
        const double exact = (double)hc.flags / ((double)K * (double)n);
        const double slack = 1.05 * ((double)n + 4.0) * std::ldexp(1.0, -24) * exact + 1e-12;
        float mean;
        if (!g.exact_trace && std::fabs(exact - (double)g.delta) > slack + 1e-9 * g.delta) {
            mean = (float)exact;
        } else {
            h_nflag.resize(n);
            NNM_CUDA_TRY(cudaMemcpy(h_nflag.data(), ws.nflag.p, n, cudaMemcpyDeviceToHost));
            mean = host_mean(h_nflag, n, K);
        }
        g.trace.push_back(mean);
        const bool converged = (std::fabs(exact - (double)g.delta) > slack + 1e-9 * g.delta)
                                   ? (exact < (double)g.delta)
                                   : (mean < g.delta);
        if (converged || (g.max_iter && it + 1 >= g.max_iter)) {
            g.carry = track;
            break;
        }
        if (it + 1 >= 100000) {
            ctx.last_error = "NN-Descent did not converge";
            return 6;
        }
    }
    return 0;
}

}  // namespace nnm
