// Initial graphs from the learned codes ("candidates bucketed by the codes").
//
// Views: for v = 0..V-1 the key of a row is its 32-bit code rotated left by
// 8v bits, so that every byte of the code leads one ordering.  Each leaf's
// rows are sorted by (key, row) -- a bitonic sort of 64-bit words, one
// segment of P = 2^m slots per (view, leaf), all segments in the same
// launches.  Rows next to each other in a view share a long code prefix.
//
// Leaf init (k_learned_rows): a row's candidates are the rows within +-8
// positions of it in each of the 4 views of its leaf (64 slots); the k
// nearest distinct ones (exact distances) form its initial pool, topped up
// with random rows when fewer than k are found.
//
// Merge cross samples (k_learned_cross): a row keeps its best k - cut
// entries; its cut new entries are the nearest rows of the other leaves
// among those found next to its key in each view of each other leaf
// (binary search, then a window), topped up with random rows of the other
// leaves when fewer are found.
#include <algorithm>

#include "nnm_builders.h"
#include "nnm_launch.h"
#include "nnm_learned.h"

namespace nnm {
namespace {

constexpr uint32_t NVIEW = 4;
constexpr uint32_t NCAND = 64;    // candidate slots per row (2 per lane)
constexpr int IW = 8;             // warps per block
constexpr uint32_t BLK = 2048;    // elements sorted in shared memory per block
constexpr unsigned FULLM = 0xffffffffu;
constexpr uint32_t NO_ID = 0xffffffffu;

__device__ __forceinline__ uint32_t rotl(uint32_t v, uint32_t s) { return s ? (v << s) | (v >> (32 - s)) : v; }

__device__ __forceinline__ void cswap(unsigned long long& a, unsigned long long& b, bool asc) {
    if ((a > b) == asc) {
        const unsigned long long t = a;
        a = b;
        b = t;
    }
}

__global__ void k_views_fill(unsigned long long* keys, const uint32_t* codes, const uint32_t* leaf_off,
                             uint32_t nleaf, uint32_t P, uint32_t nseg) {
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (size_t)nseg * P) return;
    const uint32_t seg = (uint32_t)(t / P), i = (uint32_t)(t - (size_t)seg * P);
    const uint32_t v = seg / nleaf, l = seg - v * nleaf;
    const uint32_t lo = leaf_off[l], L = leaf_off[l + 1] - lo;
    unsigned long long k = ~0ull;
    if (i < L) {
        const uint32_t row = lo + i;
        k = ((unsigned long long)rotl(codes[row], 8 * v) << 32) | row;
    }
    keys[t] = k;
}

// Bitonic sort (Batcher 1968) of every P-slot segment, ascending.  The
// direction of a compare at stage (k, j) follows bit k of the index within
// the segment.  Thread i compares slots a = 2i - (i mod j) and a + j.
__global__ void __launch_bounds__(1024) k_bitonic_block(unsigned long long* keys, uint32_t P) {
    __shared__ unsigned long long s[BLK];
    const size_t base = (size_t)blockIdx.x * BLK;
    const uint32_t seg_base = (uint32_t)(base & (P - 1));
    for (uint32_t i = threadIdx.x; i < BLK; i += 1024) s[i] = keys[base + i];
    __syncthreads();
    for (uint32_t k = 2; k <= BLK; k <<= 1)
        for (uint32_t j = k >> 1; j > 0; j >>= 1) {
            const uint32_t i = threadIdx.x, a = 2 * i - (i & (j - 1)), b = a + j;
            cswap(s[a], s[b], (((seg_base + a) & k) == 0));
            __syncthreads();
        }
    for (uint32_t i = threadIdx.x; i < BLK; i += 1024) keys[base + i] = s[i];
}

__global__ void k_bitonic_global(unsigned long long* keys, size_t total, uint32_t P, uint32_t k, uint32_t j) {
    const size_t h = (size_t)blockIdx.x * blockDim.x + threadIdx.x;  // one thread per compared pair
    if (h >= total / 2) return;
    const size_t a = 2 * h - (h & (j - 1)), b = a + j;
    cswap(keys[a], keys[b], (((uint32_t)(a & (P - 1)) & k) == 0));
}

__global__ void __launch_bounds__(1024) k_bitonic_merge_block(unsigned long long* keys, uint32_t P, uint32_t k) {
    __shared__ unsigned long long s[BLK];
    const size_t base = (size_t)blockIdx.x * BLK;
    const uint32_t seg_base = (uint32_t)(base & (P - 1));
    for (uint32_t i = threadIdx.x; i < BLK; i += 1024) s[i] = keys[base + i];
    __syncthreads();
    const bool asc = ((seg_base & k) == 0);  // k >= 2*BLK: one direction per block
    for (uint32_t j = BLK / 2; j > 0; j >>= 1) {
        const uint32_t i = threadIdx.x, a = 2 * i - (i & (j - 1)), b = a + j;
        cswap(s[a], s[b], asc);
        __syncthreads();
    }
    for (uint32_t i = threadIdx.x; i < BLK; i += 1024) keys[base + i] = s[i];
}

__global__ void k_views_pos(const unsigned long long* keys, const uint32_t* leaf_off, uint32_t nleaf, uint32_t P,
                            uint32_t nseg, uint32_t n, uint32_t* pos) {
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (size_t)nseg * P) return;
    const uint32_t seg = (uint32_t)(t / P), i = (uint32_t)(t - (size_t)seg * P);
    const uint32_t v = seg / nleaf, l = seg - v * nleaf;
    if (i >= leaf_off[l + 1] - leaf_off[l]) return;
    pos[(size_t)v * n + (uint32_t)(keys[t] & 0xffffffffu)] = i;
}

// Appends distinct random ids from [0, range) minus [skip_lo, skip_hi)
// until ents holds `want` entries; every id is checked against ents[0, cnt)
// and against row_self.  Warp-wide; returns the new count.
__device__ uint32_t random_fill(SortEnt* ents, uint32_t cnt, uint32_t want, uint32_t row_self, uint32_t range,
                                uint32_t skip_lo, uint32_t skip_hi, const Philox& ph, uint32_t row, uint32_t phase,
                                const float* x, uint32_t dp, int metric, const float* xrow) {
    const int lane = threadIdx.x & 31;
    const uint32_t span = skip_hi - skip_lo;
    for (uint32_t round = 0; cnt < want && round < 64; round++) {
        const uint32_t s = bounded(ph(row, phase, 1000 + round, (uint32_t)lane).x, range - span);
        const uint32_t id = s < skip_lo ? s : s + span;
        bool ok = id != row_self;
        for (uint32_t l = 0; l < cnt && ok; l++)
            if ((ents[l].id & ID_MASK) == id) ok = false;
        const unsigned same = __match_any_sync(FULLM, id);
        if ((int)(__ffs(same) - 1) != lane) ok = false;
        const unsigned bal = __ballot_sync(FULLM, ok);
        const uint32_t r = cnt + __popc(bal & ((1u << lane) - 1u));
        float dd = 0.f;
        if (ok && r < want) dd = dist_seq_rt(metric, xrow, x + (size_t)id * dp, dp);
        __syncwarp();
        if (ok && r < want) ents[r] = SortEnt{dd, id | FLAG_BIT};
        cnt = min(want, cnt + __popc(bal));
        __syncwarp();
    }
    return cnt;
}

// Where candidate distances come from: the u8 copy and norms when the
// tensor-core join prepared them (exact integer dot products, dp4a), else
// the FP32 vectors with the reference's sequential sum.  Both give the
// exact distance of the data.
struct DistSrc {
    const float* x;
    uint32_t dp;
    int metric;
    const uint8_t* xq;
    const uint32_t* nrm;
    uint32_t kq;
};

__device__ __forceinline__ float cand_dist(const DistSrc& s, uint32_t r, uint32_t c) {
    if (s.xq) {
        const uint4* a = reinterpret_cast<const uint4*>(s.xq + (size_t)r * s.kq);
        const uint4* b = reinterpret_cast<const uint4*>(s.xq + (size_t)c * s.kq);
        unsigned dot = 0;
        for (uint32_t i = 0; i < s.kq / 16; i++) {
            const uint4 u = a[i], v = b[i];
            dot = __dp4a(u.x, v.x, dot);
            dot = __dp4a(u.y, v.y, dot);
            dot = __dp4a(u.z, v.z, dot);
            dot = __dp4a(u.w, v.w, dot);
        }
        return (float)((int)(s.nrm[r] + s.nrm[c]) - 2 * (int)dot);
    }
    return dist_seq_rt(s.metric, s.x + (size_t)r * s.dp, s.x + (size_t)c * s.dp, s.dp);
}

// Sorts e[0, cnt), cnt <= 64, by (distance, id word): a warp bitonic sort of
// 64-bit keys, two per lane (lane l holds positions 2l and 2l + 1).
__device__ void warp_sort64(SortEnt* e, uint32_t cnt) {
    const int lane = threadIdx.x & 31;
    unsigned long long v[2];
#pragma unroll
    for (int h = 0; h < 2; h++) {
        const uint32_t i = 2 * lane + h;
        v[h] = i < cnt ? ((unsigned long long)__float_as_uint(e[i].dist) << 32) | e[i].id : ~0ull;
    }
    __syncwarp();
#pragma unroll
    for (uint32_t k = 2; k <= 64; k <<= 1) {
#pragma unroll
        for (uint32_t j = k >> 1; j > 0; j >>= 1) {
            if (j == 1) {
                const bool asc = ((2 * lane) & k) == 0;
                if ((v[0] > v[1]) == asc) {
                    const unsigned long long t = v[0];
                    v[0] = v[1];
                    v[1] = t;
                }
            } else {
#pragma unroll
                for (int h = 0; h < 2; h++) {
                    const uint32_t i = 2 * lane + h;
                    const unsigned long long o = __shfl_xor_sync(FULLM, v[h], j >> 1);
                    const bool lower = (i & j) == 0, asc = (i & k) == 0;
                    v[h] = (lower == asc) ? min(v[h], o) : max(v[h], o);
                }
            }
        }
    }
#pragma unroll
    for (int h = 0; h < 2; h++) {
        const uint32_t i = 2 * lane + h;
        if (i < cnt) e[i] = SortEnt{__uint_as_float((uint32_t)(v[h] >> 32)), (uint32_t)v[h]};
    }
    __syncwarp();
}

// Keeps the first of equal ids among the 64 candidate slots (c0 at slot
// lane, c1 at slot lane + 32) and compacts the kept ones with their exact
// distances to row r into out[]; returns how many.
__device__ uint32_t compact_candidates(uint32_t* cid, uint32_t c0, uint32_t c1, SortEnt* out, const DistSrc& ds,
                                       uint32_t r) {
    const int lane = threadIdx.x & 31;
    cid[lane] = c0;
    cid[lane + 32] = c1;
    __syncwarp();
    bool k0 = c0 != NO_ID, k1 = c1 != NO_ID;
    for (uint32_t s = 0; s < NCAND && (k0 || k1); s++) {
        const uint32_t c = cid[s];
        if (k0 && s < (uint32_t)lane && c == c0) k0 = false;
        if (k1 && s < (uint32_t)lane + 32 && c == c1) k1 = false;
    }
    const unsigned b0 = __ballot_sync(FULLM, k0), b1 = __ballot_sync(FULLM, k1);
    const unsigned lt = (1u << lane) - 1u;
    if (k0) out[__popc(b0 & lt)] = SortEnt{cand_dist(ds, r, c0), c0 | FLAG_BIT};
    if (k1) out[__popc(b0) + __popc(b1 & lt)] = SortEnt{cand_dist(ds, r, c1), c1 | FLAG_BIT};
    __syncwarp();
    return __popc(b0) + __popc(b1);
}

struct RowsArgs {
    const float* x;  // the leaf's vectors (local row 0 = parent row base)
    uint32_t dp, K;
    int metric;
    uint32_t* pid;
    float* pdist;
    uint32_t n, base;  // leaf rows, parent row of local row 0
    const unsigned long long* keys;
    const uint32_t* pos;
    uint32_t P, nleaf, leaf, npar;  // npar: rows of the parent (pos stride)
    uint32_t seed, phase;
    IterCounters* ctr;
    DistSrc ds;
};

__global__ void __launch_bounds__(IW * 32) k_learned_rows(RowsArgs a) {
    __shared__ SortEnt ents[IW][NCAND + 32];
    __shared__ uint32_t cid[IW][NCAND];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t row = blockIdx.x * IW + w;
    if (row >= a.n) return;
    const uint32_t gr = a.base + row;
    // candidate slots: view lane / 8, offsets -(o+1) and +(o+1), o = lane % 8
    const uint32_t v = lane >> 3, o = lane & 7;
    const uint32_t p = a.pos[(size_t)v * a.npar + gr];
    const unsigned long long* seg = a.keys + (size_t)(v * a.nleaf + a.leaf) * a.P;
    uint32_t c0 = NO_ID, c1 = NO_ID;
    if (p >= o + 1) c0 = (uint32_t)(seg[p - o - 1] & 0xffffffffu) - a.base;
    if (p + o + 1 < a.n) c1 = (uint32_t)(seg[p + o + 1] & 0xffffffffu) - a.base;
    const float* xr = a.x + (size_t)row * a.dp;
    uint32_t cnt = compact_candidates(cid[w], c0, c1, ents[w], a.ds, row);
    if (cnt < a.K) {
        const Philox ph{a.seed, 0x6e6e6d03u};
        cnt = random_fill(ents[w], cnt, a.K, row, a.n, 0, 0, ph, row, a.phase, a.x, a.dp, a.metric, xr);
        if (cnt < a.K) {
            if (lane == 0) atomicOr(&a.ctr->error, (unsigned)DERR_CROSS_SAMPLE);
            return;
        }
    }
    warp_sort64(ents[w], cnt);
    if (lane < (int)a.K) {
        a.pid[(size_t)row * a.K + lane] = ents[w][lane].id;
        a.pdist[(size_t)row * a.K + lane] = ents[w][lane].dist;
    }
}

struct CrossArgsL {
    const float* x;
    uint32_t dp, K;
    int metric;
    uint32_t *pid, *cpid;
    float *pdist, *cpdist;
    uint32_t n, keep;
    const uint32_t* codes;
    const unsigned long long* keys;
    const uint32_t* leaf_off;
    uint32_t P, nleaf, nview, npair, win;  // (view, other leaf) pairs used (<= 32), window per pair
    uint32_t seed, phase;
    IterCounters* ctr;
    DistSrc ds;
    const unsigned long long* fence;  // every VFENCE-th key of each segment (P / VFENCE a segment)
};

__device__ __forceinline__ uint32_t leaf_of_row(uint32_t id, const uint32_t* off, uint32_t nleaf) {
    uint32_t lo = 0, hi = nleaf;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (id >= off[mid]) lo = mid;
        else hi = mid;
    }
    return lo;
}

// (view, other-leaf index) of candidate pair q of a row.  When every
// (view, other leaf) pair fits, all are taken; otherwise the row takes
// npair / nview leaves spaced evenly over the other leaves, rotated by a
// per-row draw, in each of nview views.
__device__ __forceinline__ void cross_pair(uint32_t q, uint32_t nl1, uint32_t nview, uint32_t npair, uint32_t rot,
                                           uint32_t& v, uint32_t& lo) {
    if (nview * nl1 <= npair) {
        v = q / nl1;
        lo = q - v * nl1;
    } else {
        const uint32_t nj = npair / nview, j = q / nview;
        v = q - j * nview;
        lo = (uint32_t)(((unsigned long long)j * nl1 / nj + rot) % nl1);
    }
}

__global__ void __launch_bounds__(IW * 32) k_learned_cross(CrossArgsL a) {
    __shared__ SortEnt ents[IW][NCAND + 32];
    __shared__ uint32_t cid[IW][NCAND];
    __shared__ uint32_t cpos[IW][32];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t row = blockIdx.x * IW + w;
    if (row >= a.n) return;
    const uint32_t K = a.K, keep = a.keep, need = K - keep;
    const uint32_t leaf = leaf_of_row(row, a.leaf_off, a.nleaf);
    const uint32_t nl1 = a.nleaf - 1, npair = a.npair;
    // own entries: best `keep` stay, the rest go to the compensation list
    SortEnt* e = ents[w];
    if (lane < (int)K) e[lane] = SortEnt{a.pdist[(size_t)row * K + lane], a.pid[(size_t)row * K + lane]};
    __syncwarp();
    if (lane < (int)need) {
        a.cpid[(size_t)row * K + lane] = e[keep + lane].id;
        a.cpdist[(size_t)row * K + lane] = e[keep + lane].dist;
    }
    __syncwarp();
    const uint32_t rot = bounded(Philox{a.seed, 0x6e6e6d05u}(row, a.phase, 0, 0).x, nl1);
    // lane q < npair: lower bound of this row's key in its pair q
    if (lane < (int)npair) {
        uint32_t v, lo;
        cross_pair(lane, nl1, a.nview, npair, rot, v, lo);
        const uint32_t l2 = lo < leaf ? lo : lo + 1;
        const unsigned long long key = (unsigned long long)rotl(a.codes[row], 8 * v) << 32;
        const unsigned long long* seg = a.keys + (size_t)(v * a.nleaf + l2) * a.P;
        const uint32_t L = a.leaf_off[l2 + 1] - a.leaf_off[l2];
        // the fences (keys VFENCE i < L, read through L1) narrow the search
        // to one window of VFENCE keys: the first fence >= key is at fi, so
        // the lower bound lies in ((fi - 1) VFENCE, fi VFENCE], or past the
        // last fence when fi is the count
        const unsigned long long* fs = a.fence + (size_t)(v * a.nleaf + l2) * (a.P / VFENCE);
        const uint32_t nfv = (L + VFENCE - 1) / VFENCE;
        uint32_t fb = 0, ft = nfv;
        while (fb < ft) {
            const uint32_t mid = (fb + ft) >> 1;
            if (__ldg(fs + mid) < key) fb = mid + 1;
            else ft = mid;
        }
        uint32_t b = fb == 0 ? 0u : (fb - 1) * VFENCE + 1, t = fb == nfv ? L : fb * VFENCE;
        while (b < t) {
            const uint32_t mid = (b + t) >> 1;
            if (seg[mid] < key) b = mid + 1;
            else t = mid;
        }
        cpos[w][lane] = b;
    }
    __syncwarp();
    // candidate slot s: pair s / (2 win), offset s % (2 win) - win
    uint32_t c[2] = {NO_ID, NO_ID};
    for (int h = 0; h < 2; h++) {
        const uint32_t s = lane + 32 * h, per = 2 * a.win;
        if (s < npair * per) {
            const uint32_t q = s / per, off = s - q * per;
            uint32_t v, lo;
            cross_pair(q, nl1, a.nview, npair, rot, v, lo);
            const uint32_t l2 = lo < leaf ? lo : lo + 1;
            const uint32_t L = a.leaf_off[l2 + 1] - a.leaf_off[l2];
            const int64_t pp = (int64_t)cpos[w][q] + (int64_t)off - (int64_t)a.win;
            if (pp >= 0 && pp < (int64_t)L)
                c[h] = (uint32_t)(a.keys[(size_t)(v * a.nleaf + l2) * a.P + (size_t)pp] & 0xffffffffu);
        }
    }
    const float* xr = a.x + (size_t)row * a.dp;
    // candidates go after the kept entries (they are rows of other leaves,
    // so they cannot repeat a kept id)
    SortEnt* cand = e + keep;
    uint32_t cnt = compact_candidates(cid[w], c[0], c[1], cand, a.ds, row);
    if (cnt < need) {
        const Philox ph{a.seed, 0x6e6e6d04u};
        cnt = random_fill(cand, cnt, need, row, a.n, a.leaf_off[leaf], a.leaf_off[leaf + 1], ph, row, a.phase, a.x,
                          a.dp, a.metric, xr);
        if (cnt < need) {
            if (lane == 0) atomicOr(&a.ctr->error, (unsigned)DERR_CROSS_SAMPLE);
            return;
        }
    }
    // the `need` nearest candidates, then the pool sorted
    warp_sort64(cand, cnt);
    warp_sort64(e, K);
    if (lane < (int)K) {
        a.pid[(size_t)row * K + lane] = e[lane].id;
        a.pdist[(size_t)row * K + lane] = e[lane].dist;
    }
}

// fence[i] = keys[VFENCE i]: segments are P keys long, P a multiple of
// VFENCE, so fence i / (P / VFENCE) of segment (i * VFENCE) / P.
__global__ void k_view_fences(const unsigned long long* keys, size_t nfence, unsigned long long* fence) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nfence) fence[i] = keys[i * VFENCE];
}

uint32_t pow2_at_least(uint32_t v) {
    uint32_t p = 1;
    while (p < v) p <<= 1;
    return p;
}

}  // namespace

int views_build(Ctx& ctx, const GraphDev& g, const std::vector<uint32_t>& leaf_off, CodeViews& out) {
    const uint32_t nleaf = (uint32_t)leaf_off.size() - 1;
    uint32_t Lmax = 0;
    for (uint32_t l = 0; l < nleaf; l++) Lmax = std::max(Lmax, leaf_off[l + 1] - leaf_off[l]);
    const uint32_t P = pow2_at_least(std::max(Lmax, BLK)), nseg = NVIEW * nleaf;
    const size_t total = (size_t)nseg * P;
    GraphStore& s = ctx.store;
    NNM_CUDA_TRY(s.vkeys.ensure(total * 8));
    NNM_CUDA_TRY(s.vpos.ensure((size_t)NVIEW * g.n * 4));
    NNM_CUDA_TRY(s.voff.ensure(leaf_off.size() * 4));
    NNM_CUDA_TRY(cudaMemcpyAsync(s.voff.p, leaf_off.data(), leaf_off.size() * 4, cudaMemcpyHostToDevice, ctx.stream));
    unsigned long long* keys = s.vkeys.as<unsigned long long>();
    const uint32_t* off = s.voff.as<uint32_t>();
    cudaStream_t st = ctx.stream;
    k_views_fill<<<blocks_for(total, 256), 256, 0, st>>>(keys, g.codes, off, nleaf, P, nseg); count_launch();
    k_bitonic_block<<<(unsigned)(total / BLK), 1024, 0, st>>>(keys, P); count_launch();
    for (uint32_t k = 2 * BLK; k <= P; k <<= 1) {
        for (uint32_t j = k >> 1; j >= BLK; j >>= 1) {
            k_bitonic_global<<<blocks_for(total / 2, 256), 256, 0, st>>>(keys, total, P, k, j); count_launch();
        }
        k_bitonic_merge_block<<<(unsigned)(total / BLK), 1024, 0, st>>>(keys, P, k); count_launch();
    }
    k_views_pos<<<blocks_for(total, 256), 256, 0, st>>>(keys, off, nleaf, P, nseg, g.n, s.vpos.as<uint32_t>()); count_launch();
    NNM_CUDA_TRY(cudaGetLastError());
    out.V = NVIEW;
    out.nleaf = nleaf;
    out.P = P;
    out.n = g.n;
    out.leaf_off = leaf_off;
    out.keys = keys;
    out.pos = s.vpos.as<uint32_t>();
    // the fences: key VFENCE i of every segment
    const size_t nfence = total / VFENCE;
    NNM_CUDA_TRY(s.vfence.ensure(nfence * 8));
    k_view_fences<<<blocks_for(nfence, 256), 256, 0, st>>>(keys, nfence, s.vfence.as<unsigned long long>()); count_launch();
    NNM_CUDA_TRY(cudaGetLastError());
    out.fence = s.vfence.as<unsigned long long>();
    return 0;
}

int learned_rows(Ctx& ctx, GraphDev& s, const CodeViews& vw, uint32_t leaf) {
    NNM_CUDA_TRY(ctx.ws.counters.ensure(sizeof(IterCounters) + 64));
    NNM_CUDA_TRY(cudaMemsetAsync(ctx.ws.counters.p, 0, sizeof(IterCounters), ctx.stream));
    RowsArgs ra{s.x, s.dp, s.K, s.metric, s.pid, s.pdist, s.n, vw.leaf_off[leaf], vw.keys, vw.pos, vw.P, vw.nleaf,
                leaf, vw.n, s.seed, s.phase++, ctx.ws.counters.as<IterCounters>(),
                DistSrc{s.x, s.dp, s.metric, s.tc_kind == 0 ? s.xq : nullptr, s.nrm, s.kq}};
    k_learned_rows<<<blocks_for(s.n, IW), IW * 32, 0, ctx.stream>>>(ra); count_launch();
    NNM_CUDA_TRY(cudaGetLastError());
    return check_counters(ctx);
}

int learned_cross(Ctx& ctx, GraphDev& g, const CodeViews& vw, const uint32_t* d_leaf_off) {
    NNM_CUDA_TRY(ctx.ws.counters.ensure(sizeof(IterCounters) + 64));
    NNM_CUDA_TRY(cudaMemsetAsync(ctx.ws.counters.p, 0, sizeof(IterCounters), ctx.stream));
    const uint32_t nl1 = vw.nleaf - 1;
    // (view, other leaf) pairs: all views of every other leaf while that is
    // at most 32 pairs, else fewer views, and with more than 32 other leaves
    // view 0 of 32 leaves spread over them (per row); the 64 candidate
    // slots are shared out evenly
    const uint32_t nview = std::max<uint32_t>(1, std::min<uint32_t>(vw.V, 32 / nl1));
    const uint32_t npair = std::min<uint32_t>(nview * nl1, 32);
    const uint32_t win = std::max<uint32_t>(1, NCAND / (2 * npair));
    CrossArgsL ca{g.x, g.dp, g.K, g.metric, g.pid, g.cpid, g.pdist, g.cpdist, g.n, g.K - g.cut, g.codes, vw.keys,
                  d_leaf_off, vw.P, vw.nleaf, nview, npair, win, g.seed, g.phase++,
                  ctx.ws.counters.as<IterCounters>(), DistSrc{g.x, g.dp, g.metric, g.tc_kind == 0 ? g.xq : nullptr, g.nrm, g.kq},
                  vw.fence};
    k_learned_cross<<<blocks_for(g.n, IW), IW * 32, 0, ctx.stream>>>(ca); count_launch();
    NNM_CUDA_TRY(cudaGetLastError());
    return check_counters(ctx);
}

}  // namespace nnm
