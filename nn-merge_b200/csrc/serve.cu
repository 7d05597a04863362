// Fast batched LySearch (NNM_SERVE_FAST): the per-query steps of
// LySearch::knnSearch (lysearch.cpp:363-437) and nndHNSWSrch (:236-322),
// laid out for throughput rather than for the reference's float rounding.
//
// One warp per query; persistent warps pull queries from a counter, so
// queries of different beam widths balance.
//   - distances: a whole warp per distance, lane l holding components
//     [4l, 4l+4) (+128 per further float4) of the query in registers; a
//     row is one coalesced 512-byte read for d = 128.  Up to 32 distances
//     are evaluated together and reduced by a transposing butterfly (31
//     shuffles for 32 sums), after which lane j holds distance j.  The
//     summation order differs from the reference's sequential sum.
//   - greedy descent on the upper layers: the reference's rule (move to the
//     first strictly nearer neighbour of the minimum distance in list order,
//     repeat until no move) evaluated a list chunk at a time.
//   - beam: the reference keeps a result max-heap of size topk and a
//     candidate heap, and stops when the nearest candidate is farther than
//     the worst result.  Every candidate that can still be expanded is in
//     the result set, so both heaps are replaced by one array of at most
//     `beam` entries in shared memory, sorted by (distance, id), with an
//     "expanded" bit per entry: expand the first unexpanded entry, merge the
//     accepted neighbours (distance below the worst entry, or the beam not
//     full) into place (only the entries after the first new one move),
//     stop when every entry is expanded.
//   - width: a step expands the first min(width, beam / 64) unexpanded
//     entries together, reading their lists as one sequence of 32-id chunks,
//     so that the dependent loads (offsets, lists, visited bits, rows) of
//     several nodes are in flight at once; width 1 is strict best-first.
//   - visited set: one bitmap per warp slot in HBM, cleared after each query
//     from the list of ids it set.
#include <algorithm>
#include <cmath>

#include "nnm_hier.h"
#include "nnm_launch.h"

namespace nnm {
namespace {
constexpr unsigned FULL = 0xffffffffu;
constexpr int FW = 4;                    // warps per block
constexpr uint32_t FVCAP = 65536;        // visited ids recorded per warp slot
constexpr uint32_t EXP_BIT = 1u << 31;   // beam entry already expanded
constexpr uint32_t IDM = 0x7fffffffu;
constexpr uint32_t FAST_MAX_DP = 512;    // 4 float4 per lane
constexpr uint32_t GROUP = 4;            // 32-id chunks of a step whose loads and atomics overlap
constexpr uint32_t WARP_EXTRA = 256 + GROUP * 32 * 4;  // nd, ni and fr after the two beam arrays

// self-check codes, shared with the exact kernel's report
enum : unsigned { FERR_LOOP = 4u, FERR_BAD_ID = 8u, FERR_BEAM_RANGE = 32u };

struct ServeArgs {
    const float* x;
    uint32_t dp4;  // float4 per row
    uint32_t L;
    uint64_t off_base[16];
    uint32_t nrows[16];
    const uint64_t* off_all;
    const uint32_t* adj_all;
    const float* q;
    uint32_t nq;
    const uint32_t* beams;
    uint32_t beam, cap, out_k;
    uint32_t entry;
    const uint32_t* probes;
    uint32_t nprobe, g0;
    uint32_t* out_ids;
    float* out_d;
    uint32_t* visited;
    uint32_t words;
    uint32_t* vlist;
    uint32_t width;  // most unexpanded entries expanded together (1..4)
    uint32_t flat;               // nndFlatSrch: random seeds, no descent
    const uint32_t* flat_off;    // seeds of beam width b at flat_pool + flat_off[b]
    const uint32_t* flat_pool;
    unsigned* next_q;
    unsigned* overflow;
    unsigned long long* ncmps;
    unsigned long long* nexp;
};

template <int M>
__device__ __forceinline__ float term(float a, float b, float acc) {
    const float t = a - b;
    if (M == L2) return fmaf(t, t, acc);
    if (M == L1) return acc + fabsf(t);
    return (a != 0.f || b != 0.f) ? acc + t * t / (a + b) : acc;
}
template <int M>
__device__ __forceinline__ float part4(const float4 q, const float4 r, float acc) {
    acc = term<M>(q.x, r.x, acc);
    acc = term<M>(q.y, r.y, acc);
    acc = term<M>(q.z, r.z, acc);
    return term<M>(q.w, r.w, acc);
}

// Distances from the query (qr, spread over the warp) to the rows whose ids
// lanes 0..nf-1 hold in fid (nf <= 32, warp-uniform).  Lane j returns the
// distance of row j (0 for j >= nf).
template <int M, int QV>
__device__ __forceinline__ float warp_dists(const float4 (&qr)[QV], const float4* __restrict__ x4, uint32_t dp4,
                                            uint32_t fid, uint32_t nf, uint32_t lane) {
    constexpr int NB = QV == 1 ? 8 : (QV == 2 ? 4 : 2);  // rows in flight per lane
    if (nf <= (uint32_t)NB) {
        // few rows: one xor-shuffle reduction per row.  Its sum tree pairs
        // lanes l and l^s at width s = 16, 8, .., 1 exactly as the
        // transposing butterfly below does, so the sums are the same bits.
        float4 r[NB][QV];
#pragma unroll
        for (int b = 0; b < NB; b++) {
            const uint32_t id = __shfl_sync(FULL, fid, b);
#pragma unroll
            for (int t = 0; t < QV; t++) {
                const uint32_t c4 = lane + 32u * t;
                r[b][t] = make_float4(0.f, 0.f, 0.f, 0.f);
                if ((uint32_t)b < nf && c4 < dp4) r[b][t] = __ldg(x4 + (size_t)id * dp4 + c4);
            }
        }
        float out = 0.f;
#pragma unroll
        for (int b = 0; b < NB; b++) {
            if ((uint32_t)b < nf) {
                float sum = 0.f;
#pragma unroll
                for (int t = 0; t < QV; t++) sum = part4<M>(qr[t], r[b][t], sum);
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(FULL, sum, o);
                if (lane == (uint32_t)b) out = sum;
            }
        }
        return out;
    }
    float v[32];
#pragma unroll
    for (int j = 0; j < 32; j++) v[j] = 0.f;
#pragma unroll
    for (int j0 = 0; j0 < 32; j0 += NB) {
        if ((uint32_t)j0 < nf) {
            float4 r[NB][QV];
#pragma unroll
            for (int b = 0; b < NB; b++) {
                const uint32_t id = __shfl_sync(FULL, fid, j0 + b);
#pragma unroll
                for (int t = 0; t < QV; t++) {
                    const uint32_t c4 = lane + 32u * t;
                    r[b][t] = make_float4(0.f, 0.f, 0.f, 0.f);
                    if ((uint32_t)(j0 + b) < nf && c4 < dp4) r[b][t] = __ldg(x4 + (size_t)id * dp4 + c4);
                }
            }
#pragma unroll
            for (int b = 0; b < NB; b++)
#pragma unroll
                for (int t = 0; t < QV; t++) v[j0 + b] = part4<M>(qr[t], r[b][t], v[j0 + b]);
        }
    }
    // transposing butterfly: after the level of width s, v[i] holds the
    // partial sum of distance (lane's upper bits) + i over 2x more lanes
#pragma unroll
    for (int s = 16; s >= 1; s >>= 1) {
        const bool up = (lane & s) != 0;
#pragma unroll
        for (int i = 0; i < s; i++) {
            const float send = up ? v[i] : v[i + s];
            const float keep = up ? v[i + s] : v[i];
            v[i] = keep + __shfl_xor_sync(FULL, send, s);
        }
    }
    return v[0];
}

__device__ __forceinline__ bool key_less(float da, uint32_t ia, float db, uint32_t ib) {
    return da < db || (da == db && ia < ib);
}

// Smallest d over lanes < valid, ties to the lowest lane.
__device__ __forceinline__ void warp_argmin(float d, uint32_t valid, uint32_t lane, float& md, uint32_t& ml) {
    float m = lane < valid ? d : INFINITY;
    uint32_t l = lane < valid ? lane : 32u;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const float om = __shfl_xor_sync(FULL, m, o);
        const uint32_t ol = __shfl_xor_sync(FULL, l, o);
        if (om < m || (om == m && ol < l)) {
            m = om;
            l = ol;
        }
    }
    md = m;
    ml = l;
}

// Bitonic sort of one (d, id) pair per lane over lanes [0, w), w a power of
// two (warp-uniform); ascending by (d, id).  Lanes >= w are left as they are.
__device__ __forceinline__ void warp_sort(float& d, uint32_t& id, uint32_t lane, uint32_t w) {
#pragma unroll
    for (uint32_t k = 2; k <= 32; k <<= 1) {
        if (k > w) break;
#pragma unroll
        for (uint32_t j = k >> 1; j > 0; j >>= 1) {
            const float od = __shfl_xor_sync(FULL, d, j);
            const uint32_t oi = __shfl_xor_sync(FULL, id, j);
            const bool asc = (lane & k) == 0 || k == w;
            const bool low = (lane & j) == 0;
            const bool other_less = key_less(od, oi, d, id);
            const bool other_more = key_less(d, id, od, oi);
            if ((low == asc) ? other_less : other_more) {
                d = od;
                id = oi;
            }
        }
    }
}

// Five CTAs per SM (registers capped at 96, a few spilled): the kernel is
// bound by memory latency, and 20 warps per SM hide it better than 16 --
// 6 % faster on the 1M hierarchy than the uncapped 126 registers; six CTAs
// spill more and lose again.
template <int M, int QV>
__global__ void __launch_bounds__(FW * 32, 5) k_serve(ServeArgs a) {
    extern __shared__ __align__(16) unsigned char smem[];
    const uint32_t w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t slot = blockIdx.x * FW + w;
    unsigned char* base = smem + (size_t)w * ((size_t)a.cap * 16 + WARP_EXTRA);
    float* bd = reinterpret_cast<float*>(base);
    uint32_t* bi = reinterpret_cast<uint32_t*>(bd + a.cap);
    float* td = reinterpret_cast<float*>(bi + a.cap);
    uint32_t* ti = reinterpret_cast<uint32_t*>(td + a.cap);
    float* nd = reinterpret_cast<float*>(ti + a.cap);
    uint32_t* ni = reinterpret_cast<uint32_t*>(nd + 32);
    uint32_t* fr = ni + 32;  // fresh ids of one group of a step
    uint32_t* vis = a.visited + (size_t)slot * a.words;
    uint32_t* vl = a.vlist + (size_t)slot * FVCAP;
    const float4* x4 = reinterpret_cast<const float4*>(a.x);
    const uint32_t nlast = a.nrows[a.L - 1];
    unsigned long long cmps = 0, nexp = 0;
    for (;;) {
        uint32_t qi = 0;
        if (lane == 0) qi = atomicAdd(a.next_q, 1u);
        qi = __shfl_sync(FULL, qi, 0);
        if (qi >= a.nq) break;
        uint32_t ef = a.beams ? a.beams[qi] : a.beam;
        if (ef < a.out_k || ef > a.cap) {
            if (lane == 0) atomicOr(a.overflow, FERR_BEAM_RANGE);
            ef = min(max(ef, a.out_k), a.cap);
        }
        // expansions per step: wide beams take up to a.width, narrow ones 1
        const uint32_t width = max(1u, min(a.width, ef / 64));
        float4 qr[QV];
#pragma unroll
        for (int t = 0; t < QV; t++) {
            const uint32_t c4 = lane + 32u * t;
            qr[t] = c4 < a.dp4 ? __ldg(reinterpret_cast<const float4*>(a.q) + (size_t)qi * a.dp4 + c4)
                               : make_float4(0.f, 0.f, 0.f, 0.f);
        }
        // entry
        uint32_t cur = 0, g0;
        float cur_d = 0.f;
        if (a.flat) {
            g0 = a.L - 1;  // nndFlatSrch: no descent; the seeds start the beam
        } else if (a.probes) {
            g0 = a.g0;
            uint32_t pid = 0;
            if (lane < a.nprobe) {
                pid = a.probes[(size_t)qi * a.nprobe + lane];
                if (pid >= a.nrows[g0]) {
                    atomicOr(a.overflow, FERR_BAD_ID);
                    pid = 0;
                }
            }
            const float pd = warp_dists<M, QV>(qr, x4, a.dp4, pid, a.nprobe, lane);
            uint32_t l;
            warp_argmin(pd, a.nprobe, lane, cur_d, l);
            cur = __shfl_sync(FULL, pid, l & 31);
            cmps += a.nprobe;
        } else {
            g0 = 0;
            cur = a.entry;
            cur_d = __shfl_sync(FULL, warp_dists<M, QV>(qr, x4, a.dp4, cur, 1, lane), 0);
            cmps++;
        }
        // greedy descent (lysearch.cpp:397-420); upper-layer ids were checked
        // against their layers when the index was made
        for (uint32_t g = g0; g + 1 < a.L; g++) {
            const uint64_t* off = a.off_all + a.off_base[g];
            uint32_t moves = 0;
            for (;;) {
                if (cur >= a.nrows[g] || ++moves > a.nrows[g]) {
                    if (lane == 0) atomicOr(a.overflow, cur >= a.nrows[g] ? FERR_BAD_ID : FERR_LOOP);
                    cur = 0;
                    break;
                }
                const uint64_t b = off[cur], e = off[cur + 1];
                float best = cur_d;
                uint32_t bid = cur;
                for (uint64_t c0 = b; c0 < e; c0 += 32) {
                    const uint32_t cnt = (uint32_t)(e - c0 < 32 ? e - c0 : 32);
                    const uint32_t nn = lane < cnt ? a.adj_all[c0 + lane] : 0u;
                    const float dd = warp_dists<M, QV>(qr, x4, a.dp4, nn, cnt, lane);
                    cmps += cnt;
                    float md;
                    uint32_t ml;
                    warp_argmin(dd, cnt, lane, md, ml);
                    const uint32_t mid = __shfl_sync(FULL, nn, ml & 31);
                    if (md < best) {
                        best = md;
                        bid = mid;
                    }
                }
                if (bid == cur) break;
                cur = bid;
                cur_d = best;
            }
        }
        // beam on the last layer
        const uint64_t* off = a.off_all + a.off_base[a.L - 1];
        uint32_t m = 0, p = 0, nvis = 0;
        // Offers the fresh rows whose ids lanes [0, nf) hold: distances, the
        // ones below the worst entry of a full beam sorted by a bitonic
        // network over those lanes and merged in place -- entries before the
        // first new one keep their slots; the suffix [lo0, m) is staged, then
        // every entry of the merged range [lo0, m2) is written once.
        auto offer = [&](uint32_t fid, uint32_t nf) {
            cmps += nf;
            const float dd = warp_dists<M, QV>(qr, x4, a.dp4, fid, nf, lane);
            bool acc = lane < nf;
            if (m >= ef) acc = acc && key_less(dd, fid, bd[m - 1], bi[m - 1] & IDM);
            const uint32_t nk = __popc(__ballot_sync(FULL, acc));
            if (nk == 0) return;
            float kd = acc ? dd : INFINITY;
            uint32_t kid = acc ? fid : 0xffffffffu;
            uint32_t w = 1;
            while (w < nf) w <<= 1;
            warp_sort(kd, kid, lane, w);
            __syncwarp();
            nd[lane] = kd;
            ni[lane] = kid;
            const uint32_t m2 = min(ef, m + nk);
            uint32_t npos = 0;
            if (lane < nk) {
                uint32_t lo = 0, hi = m;
                while (lo < hi) {
                    const uint32_t md = (lo + hi) >> 1;
                    if (key_less(bd[md], bi[md] & IDM, kd, kid)) lo = md + 1;
                    else hi = md;
                }
                npos = lane + lo;
            }
            const uint32_t lo0 = __shfl_sync(FULL, npos, 0);
            for (uint32_t i = lo0 + lane; i < m; i += 32) {
                td[i - lo0] = bd[i];
                ti[i - lo0] = bi[i];
            }
            __syncwarp();
            for (uint32_t i = lo0 + lane; i < m; i += 32) {
                const float d0 = td[i - lo0];
                const uint32_t i0 = ti[i - lo0];
                uint32_t lo = 0, hi = nk;
                while (lo < hi) {
                    const uint32_t md = (lo + hi) >> 1;
                    if (key_less(nd[md], ni[md], d0, i0 & IDM)) lo = md + 1;
                    else hi = md;
                }
                if (i + lo < m2) {
                    bd[i + lo] = d0;
                    bi[i + lo] = i0;
                }
            }
            if (lane < nk && npos < m2) {
                bd[npos] = kd;
                bi[npos] = kid;
            }
            __syncwarp();
            m = m2;
            if (lo0 < p) p = lo0;
        };
        if (a.flat) {
            // nndFlatSrch (lysearch.cpp:455-472): the beam's getRndSds seeds
            const uint32_t* sd = a.flat_pool + a.flat_off[ef];
            for (uint32_t c0 = 0; c0 < ef; c0 += 32) {
                const uint32_t cnt = min(32u, ef - c0);
                uint32_t id = 0;
                if (lane < cnt) {
                    id = sd[c0 + lane];
                    atomicOr(&vis[id >> 5], 1u << (id & 31));
                    if (nvis + lane < FVCAP) vl[nvis + lane] = id;
                }
                nvis += cnt;
                offer(id, cnt);
            }
        } else if (cur < nlast) {
            if (lane == 0) {
                bd[0] = cur_d;
                bi[0] = cur;
                atomicOr(&vis[cur >> 5], 1u << (cur & 31));
                vl[0] = cur;
            }
            m = 1;
            nvis = 1;
        } else if (lane == 0) {
            atomicOr(a.overflow, FERR_BAD_ID);
        }
        __syncwarp();
        uint32_t expansions = 0;
        for (;;) {
            __syncwarp();  // the expanded marks and the last merge are visible
            // the first `width` unexpanded entries; lane e keeps the e-th one
            uint32_t ne = 0, mine = 0, mypos = 0, last = 0;
            for (uint32_t s0 = p; s0 < m && ne < width; s0 += 32) {
                unsigned bal = __ballot_sync(FULL, s0 + lane < m && !(bi[s0 + lane] & EXP_BIT));
                while (bal && ne < width) {
                    last = s0 + __ffs(bal) - 1;
                    bal &= bal - 1;
                    if (lane == ne) {
                        mine = bi[last] & IDM;
                        mypos = last;
                    }
                    ne++;
                }
            }
            if (ne == 0) break;
            expansions += ne;
            if (expansions > nlast) {
                if (lane == 0) atomicOr(a.overflow, FERR_LOOP);
                break;
            }
            p = last + 1;
            __syncwarp();
            if (lane < ne) bi[mypos] = mine | EXP_BIT;
            nexp += ne;
            // the selected nodes' lists, read as one sequence of `total` ids:
            // entry t belongs to list e when end_{e-1} <= t < end_e
            uint64_t lb = 0, le = 0;
            if (lane < ne) {
                lb = off[mine];
                le = off[mine + 1];
            }
            const uint32_t len = (uint32_t)(le - lb);
            uint32_t pre = len;
#pragma unroll
            for (int o = 1; o < 4; o <<= 1) {
                const uint32_t v = __shfl_up_sync(FULL, pre, o);
                if (lane >= (uint32_t)o) pre += v;
            }
            const uint32_t end0 = __shfl_sync(FULL, pre, 0), end1 = __shfl_sync(FULL, pre, 1),
                           end2 = __shfl_sync(FULL, pre, 2), total = __shfl_sync(FULL, pre, 3);
            const uint64_t base_l = lb - (pre - len);  // list e: adjacency index base_e + t
            const uint64_t base0 = __shfl_sync(FULL, base_l, 0), base1 = __shfl_sync(FULL, base_l, 1),
                           base2 = __shfl_sync(FULL, base_l, 2), base3 = __shfl_sync(FULL, base_l, 3);
            // the step's ids GROUP x 32 at a time: every list load, then every
            // visited-bit atomic, is in flight at once; the fresh ids are
            // gathered in list order and offered 32 at a time (the beam after
            // a step is the best of the union whatever the order of offers)
            for (uint32_t t0 = 0; t0 < total; t0 += 32 * GROUP) {
                uint32_t nn[GROUP];
                bool fresh[GROUP];
#pragma unroll
                for (uint32_t c = 0; c < GROUP; c++) {
                    const uint32_t t = t0 + 32 * c + lane;
                    nn[c] = 0;
                    if (t < total) {
                        const uint64_t bs = t < end0 ? base0 : (t < end1 ? base1 : (t < end2 ? base2 : base3));
                        nn[c] = a.adj_all[bs + t];
                    }
                }
#pragma unroll
                for (uint32_t c = 0; c < GROUP; c++) {
                    fresh[c] = false;
                    if (t0 + 32 * c + lane < total) {
                        const uint32_t old = atomicOr(&vis[nn[c] >> 5], 1u << (nn[c] & 31));
                        fresh[c] = !(old & (1u << (nn[c] & 31)));
                    }
                }
                uint32_t nf = 0;
                __syncwarp();  // the last offer() has finished with fr
#pragma unroll
                for (uint32_t c = 0; c < GROUP; c++) {
                    const unsigned fb = __ballot_sync(FULL, fresh[c]);
                    if (fresh[c]) {
                        const uint32_t r = nf + __popc(fb & ((1u << lane) - 1u));
                        fr[r] = nn[c];
                        if (nvis + r < FVCAP) vl[nvis + r] = nn[c];
                    }
                    nf += __popc(fb);
                }
                nvis += nf;
                __syncwarp();
                for (uint32_t f0 = 0; f0 < nf; f0 += 32) {
                    const uint32_t cnt = min(32u, nf - f0);
                    const uint32_t fid = lane < cnt ? fr[f0 + lane] : 0u;
                    offer(fid, cnt);
                }
            }
        }
        // results: the first out_k entries
        for (uint32_t t = lane; t < a.out_k; t += 32) {
            const size_t o = (size_t)qi * a.out_k + t;
            a.out_ids[o] = t < m ? (bi[t] & IDM) : 0xffffffffu;
            if (a.out_d) a.out_d[o] = t < m ? bd[t] : 0.f;
        }
        // clear this query's visited bits
        if (nvis <= FVCAP) {
            for (uint32_t t = lane; t < nvis; t += 32) {
                const uint32_t id = vl[t];
                atomicAnd(&vis[id >> 5], ~(1u << (id & 31)));
            }
        } else {
            for (uint32_t t = lane; t < a.words; t += 32) vis[t] = 0;
        }
        __syncwarp();
    }
    for (int o = 16; o > 0; o >>= 1) cmps += __shfl_xor_sync(FULL, cmps, o);
    if (lane == 0) {
        atomicAdd(a.ncmps, cmps / 32);
        atomicAdd(a.nexp, nexp);
    }
}

using ServeFn = void (*)(ServeArgs);
template <int M>
ServeFn pick_qv(uint32_t qv) {
    return qv == 1 ? k_serve<M, 1> : (qv == 2 ? k_serve<M, 2> : k_serve<M, 4>);
}
}  // namespace

int index_run_fast(Ctx& ctx, IndexDev& ix, const SearchReq& r) {
    cudaStream_t st = ctx.stream;
    if (ix.dp > FAST_MAX_DP) {
        ctx.last_error = "fast search supports d <= 512";
        return 1;
    }
    const uint32_t dp4 = ix.dp / 4;
    const uint32_t qv = dp4 <= 32 ? 1 : (dp4 <= 64 ? 2 : 4);
    const ServeFn fn = ix.metric == L2 ? pick_qv<L2>(qv) : (ix.metric == L1 ? pick_qv<L1>(qv) : pick_qv<CHI2>(qv));
    const size_t smem = (size_t)FW * ((size_t)r.beam_max * 16 + WARP_EXTRA);
    NNM_CUDA_TRY(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int nsm = 148, per_sm = 1;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, ctx.device);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, FW * 32, smem);
    const uint32_t blocks = (uint32_t)std::min(std::max(1, per_sm), 8) * (uint32_t)nsm;
    const uint32_t words = (ix.n + 31) / 32;
    const size_t slots = (size_t)blocks * FW;
    if (ix.visited.bytes < slots * words * 4) {
        NNM_CUDA_TRY(ix.visited.ensure(slots * words * 4));
        NNM_CUDA_TRY(cudaMemsetAsync(ix.visited.p, 0, slots * words * 4, st));
    }
    NNM_CUDA_TRY(ix.vlist.ensure(slots * FVCAP * 4));
    ServeArgs a{};
    a.x = ix.x.as<float>();
    a.dp4 = dp4;
    a.L = ix.L;
    for (uint32_t g = 0; g < ix.L; g++) {
        a.off_base[g] = ix.off_base[g];
        a.nrows[g] = ix.nrows[g];
    }
    a.off_all = ix.off.as<uint64_t>();
    a.adj_all = ix.adj.as<uint32_t>();
    a.q = r.q;
    a.nq = r.nq;
    a.beams = r.beams;
    a.beam = r.beam;
    a.cap = r.beam_max;
    a.out_k = r.out_k;
    a.entry = ix.entry;
    a.probes = r.probes;
    a.nprobe = r.nprobe;
    a.g0 = r.g0;
    a.out_ids = r.out_ids;
    a.out_d = r.out_d;
    a.visited = ix.visited.as<uint32_t>();
    a.words = words;
    a.vlist = ix.vlist.as<uint32_t>();
    a.width = ix.width;
    a.flat = r.flat;
    a.flat_off = r.flat_off;
    a.flat_pool = r.flat_pool;
    unsigned char* c = ix.ctr.as<unsigned char>();
    a.next_q = reinterpret_cast<unsigned*>(c);
    a.overflow = reinterpret_cast<unsigned*>(c + 4);
    a.ncmps = reinterpret_cast<unsigned long long*>(c + 8);
    a.nexp = reinterpret_cast<unsigned long long*>(c + 16);
    fn<<<blocks, FW * 32, smem, st>>>(a); count_launch();
    NNM_CUDA_TRY(cudaGetLastError());
    return 0;
}

}  // namespace nnm
