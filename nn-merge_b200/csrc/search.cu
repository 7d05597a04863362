// Batched LySearch (lysearch.cpp:363-437 with nndHNSWSrch :236-322).
//
// One warp per query, persistent warps pulling queries from a counter so
// that queries of different beam widths balance.  Per query:
//   - entry point: one global id, rand() % |layer 0| after srand(seed)
//     (lysearch.cpp:382); or, for nndFlatSrch (lysearch.cpp:439-520), no
//     descent and `topk` getRndSds seeds of the last layer in both heaps;
//   - greedy 1-NN descent through layers 0..L-2 (lysearch.cpp:397-420): the
//     distances of a node's neighbours are computed in parallel, one
//     neighbour per lane, and the moves are then applied in list order, as
//     the reference's loop does;
//   - best-first beam search on the last layer with the reference's two
//     std::priority_queue<pair<float,unsigned>> heaps (results: max-heap on
//     distance, size <= topk, in shared memory; candidates: max-heap on
//     minus the distance, in a per-warp HBM slot).  Lane 0 replays
//     libstdc++'s push_heap/pop_heap steps exactly, so the order among equal
//     distances -- which the heaps decide -- is the reference's too.  The
//     neighbours of an expanded node are checked against a per-warp visited
//     bitmap and their distances computed in parallel first, then offered in
//     list order.
// Distances are the reference's sequential float sums (one lane per
// distance), equal to vmath.cpp:56-88 bit for bit.
#include <algorithm>
#include <string>
#include <vector>

#include "nnm_hier.h"
#include "nnm_launch.h"

namespace nnm {
namespace {
constexpr unsigned FULL = 0xffffffffu;
constexpr int SWARPS = 4;         // warps per block
constexpr uint32_t VCAP = 16384;  // visited-list capacity per warp slot
constexpr uint32_t CCAP = 32768;  // candidate-heap capacity per warp slot

// Element of the reference's priority queues: pair<float, unsigned>,
// compared on .first only (CompareByFirst, lysearch.h:37-42).
struct HP {
    float f;
    uint32_t id;
};

// libstdc++ push_heap / pop_heap on a max-heap by .f (one thread).
__device__ __forceinline__ void heap_push(HP* h, uint32_t& n, HP v) {
    int hole = (int)n++;
    int parent = (hole - 1) / 2;
    while (hole > 0 && h[parent].f < v.f) {
        h[hole] = h[parent];
        hole = parent;
        parent = (hole - 1) / 2;
    }
    h[hole] = v;
}
__device__ __forceinline__ void heap_pop(HP* h, uint32_t& n) {
    if (n == 0) return;
    if (n > 1) {
        const int len = (int)n - 1;
        HP v = h[len];
        h[len] = h[0];
        int hole = 0, second = 0;
        while (second < (len - 1) / 2) {
            second = 2 * (second + 1);
            if (h[second].f < h[second - 1].f) second--;
            h[hole] = h[second];
            hole = second;
        }
        if ((len & 1) == 0 && second == (len - 2) / 2) {
            second = 2 * (second + 1);
            h[hole] = h[second - 1];
            hole = second - 1;
        }
        int parent = (hole - 1) / 2;
        while (hole > 0 && h[parent].f < v.f) {
            h[hole] = h[parent];
            hole = parent;
            parent = (hole - 1) / 2;
        }
        h[hole] = v;
    }
    n--;
}

struct SearchArgs {
    const float* x;
    uint32_t dp;
    int metric;
    uint32_t L;
    uint64_t off_base[16];  // start of layer g's offsets in off_all
    const uint64_t* off_all;
    const uint32_t* adj_all;
    const float* q;
    uint32_t nq, topk, entry, n;
    const uint32_t* beams;   // per-query beam widths, or null: topk for all
    uint32_t beam_cap;       // largest beam width (shared-memory sizing)
    uint32_t out_k;          // results written per query
    const uint32_t* probes;  // learned entries: nq x nprobe rows of layer g0, or null
    uint32_t nprobe, g0;
    uint32_t flat;           // nndFlatSrch: random seeds of the last layer, no descent
    const uint32_t* flat_off;   // seeds of beam width b at flat_pool + flat_off[b]
    const uint32_t* flat_pool;
    uint32_t* out_ids;
    float* out_d;
    uint32_t* visited;  // per warp slot: ceil(n/32) words
    uint32_t words;
    uint32_t* vlist;    // per warp slot: VCAP ids
    HP* cand;           // per warp slot: CCAP entries
    unsigned* next_q;
    unsigned long long* ncmps;
    unsigned long long* nexp;
    unsigned* overflow;     // bit 0: candidate heap full; bits 1..: self-check failures
    uint32_t nrows[16];     // rows of each layer
};

enum : unsigned {
    SERR_HEAP = 1u,        // candidate heap capacity reached
    SERR_GREEDY_CAP = 2u,  // greedy descent made more moves than the layer has rows
    SERR_BEAM_CAP = 4u,    // beam search expanded more nodes than the layer has rows
    SERR_BAD_ID = 8u,      // a node id outside its layer
    SERR_BEAM_RANGE = 32u, // a per-query beam width outside [out_k, beam_cap]
};

__global__ void k_search(SearchArgs a) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t slot = blockIdx.x * SWARPS + w;
    const size_t wbytes = (size_t)a.dp * 4 + (size_t)(a.beam_cap + 1) * 8 + 32 * 8;
    unsigned char* base = smem + (size_t)w * ((wbytes + 15) & ~(size_t)15);
    float* qv = reinterpret_cast<float*>(base);
    HP* top = reinterpret_cast<HP*>(base + (size_t)a.dp * 4);
    float* stage_d = reinterpret_cast<float*>(top + a.beam_cap + 1);
    uint32_t* stage_i = reinterpret_cast<uint32_t*>(stage_d + 32);
    uint32_t* vis = a.visited + (size_t)slot * a.words;
    uint32_t* vl = a.vlist + (size_t)slot * VCAP;
    HP* cand = a.cand + (size_t)slot * CCAP;
    unsigned long long cmps = 0, nexp = 0;
    for (;;) {
        unsigned qi = 0;
        if (lane == 0) qi = atomicAdd(a.next_q, 1u);
        qi = __shfl_sync(FULL, qi, 0);
        if (qi >= a.nq) break;
        uint32_t topk = a.beams ? a.beams[qi] : a.topk;
        if (topk < a.out_k || topk > a.beam_cap) {
            if (lane == 0) atomicOr(a.overflow, SERR_BEAM_RANGE);
            topk = min(max(topk, a.out_k), a.beam_cap);
        }
        for (uint32_t t = lane; t < a.dp; t += 32) qv[t] = a.q[(size_t)qi * a.dp + t];
        __syncwarp();
        uint32_t cur = a.entry, g0 = 0;
        float cur_d = 0.f;
        if (a.flat) {
            g0 = a.L - 1;  // nndFlatSrch (lysearch.cpp:439-520): no descent
        } else if (a.probes) {
            // learned entries: the first nearest of the probed rows of layer g0,
            // taken in probe order as the descent takes a list
            g0 = a.g0;
            uint32_t pid = 0;
            float pd = 0.f;
            if (lane < a.nprobe) {
                pid = a.probes[(size_t)qi * a.nprobe + lane];
                if (pid < a.nrows[g0]) pd = dist_seq_rt(a.metric, qv, a.x + (size_t)pid * a.dp, a.dp);
                else atomicOr(a.overflow, SERR_BAD_ID);
            }
            cur = __shfl_sync(FULL, pid, 0);
            cur_d = __shfl_sync(FULL, pd, 0);
            for (uint32_t j = 1; j < a.nprobe; j++) {
                const float oj = __shfl_sync(FULL, pd, j);
                const uint32_t ij = __shfl_sync(FULL, pid, j);
                if (oj < cur_d) {
                    cur_d = oj;
                    cur = ij;
                }
            }
            cmps += a.nprobe;
            if (cur >= a.nrows[g0]) cur = 0;
        } else {
            cur_d = dist_seq_rt(a.metric, qv, a.x + (size_t)cur * a.dp, a.dp);
            cmps++;
        }
        // greedy descent on the upper layers (lysearch.cpp:397-420)
        for (uint32_t g = g0; g + 1 < a.L; g++) {
            const uint64_t* off = a.off_all + a.off_base[g];
            bool moved = true;
            uint32_t moves = 0;
            while (moved) {
                moved = false;
                if (cur >= a.nrows[g] || ++moves > a.nrows[g]) {
                    if (lane == 0) atomicOr(a.overflow, cur >= a.nrows[g] ? SERR_BAD_ID : SERR_GREEDY_CAP);
                    break;
                }
                const uint64_t b = off[cur], e = off[cur + 1];  // the list of the node at loop entry
                for (uint64_t c0 = b; c0 < e; c0 += 32) {
                    uint32_t nn = 0;
                    float dd = 0.f;
                    if (c0 + lane < e) {
                        nn = a.adj_all[c0 + lane];
                        dd = dist_seq_rt(a.metric, qv, a.x + (size_t)nn * a.dp, a.dp);
                    }
                    const uint32_t cnt = (uint32_t)(e - c0 < 32 ? e - c0 : 32);
                    cmps += cnt;
                    for (uint32_t j = 0; j < cnt; j++) {
                        const float oj = __shfl_sync(FULL, dd, j);
                        const uint32_t ij = __shfl_sync(FULL, nn, j);
                        if (oj < cur_d) {
                            cur_d = oj;
                            cur = ij;
                            moved = true;
                        }
                    }
                }
            }
        }
        // beam search on the last layer (nndHNSWSrch, lysearch.cpp:236-322)
        const uint64_t* off = a.off_all + a.off_base[a.L - 1];
        uint32_t ntop = 0, ncand = 0, nvis = 1;
        bool vis_overflow = false;
        bool start_ok = true;
        if (a.flat) {
            // the getRndSds seeds of this beam width, pushed in draw order
            // (lysearch.cpp:462-472); their distances in parallel first
            const uint32_t* sd = a.flat_pool + a.flat_off[topk];
            nvis = 0;
            for (uint32_t c0 = 0; c0 < topk; c0 += 32) {
                const uint32_t cnt = min(32u, topk - c0);
                if (lane < cnt) {
                    const uint32_t id = sd[c0 + lane];
                    stage_i[lane] = id;
                    stage_d[lane] = dist_seq_rt(a.metric, qv, a.x + (size_t)id * a.dp, a.dp);
                    atomicOr(&vis[id >> 5], 1u << (id & 31));
                    if (nvis + lane < VCAP) vl[nvis + lane] = id;
                }
                __syncwarp();
                if (lane == 0)
                    for (uint32_t r = 0; r < cnt; r++) {
                        if (ncand >= CCAP) {
                            atomicOr(a.overflow, SERR_HEAP);
                            break;
                        }
                        heap_push(cand, ncand, HP{-stage_d[r], stage_i[r]});
                        heap_push(top, ntop, HP{stage_d[r], stage_i[r]});
                    }
                __syncwarp();
                nvis += cnt;
                cmps += cnt;
            }
            if (nvis > VCAP) vis_overflow = true;
        } else {
            start_ok = cur < a.nrows[a.L - 1];  // false only after a failed greedy check
            if (lane == 0 && start_ok) {
                heap_push(cand, ncand, HP{-cur_d, cur});
                heap_push(top, ntop, HP{cur_d, cur});
                atomicOr(&vis[cur >> 5], 1u << (cur & 31));
                vl[0] = cur;
            }
        }
        ncand = __shfl_sync(FULL, ncand, 0);
        ntop = __shfl_sync(FULL, ntop, 0);
        __syncwarp();
        if (!start_ok) nvis = 0;
        float lwbnd = 0.f;
        if (lane == 0 && start_ok) lwbnd = top[0].f;
        lwbnd = __shfl_sync(FULL, lwbnd, 0);
        const uint32_t nlast = a.nrows[a.L - 1];
        uint32_t expansions = 0;
        while (ncand > 0) {
            // Lane 0 alone reads the heaps and broadcasts through registers:
            // a value every lane loaded itself could be re-read after lane
            // 0's next update, and lanes that disagree would diverge.
            HP c{0.f, 0u};
            if (lane == 0) c = cand[0];
            c.f = __shfl_sync(FULL, c.f, 0);
            c.id = __shfl_sync(FULL, c.id, 0);
            if (-c.f > lwbnd) break;
            if (c.id >= nlast || ++expansions > nlast + 1) {
                if (lane == 0) atomicOr(a.overflow, c.id >= nlast ? SERR_BAD_ID : SERR_BEAM_CAP);
                break;
            }
            if (lane == 0) heap_pop(cand, ncand);
            ncand = __shfl_sync(FULL, ncand, 0);
            nexp++;
            const uint64_t b = off[c.id], e = off[c.id + 1];
            for (uint64_t c0 = b; c0 < e; c0 += 32) {
                uint32_t nn = 0;
                bool fresh = false;
                if (c0 + lane < e) {
                    nn = a.adj_all[c0 + lane];
                    if (nn < nlast) {
                        const uint32_t old = atomicOr(&vis[nn >> 5], 1u << (nn & 31));
                        fresh = !(old & (1u << (nn & 31)));
                    } else {
                        atomicOr(a.overflow, SERR_BAD_ID);
                    }
                }
                const unsigned fb = __ballot_sync(FULL, fresh);
                if (fresh) {
                    const uint32_t r = __popc(fb & ((1u << lane) - 1u));
                    if (nvis + r < VCAP) vl[nvis + r] = nn;
                    stage_d[r] = dist_seq_rt(a.metric, qv, a.x + (size_t)nn * a.dp, a.dp);
                    stage_i[r] = nn;
                }
                const uint32_t nf = __popc(fb);
                nvis += nf;
                if (nvis > VCAP) vis_overflow = true;
                cmps += nf;
                __syncwarp();
                if (lane == 0) {  // offers in list order (lysearch.cpp:284-295)
                    for (uint32_t r = 0; r < nf; r++) {
                        const float dj = stage_d[r];
                        if (top[0].f > dj || ntop < topk) {
                            if (ncand >= CCAP) {
                                atomicOr(a.overflow, SERR_HEAP);
                                continue;
                            }
                            heap_push(cand, ncand, HP{-dj, stage_i[r]});
                            heap_push(top, ntop, HP{dj, stage_i[r]});
                            if (ntop > topk) heap_pop(top, ntop);
                        }
                    }
                }
                __syncwarp();
                ncand = __shfl_sync(FULL, ncand, 0);
                ntop = __shfl_sync(FULL, ntop, 0);
                float lw = 0.f;
                if (lane == 0) lw = top[0].f;
                lwbnd = __shfl_sync(FULL, lw, 0);
            }
        }
        // results ascending, popped from the max-heap into place (lysearch.cpp:302-312);
        // the first out_k are kept
        if (lane == 0) {
            const size_t o = (size_t)qi * a.out_k;
            for (uint32_t t = ntop; t < a.out_k; t++) {
                a.out_ids[o + t] = 0xffffffffu;
                if (a.out_d) a.out_d[o + t] = 0.f;
            }
            for (int loc = (int)ntop - 1; loc >= 0; loc--) {
                if ((uint32_t)loc < a.out_k) {
                    a.out_ids[o + loc] = top[0].id;
                    if (a.out_d) a.out_d[o + loc] = top[0].f;
                }
                heap_pop(top, ntop);
            }
        }
        // clear the visited bits of this query
        if (!vis_overflow) {
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
    if (lane == 0 && a.ncmps) atomicAdd(a.ncmps, cmps / 32);
    if (lane == 0 && a.nexp) atomicAdd(a.nexp, nexp);
}
}  // namespace

int index_upload(Ctx& ctx, IndexDev& ix, const float* x, uint64_t n, uint32_t d, const nnm_layers* layers,
                 uint32_t seed, uint32_t metric) {
    cudaStream_t st = ctx.stream;
    const uint32_t dp = (d + 3) & ~3u;
    const uint32_t L = layers->nlayers;
    if (L == 0 || L > 16) {
        ctx.last_error = "search needs 1..16 layers";
        return 1;
    }
    // Layers must be nested prefixes whose ids stay inside their own layer;
    // anything else is rejected here rather than read out of bounds.
    for (uint32_t g = 0; g < L; g++) {
        const uint32_t nr = layers->nrows[g];
        if (nr == 0 || (g + 1 < L && nr > layers->nrows[g + 1]) || nr > n || !layers->off[g] ||
            (!layers->adj[g] && layers->off[g][nr] > 0)) {
            ctx.last_error = "search layers are not nested prefixes of the data set";
            return 1;
        }
        if (layers->off[g][0] != 0) {
            ctx.last_error = "layer offsets must start at 0";
            return 1;
        }
        for (uint32_t i = 0; i < nr; i++)
            if (layers->off[g][i + 1] < layers->off[g][i]) {
                ctx.last_error = "layer offsets must be non-decreasing";
                return 1;
            }
        for (uint64_t t = 0; t < layers->off[g][nr]; t++)
            if (layers->adj[g][t] >= nr) {
                ctx.last_error = "a layer lists an id outside the layer";
                return 1;
            }
    }
    // entry point: the first std::rand() after srand(seed) (lysearch.cpp:382)
    GlibcBase gb = glibc_base(seed);
    uint32_t r0;
    {
        // rand() #0 = s[310] >> 1, s[i] = s[i-3] + s[i-31]
        std::vector<uint32_t> s(gb.s, gb.s + 62);
        while (s.size() <= 310) s.push_back(s[s.size() - 3] + s[s.size() - 31]);
        r0 = s[310] >> 1;
    }
    ix.n = (uint32_t)n;
    ix.d = d;
    ix.dp = dp;
    ix.L = L;
    ix.metric = metric;
    ix.seed = seed;
    ix.entry = r0 % layers->nrows[0];
    uint64_t off_total = 0, adj_total = 0;
    for (uint32_t g = 0; g < L; g++) {
        ix.nrows[g] = layers->nrows[g];
        ix.off_base[g] = off_total;
        off_total += (uint64_t)layers->nrows[g] + 1;
        adj_total += layers->off[g][layers->nrows[g]];
    }
    NNM_CUDA_TRY(ix.x.ensure((size_t)n * dp * 4));
    NNM_CUDA_TRY(ix.off.ensure(off_total * 8));
    NNM_CUDA_TRY(ix.adj.ensure(std::max<uint64_t>(adj_total, 1) * 4));
    NNM_CUDA_TRY(ix.ctr.ensure(64));
    if (dp == d) {
        NNM_CUDA_TRY(cudaMemcpyAsync(ix.x.p, x, (size_t)n * d * 4, cudaMemcpyHostToDevice, st));
    } else {
        NNM_CUDA_TRY(cudaMemset2DAsync(ix.x.p, dp * 4, 0, dp * 4, n, st));
        NNM_CUDA_TRY(cudaMemcpy2DAsync(ix.x.p, dp * 4, x, d * 4, d * 4, n, cudaMemcpyHostToDevice, st));
    }
    // offsets rebased onto one adjacency array; the copies wait for the
    // stream's earlier work through the synchronous calls below
    NNM_CUDA_TRY(cudaStreamSynchronize(st));
    adj_total = 0;
    for (uint32_t g = 0; g < L; g++) {
        std::vector<uint64_t> off(layers->off[g], layers->off[g] + layers->nrows[g] + 1);
        for (auto& v : off) v += adj_total;
        NNM_CUDA_TRY(cudaMemcpy(ix.off.as<uint64_t>() + ix.off_base[g], off.data(), off.size() * 8,
                                cudaMemcpyHostToDevice));
        uint64_t cnt = layers->off[g][layers->nrows[g]];
        if (cnt) NNM_CUDA_TRY(cudaMemcpy(ix.adj.as<uint32_t>() + adj_total, layers->adj[g], cnt * 4, cudaMemcpyHostToDevice));
        adj_total += cnt;
    }
    return 0;
}

int index_run_exact(Ctx& ctx, IndexDev& ix, const SearchReq& r) {
    cudaStream_t st = ctx.stream;
    const uint32_t dp = ix.dp;
    int nsm = 148;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, ctx.device);
    const size_t wbytes = (size_t)dp * 4 + (size_t)(r.beam_max + 1) * 8 + 32 * 8;
    const size_t smem = (size_t)SWARPS * ((wbytes + 15) & ~(size_t)15) + 64;
    if (smem > 200 * 1024) {
        ctx.last_error = "beam too wide for shared memory at this dimension";
        return 1;
    }
    NNM_CUDA_TRY(cudaFuncSetAttribute(k_search, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 1;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_search, SWARPS * 32, smem);
    const uint32_t blocks = (uint32_t)std::min(std::max(1, per_sm), 4) * (uint32_t)nsm;
    const uint32_t words = (uint32_t)((ix.n + 31) / 32);
    const size_t slots = (size_t)blocks * SWARPS;
    if (ix.visited.bytes < slots * words * 4) {
        NNM_CUDA_TRY(ix.visited.ensure(slots * words * 4));
        NNM_CUDA_TRY(cudaMemsetAsync(ix.visited.p, 0, slots * words * 4, st));
    }
    NNM_CUDA_TRY(ix.vlist.ensure(slots * VCAP * 4));
    NNM_CUDA_TRY(ix.cand.ensure(slots * CCAP * sizeof(HP)));
    SearchArgs a{};
    a.x = ix.x.as<float>();
    a.dp = dp;
    a.metric = (int)ix.metric;
    a.L = ix.L;
    for (uint32_t g = 0; g < ix.L; g++) {
        a.off_base[g] = ix.off_base[g];
        a.nrows[g] = ix.nrows[g];
    }
    a.off_all = ix.off.as<uint64_t>();
    a.adj_all = ix.adj.as<uint32_t>();
    a.q = r.q;
    a.nq = r.nq;
    a.topk = r.beam;
    a.entry = ix.entry;
    a.n = ix.n;
    a.beams = r.beams;
    a.beam_cap = r.beam_max;
    a.out_k = r.out_k;
    a.probes = r.probes;
    a.nprobe = r.nprobe;
    a.g0 = r.g0;
    a.flat = r.flat;
    a.flat_off = r.flat_off;
    a.flat_pool = r.flat_pool;
    a.out_ids = r.out_ids;
    a.out_d = r.out_d;
    a.visited = ix.visited.as<uint32_t>();
    a.words = words;
    a.vlist = ix.vlist.as<uint32_t>();
    a.cand = ix.cand.as<HP>();
    unsigned char* c = ix.ctr.as<unsigned char>();
    a.next_q = reinterpret_cast<unsigned*>(c);
    a.overflow = reinterpret_cast<unsigned*>(c + 4);
    a.ncmps = reinterpret_cast<unsigned long long*>(c + 8);
    a.nexp = reinterpret_cast<unsigned long long*>(c + 16);
    k_search<<<blocks, SWARPS * 32, smem, st>>>(a); count_launch();
    NNM_CUDA_TRY(cudaGetLastError());
    return 0;
}

// getRndSds (lysearch.cpp:206-233) with a fresh std::mt19937(seed): k
// distinct ids of [0, N) -- what nndFlatSrch draws per query with the clock
// frozen at `seed`.
static void rnd_seeds(uint32_t seed, uint32_t k, uint32_t N, uint32_t* out) {
    if (N == k) {
        for (uint32_t i = 0; i < k; i++) out[i] = i;
        return;
    }
    std::vector<uint32_t> r(k + 1);
    gen_mt19937(seed, k + 1, r.data());
    for (uint32_t i = 0; i < k; i++) out[i] = r[i] % (N - k);
    std::sort(out, out + k);
    for (uint32_t i = 1; i < k; i++)
        if (out[i] <= out[i - 1]) out[i] = out[i - 1] + 1;
    const uint32_t off = r[k] % N;
    for (uint32_t i = 0; i < k; i++) out[i] = (uint32_t)(((uint64_t)out[i] + off) % N);
}

int index_flat_seeds(Ctx& ctx, IndexDev& ix, uint32_t beam_max) {
    const uint32_t N = ix.nrows[ix.L - 1];
    if (beam_max > N) {
        ctx.last_error = "flat search: a beam width is larger than the last layer";
        return 1;
    }
    if (ix.flat_max >= beam_max) return 0;
    // seeds of every beam width 1..beam_max, concatenated
    std::vector<uint32_t> off(beam_max + 1, 0), pool;
    pool.reserve((size_t)beam_max * (beam_max + 1) / 2);
    for (uint32_t b = 1; b <= beam_max; b++) {
        off[b] = (uint32_t)pool.size();
        pool.resize(pool.size() + b);
        rnd_seeds(ix.seed, b, N, pool.data() + off[b]);
    }
    NNM_CUDA_TRY(ix.flat_off.ensure(off.size() * 4));
    NNM_CUDA_TRY(ix.flat_pool.ensure(std::max<size_t>(pool.size(), 1) * 4));
    NNM_CUDA_TRY(cudaMemcpy(ix.flat_off.p, off.data(), off.size() * 4, cudaMemcpyHostToDevice));
    NNM_CUDA_TRY(cudaMemcpy(ix.flat_pool.p, pool.data(), pool.size() * 4, cudaMemcpyHostToDevice));
    ix.flat_max = beam_max;
    return 0;
}

int index_counters(Ctx& ctx, IndexDev& ix, uint64_t* ncmps, uint64_t* nexp) {
    unsigned long long c[3] = {0, 0, 0};
    NNM_CUDA_TRY(cudaMemcpyAsync(c, ix.ctr.p, 24, cudaMemcpyDeviceToHost, ctx.stream));
    NNM_CUDA_TRY(cudaStreamSynchronize(ctx.stream));
    if (ncmps) *ncmps = c[1];
    if (nexp) *nexp = c[2];
    const unsigned serr = (unsigned)(c[0] >> 32);  // bytes 4..7
    if (serr) {
        ctx.last_error = "search self-check failed (code " + std::to_string(serr) +
                         "; 1: candidate heap full, 2/4: loop bound, 8: id outside its layer, "
                         "32: beam width outside [out_k, beam])";
        return 6;
    }
    return 0;
}

void IndexDev::release() {
    DevBuf* all[] = {&x,     &off,   &adj,  &visited, &vlist,  &cand,     &ctr,      &qpad,
                     &beams, &probes, &hid, &scores,  &out,    &flat_off, &flat_pool};
    for (auto* b : all) b->release();
}

int search_host(Ctx& ctx, const float* x, uint64_t n, uint32_t d, const nnm_layers* layers, const float* q,
                uint64_t nq, uint32_t topk, uint32_t seed, int metric, uint32_t* out_ids, float* out_dists,
                uint64_t* ncmps) {
    cudaStream_t st = ctx.stream;
    IndexDev ix;
    int rc = index_upload(ctx, ix, x, n, d, layers, seed, (uint32_t)metric);
    if (rc) {
        ix.release();
        return rc;
    }
    const uint32_t dp = ix.dp;
    DevBuf qb, ib, db;
    auto fail = [&](int code) {
        ix.release();
        qb.release();
        ib.release();
        db.release();
        return code;
    };
#define TRY_OR_FREE(call)                                      \
    do {                                                       \
        cudaError_t e_ = (call);                               \
        if (e_ != cudaSuccess) {                               \
            ctx.last_error = cudaGetErrorString(e_);           \
            return fail(e_ == cudaErrorMemoryAllocation ? 4 : 3); \
        }                                                      \
    } while (0)
    TRY_OR_FREE(qb.ensure((size_t)nq * dp * 4 + 16));
    TRY_OR_FREE(ib.ensure((size_t)nq * topk * 4 + 16));
    TRY_OR_FREE(db.ensure((size_t)nq * topk * 4 + 16));
    if (dp == d) {
        TRY_OR_FREE(cudaMemcpyAsync(qb.p, q, (size_t)nq * d * 4, cudaMemcpyHostToDevice, st));
    } else {
        TRY_OR_FREE(cudaMemset2DAsync(qb.p, dp * 4, 0, dp * 4, nq, st));
        TRY_OR_FREE(cudaMemcpy2DAsync(qb.p, dp * 4, q, d * 4, d * 4, nq, cudaMemcpyHostToDevice, st));
    }
    SearchReq r{};
    r.q = qb.as<float>();
    r.nq = (uint32_t)nq;
    r.beam = topk;
    r.beam_max = topk;
    r.out_k = topk;
    r.out_ids = ib.as<uint32_t>();
    r.out_d = db.as<float>();
    TRY_OR_FREE(cudaMemsetAsync(ix.ctr.p, 0, 64, st));
    if ((rc = index_run_exact(ctx, ix, r))) return fail(rc);
    TRY_OR_FREE(cudaMemcpyAsync(out_ids, ib.p, (size_t)nq * topk * 4, cudaMemcpyDeviceToHost, st));
    if (out_dists) TRY_OR_FREE(cudaMemcpyAsync(out_dists, db.p, (size_t)nq * topk * 4, cudaMemcpyDeviceToHost, st));
#undef TRY_OR_FREE
    rc = index_counters(ctx, ix, ncmps, nullptr);
    return fail(rc);
}

}  // namespace nnm
