// Batched LySearch (lysearch.cpp:363-437 with nndHNSWSrch :236-322).
//
// One warp per query, persistent warps pulling queries from a counter so
// that queries of different beam widths balance.  Per query:
//   - entry point: one global id, rand() % |layer 0| after srand(seed)
//     (lysearch.cpp:382);
//   - greedy 1-NN descent through layers 0..L-2 (lysearch.cpp:397-420): the
//     distances of a node's neighbours are computed in parallel, one
//     neighbour per lane, and the moves are then applied in list order, as
//     the reference's loop does;
//   - best-first beam search on the last layer: the reference's result heap
//     of size `topk` and candidate heap become one sorted shared-memory list
//     with an "expanded" mark; the next node expanded is the closest
//     unexpanded one, and the search ends when none is left (every
//     candidate the reference could still pop lies beyond its worst result).
//     Neighbours are visited once per query (a per-warp bitmap in HBM,
//     cleared through the visited list afterwards) and offered in list
//     order.
// Distances are the reference's sequential float sums (one lane per
// distance), so every distance equals vmath.cpp:56-88 bit for bit; only the
// order among exactly equal distances can differ from the reference's heaps.
#include <algorithm>
#include <vector>

#include "nnm_hier.h"

namespace nnm {
namespace {
constexpr unsigned FULL = 0xffffffffu;
constexpr int SWARPS = 4;        // warps per block
constexpr uint32_t VCAP = 16384; // visited-list capacity per warp slot

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
    uint32_t* out_ids;
    float* out_d;
    uint32_t* visited;  // per warp slot: ceil(n/32) words
    uint32_t words;
    uint32_t* vlist;    // per warp slot: VCAP ids
    unsigned* next_q;
    unsigned long long* ncmps;
};

__device__ __forceinline__ float qdist(int metric, const float* qv, const float* xr, uint32_t dp) {
    return dist_seq_rt(metric, qv, xr, dp);
}

__global__ void k_search(SearchArgs a) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t slot = blockIdx.x * SWARPS + w;
    float* qv = reinterpret_cast<float*>(smem) + (size_t)w * a.dp;
    const size_t rstride = ((size_t)a.topk * 9 + 15) & ~(size_t)15;  // keeps every warp's arrays aligned
    unsigned char* rbase = smem + (size_t)SWARPS * a.dp * 4 + (size_t)w * rstride;
    float* rd = reinterpret_cast<float*>(rbase);
    uint32_t* rid = reinterpret_cast<uint32_t*>(rbase + (size_t)a.topk * 4);
    unsigned char* rex = rbase + (size_t)a.topk * 8;
    uint32_t* vis = a.visited + (size_t)slot * a.words;
    uint32_t* vl = a.vlist + (size_t)slot * VCAP;
    unsigned long long cmps = 0;
    for (;;) {
        unsigned qi = 0;
        if (lane == 0) qi = atomicAdd(a.next_q, 1u);
        qi = __shfl_sync(FULL, qi, 0);
        if (qi >= a.nq) break;
        for (uint32_t t = lane; t < a.dp; t += 32) qv[t] = a.q[(size_t)qi * a.dp + t];
        __syncwarp();
        uint32_t cur = a.entry;
        float cur_d = qdist(a.metric, qv, a.x + (size_t)cur * a.dp, a.dp);
        cmps++;
        // greedy descent on the upper layers
        for (uint32_t g = 0; g + 1 < a.L; g++) {
            const uint64_t* off = a.off_all + a.off_base[g];
            bool moved = true;
            while (moved) {
                moved = false;
                const uint64_t b = off[cur], e = off[cur + 1];  // the list of the node at loop entry
                for (uint64_t c0 = b; c0 < e; c0 += 32) {
                    uint32_t nn = 0;
                    float dd = 0.f;
                    if (c0 + lane < e) {
                        nn = a.adj_all[c0 + lane];
                        dd = qdist(a.metric, qv, a.x + (size_t)nn * a.dp, a.dp);
                    }
                    uint32_t cnt = (uint32_t)(e - c0 < 32 ? e - c0 : 32);
                    cmps += cnt;
                    for (uint32_t j = 0; j < cnt; j++) {
                        float oj = __shfl_sync(FULL, dd, j);
                        uint32_t ij = __shfl_sync(FULL, nn, j);
                        if (oj < cur_d) {
                            cur_d = oj;
                            cur = ij;
                            moved = true;
                        }
                    }
                }
            }
        }
        // beam search on the last layer
        const uint64_t* off = a.off_all + a.off_base[a.L - 1];
        uint32_t size = 1, cursor = 0, nvis = 0;
        bool overflow = false;
        if (lane == 0) {
            rd[0] = cur_d;
            rid[0] = cur;
            rex[0] = 0;
            atomicOr(&vis[cur >> 5], 1u << (cur & 31));
            vl[0] = cur;
        }
        nvis = 1;
        __syncwarp();
        for (;;) {
            // closest unexpanded entry
            uint32_t u = 0xffffffffu;
            for (uint32_t c0 = cursor; c0 < size; c0 += 32) {
                bool un = c0 + lane < size && rex[c0 + lane] == 0;
                unsigned bal = __ballot_sync(FULL, un);
                if (bal) {
                    u = c0 + __ffs(bal) - 1;
                    break;
                }
            }
            if (u == 0xffffffffu) break;
            cursor = u;
            if (lane == 0) rex[u] = 1;
            const uint32_t c = rid[u];
            __syncwarp();
            const uint64_t b = off[c], e = off[c + 1];
            for (uint64_t c0 = b; c0 < e; c0 += 32) {
                uint32_t nn = 0;
                float dd = 0.f;
                bool fresh = false;
                if (c0 + lane < e) {
                    nn = a.adj_all[c0 + lane];
                    uint32_t old = atomicOr(&vis[nn >> 5], 1u << (nn & 31));
                    fresh = !(old & (1u << (nn & 31)));
                }
                // two lanes cannot claim the same id: a node's list has distinct ids
                unsigned fb = __ballot_sync(FULL, fresh);
                if (fresh) {
                    uint32_t r = nvis + __popc(fb & ((1u << lane) - 1u));
                    if (r < VCAP) vl[r] = nn;
                    dd = qdist(a.metric, qv, a.x + (size_t)nn * a.dp, a.dp);
                }
                nvis += __popc(fb);
                if (nvis > VCAP) overflow = true;
                cmps += __popc(fb);
                // offer the fresh neighbours in list order
                while (fb) {
                    const int j = __ffs(fb) - 1;
                    fb &= fb - 1;
                    const float dj = __shfl_sync(FULL, dd, j);
                    const uint32_t ij = __shfl_sync(FULL, nn, j);
                    const bool full = size >= a.topk;
                    if (full && !(dj < rd[size - 1])) continue;
                    // position after all entries with distance <= dj
                    uint32_t pos = 0;
                    for (uint32_t c1 = 0; c1 < size; c1 += 32) {
                        bool le = c1 + lane < size && rd[c1 + lane] <= dj;
                        pos += __popc(__ballot_sync(FULL, le));
                    }
                    const uint32_t nsz = full ? size : size + 1;
                    // shift [pos, nsz-1) right by one, back to front in lane chunks
                    for (int c1 = (int)nsz - 2; c1 >= (int)pos; c1 -= 32) {
                        int i0 = c1 - lane;
                        float vd = 0.f;
                        uint32_t vi = 0;
                        unsigned char ve = 0;
                        bool act = i0 >= (int)pos;
                        if (act) {
                            vd = rd[i0];
                            vi = rid[i0];
                            ve = rex[i0];
                        }
                        __syncwarp();
                        if (act) {
                            rd[i0 + 1] = vd;
                            rid[i0 + 1] = vi;
                            rex[i0 + 1] = ve;
                        }
                        __syncwarp();
                    }
                    if (lane == 0) {
                        rd[pos] = dj;
                        rid[pos] = ij;
                        rex[pos] = 0;
                    }
                    size = nsz;
                    if (pos < cursor) cursor = pos;
                    __syncwarp();
                }
            }
        }
        for (uint32_t t = lane; t < a.topk; t += 32) {
            a.out_ids[(size_t)qi * a.topk + t] = t < size ? rid[t] : 0xffffffffu;
            if (a.out_d) a.out_d[(size_t)qi * a.topk + t] = t < size ? rd[t] : 0.f;
        }
        // clear the visited bits of this query
        if (!overflow) {
            for (uint32_t t = lane; t < nvis; t += 32) {
                uint32_t id = vl[t];
                atomicAnd(&vis[id >> 5], ~(1u << (id & 31)));
            }
        } else {
            for (uint32_t t = lane; t < a.words; t += 32) vis[t] = 0;
        }
        __syncwarp();
    }
    for (int o = 16; o > 0; o >>= 1) cmps += __shfl_xor_sync(FULL, cmps, o);
    if (lane == 0 && a.ncmps) atomicAdd(a.ncmps, cmps / 32);
}
}  // namespace

int search_host(Ctx& ctx, const float* x, uint64_t n, uint32_t d, const nnm_layers* layers, const float* q,
                uint64_t nq, uint32_t topk, uint32_t seed, int metric, uint32_t* out_ids, float* out_dists,
                uint64_t* ncmps) {
    cudaStream_t st = ctx.stream;
    const uint32_t dp = (d + 3) & ~3u;
    const uint32_t L = layers->nlayers;
    // entry point: the first std::rand() after srand(seed) (lysearch.cpp:382)
    GlibcBase gb = glibc_base(seed);
    uint32_t r0;
    {
        // rand() #0 = s[310] >> 1, s[i] = s[i-3] + s[i-31]
        std::vector<uint32_t> s(gb.s, gb.s + 62);
        while (s.size() <= 310) s.push_back(s[s.size() - 3] + s[s.size() - 31]);
        r0 = s[310] >> 1;
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
    const uint32_t entry = r0 % layers->nrows[0];
    SearchArgs a{};
    a.dp = dp;
    a.metric = metric;
    a.L = L;
    uint64_t off_total = 0, adj_total = 0;
    for (uint32_t g = 0; g < L; g++) {
        a.off_base[g] = off_total;
        off_total += (uint64_t)layers->nrows[g] + 1;
        adj_total += layers->off[g][layers->nrows[g]];
    }
    // one device buffer: vectors | queries | offsets | adjacency
    DevBuf xb, qb, ob, ab, ib, db, vb, lb, cb;
    NNM_CUDA_TRY(xb.ensure((size_t)n * dp * 4));
    NNM_CUDA_TRY(qb.ensure((size_t)nq * dp * 4 + 16));
    NNM_CUDA_TRY(ob.ensure(off_total * 8));
    NNM_CUDA_TRY(ab.ensure(std::max<uint64_t>(adj_total, 1) * 4));
    NNM_CUDA_TRY(ib.ensure((size_t)nq * topk * 4 + 16));
    NNM_CUDA_TRY(db.ensure((size_t)nq * topk * 4 + 16));
    NNM_CUDA_TRY(cb.ensure(64));
    if (dp == d) {
        NNM_CUDA_TRY(cudaMemcpyAsync(xb.p, x, (size_t)n * d * 4, cudaMemcpyHostToDevice, st));
        NNM_CUDA_TRY(cudaMemcpyAsync(qb.p, q, (size_t)nq * d * 4, cudaMemcpyHostToDevice, st));
    } else {
        NNM_CUDA_TRY(cudaMemset2DAsync(xb.p, dp * 4, 0, dp * 4, n, st));
        NNM_CUDA_TRY(cudaMemcpy2DAsync(xb.p, dp * 4, x, d * 4, d * 4, n, cudaMemcpyHostToDevice, st));
        NNM_CUDA_TRY(cudaMemset2DAsync(qb.p, dp * 4, 0, dp * 4, nq, st));
        NNM_CUDA_TRY(cudaMemcpy2DAsync(qb.p, dp * 4, q, d * 4, d * 4, nq, cudaMemcpyHostToDevice, st));
    }
    adj_total = 0;
    for (uint32_t g = 0; g < L; g++) {
        std::vector<uint64_t> off(layers->off[g], layers->off[g] + layers->nrows[g] + 1);
        for (auto& v : off) v += adj_total;
        NNM_CUDA_TRY(cudaMemcpy(ob.as<uint64_t>() + a.off_base[g], off.data(), off.size() * 8, cudaMemcpyHostToDevice));
        uint64_t cnt = layers->off[g][layers->nrows[g]];
        if (cnt) NNM_CUDA_TRY(cudaMemcpy(ab.as<uint32_t>() + adj_total, layers->adj[g], cnt * 4, cudaMemcpyHostToDevice));
        adj_total += cnt;
    }
    int nsm = 148;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, ctx.device);
    const size_t smem = (size_t)SWARPS * dp * 4 + (size_t)SWARPS * (((size_t)topk * 9 + 15) & ~(size_t)15) + 64;
    if (smem > 200 * 1024) {
        ctx.last_error = "beam too wide for shared memory at this dimension";
        return 1;
    }
    NNM_CUDA_TRY(cudaFuncSetAttribute(k_search, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 1;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_search, SWARPS * 32, smem);
    const uint32_t blocks = (uint32_t)std::min(std::max(1, per_sm), 8) * (uint32_t)nsm;
    const uint32_t words = (uint32_t)((n + 31) / 32);
    const size_t slots = (size_t)blocks * SWARPS;
    NNM_CUDA_TRY(vb.ensure(slots * words * 4));
    NNM_CUDA_TRY(lb.ensure(slots * VCAP * 4));
    NNM_CUDA_TRY(cudaMemsetAsync(vb.p, 0, slots * words * 4, st));
    NNM_CUDA_TRY(cudaMemsetAsync(cb.p, 0, 64, st));
    a.x = xb.as<float>();
    a.off_all = ob.as<uint64_t>();
    a.adj_all = ab.as<uint32_t>();
    a.q = qb.as<float>();
    a.nq = (uint32_t)nq;
    a.topk = topk;
    a.entry = entry;
    a.n = (uint32_t)n;
    a.out_ids = ib.as<uint32_t>();
    a.out_d = db.as<float>();
    a.visited = vb.as<uint32_t>();
    a.words = words;
    a.vlist = lb.as<uint32_t>();
    a.next_q = cb.as<unsigned>();
    a.ncmps = reinterpret_cast<unsigned long long*>(cb.as<unsigned char>() + 8);
    k_search<<<blocks, SWARPS * 32, smem, st>>>(a);
    NNM_CUDA_TRY(cudaGetLastError());
    NNM_CUDA_TRY(cudaMemcpyAsync(out_ids, ib.p, (size_t)nq * topk * 4, cudaMemcpyDeviceToHost, st));
    if (out_dists) NNM_CUDA_TRY(cudaMemcpyAsync(out_dists, db.p, (size_t)nq * topk * 4, cudaMemcpyDeviceToHost, st));
    unsigned long long c = 0;
    NNM_CUDA_TRY(cudaMemcpyAsync(&c, a.ncmps, 8, cudaMemcpyDeviceToHost, st));
    NNM_CUDA_TRY(cudaStreamSynchronize(st));
    if (ncmps) *ncmps = c;
    DevBuf* all[] = {&xb, &qb, &ob, &ab, &ib, &db, &vb, &lb, &cb};
    for (auto* b : all) b->release();
    return 0;
}

}  // namespace nnm
