// DPG layers of the H-Merge hierarchy: LyNNDescent::dpg / DelaunayGraph
// (lynndescent.cpp:502-544, :640-713) with insert2topk (:546-623).
//
// Forward pass (per row, independent): scan the row's K-NN list in order
// and keep a neighbour b unless a kept entry l is closer to b than the row
// is (d(l,b) < d(i,b)), up to K/2 entries.  The reference never clears its
// list array between layers, so each row starts from its list of the
// previous layer.
//
// Reverse pass: the reference walks rows i = 0..N-1 in order and offers i to
// every entry of i's current list ("snapshot" S_i), subject to the list's
// capacity and an occlusion test.  Offers into row x arrive in ascending
// source order, and S_i is row i's list after the offers from rows < i, so
// S_i depends only on the snapshots of earlier rows.  The GPU computes this
// exactly by fixed-point rounds: guess the snapshots (the forward lists),
// generate all offers, replay each target's offers in source order
// (recording its snapshot when the source passes the target's own row),
// and repeat with the recorded snapshots until they stop changing.  By
// induction on the row order, round r reproduces the first r snapshots at
// least, and a fixed point equals the reference's sequential result.
#include <algorithm>
#include <cstdlib>
#include <vector>

#include "nnm_hier.h"
#include "nnm_launch.h"
#include "nnm_scan.h"

namespace nnm {
namespace {
constexpr unsigned FULL = 0xffffffffu;
constexpr int WPB = 8;
constexpr int MAXC = 80;  // list capacity limit (max(K/2, M) <= 64)
constexpr int EV_CH = 4096;

struct DpgCtr {
    unsigned int changed;
    unsigned int nbig;
    unsigned int error;
    unsigned int pad;
};

// insert2topk on a warp-shared list; run by one lane.
__device__ void list_insert(uint32_t* lid, float* ld, uint32_t* len, uint32_t nid, float dst, uint32_t maxSize) {
    uint32_t topk = *len, i, j;
    if (topk == 0) {
        lid[0] = nid;
        ld[0] = dst;
        *len = 1;
        return;
    }
    i = topk;
    if (ld[topk - 1] < dst && topk == maxSize) return;
    if (topk < maxSize && ld[topk - 1] < dst) {
        lid[topk] = nid;
        ld[topk] = dst;
        *len = topk + 1;
        return;
    }
    while (i > 0) {
        j = i - 1;
        if (ld[j] <= dst) break;
        i = j;
    }
    uint32_t l = i;
    while (l > 0) {
        j = l - 1;
        if (ld[j] < dst) break;
        if (lid[j] == nid) return;
        l = j;
    }
    if (topk < maxSize) {
        j = topk;
        *len = topk + 1;
    } else {
        j = maxSize - 1;
    }
    while (j > i) {
        lid[j] = lid[j - 1];
        ld[j] = ld[j - 1];
        --j;
    }
    lid[j] = nid;
    ld[j] = dst;
}

// True if some list entry l (first len) has d(l, b) < dst.  Exact
// sequential distances, one list entry per lane.
__device__ bool occluded(const float* x, uint32_t dp, int metric, const uint32_t* lid, uint32_t len, uint32_t b,
                         float dst) {
    int lane = threadIdx.x & 31;
    bool bad = false;
    for (uint32_t l = lane; l < len; l += 32)
        if (dist_seq_rt(metric, x + (size_t)lid[l] * dp, x + (size_t)b * dp, dp) < dst) bad = true;
    return __any_sync(FULL, bad);
}

struct FwdArgs {
    const float* x;
    uint32_t dp;
    int metric;
    const uint32_t* pid;
    const float* pdist;
    uint32_t K, N, C, Mo;
    const uint32_t *gid, *glen;
    const float* gdist;
    uint32_t *g1id, *g1len;
    float* g1dist;
};

__global__ void k_dpg_forward(FwdArgs a) {
    __shared__ uint32_t sid[WPB][MAXC];
    __shared__ float sd[WPB][MAXC];
    __shared__ uint32_t slen[WPB];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t i = blockIdx.x * WPB + w;
    if (i >= a.N) return;
    if (lane == 0) slen[w] = a.glen[i];
    __syncwarp();
    for (uint32_t l = lane; l < slen[w]; l += 32) {
        sid[w][l] = a.gid[(size_t)i * a.C + l];
        sd[w][l] = a.gdist[(size_t)i * a.C + l];
    }
    __syncwarp();
    for (uint32_t j = 0; j < a.K; j++) {
        const uint32_t len = __shfl_sync(FULL, slen[w], 0);  // one value for the whole warp
        if (len > a.Mo) break;
        uint32_t nb = a.pid[(size_t)i * a.K + j] & ID_MASK;
        float dst = a.pdist[(size_t)i * a.K + j];  // = distfunc(i, nb): the same exact value
        bool bad = occluded(a.x, a.dp, a.metric, sid[w], len, nb, dst);
        __syncwarp();  // every lane has read the list before lane 0 changes it
        if (!bad && lane == 0) list_insert(sid[w], sd[w], &slen[w], nb, dst, a.Mo);
        __syncwarp();
    }
    for (uint32_t l = lane; l < slen[w]; l += 32) {
        a.g1id[(size_t)i * a.C + l] = sid[w][l];
        a.g1dist[(size_t)i * a.C + l] = sd[w][l];
    }
    if (lane == 0) a.g1len[i] = slen[w];
}

__global__ void k_ev_count(const uint32_t* sid, const uint32_t* slen, uint32_t N, uint32_t C, uint32_t* ecnt) {
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t i = blockIdx.x * WPB + w;
    if (i >= N) return;
    uint32_t len = slen[i];
    for (uint32_t t = lane; t < len; t += 32) atomicAdd(&ecnt[sid[(size_t)i * C + t]], 1u);
}

__global__ void k_ev_fill(const uint32_t* sid, const float* sdist, const uint32_t* slen, uint32_t N, uint32_t C,
                          const uint64_t* eoff, uint32_t* ecur, unsigned long long* ev) {
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t i = blockIdx.x * WPB + w;
    if (i >= N) return;
    uint32_t len = slen[i];
    for (uint32_t t = lane; t < len; t += 32) {
        uint32_t x = sid[(size_t)i * C + t];
        unsigned long long v = ((unsigned long long)i << 32) | __float_as_uint(sdist[(size_t)i * C + t]);
        ev[eoff[x] + atomicAdd(&ecur[x], 1u)] = v;
    }
}

// Offers into each target sorted by source row (sources are distinct).
__global__ void k_ev_sort_small(const uint64_t* eoff, unsigned long long* ev, uint32_t N, uint32_t* big,
                                DpgCtr* ctr) {
    const uint32_t x = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (x >= N) return;
    uint64_t lo = eoff[x];
    uint32_t len = (uint32_t)(eoff[x + 1] - lo);
    if (len <= 1) return;
    if (len > 32) {
        if (lane == 0) big[atomicAdd(&ctr->nbig, 1u)] = x;
        return;
    }
    unsigned long long v = lane < (int)len ? ev[lo + lane] : ~0ull;
    for (int k = 2; k <= 32; k <<= 1)
        for (int j = k >> 1; j > 0; j >>= 1) {
            unsigned long long o = __shfl_xor_sync(FULL, v, j);
            bool take_min = ((lane & j) == 0) == ((lane & k) == 0);
            if (take_min ? (o < v) : (o > v)) v = o;
        }
    if (lane < (int)len) ev[lo + lane] = v;
}

__global__ void k_ev_sort_big(const uint64_t* eoff, unsigned long long* ev, unsigned long long* scr,
                              const uint32_t* big, const DpgCtr* ctr) {
    __shared__ unsigned long long sh[EV_CH];
    const uint32_t nbig = ctr->nbig;
    for (uint32_t bi = blockIdx.x; bi < nbig; bi += gridDim.x) {
        const uint32_t x = big[bi];
        const uint64_t lo = eoff[x];
        const uint32_t len = (uint32_t)(eoff[x + 1] - lo);
        unsigned long long* seg = ev + lo;
        for (uint32_t cs = 0; cs < len; cs += EV_CH) {
            uint32_t m = min((uint32_t)EV_CH, len - cs), P = 1;
            while (P < m) P <<= 1;
            for (uint32_t i = threadIdx.x; i < P; i += blockDim.x) sh[i] = i < m ? seg[cs + i] : ~0ull;
            __syncthreads();
            for (uint32_t k = 2; k <= P; k <<= 1)
                for (uint32_t j = k >> 1; j > 0; j >>= 1) {
                    for (uint32_t i = threadIdx.x; i < P; i += blockDim.x) {
                        uint32_t ix = i ^ j;
                        if (ix > i) {
                            unsigned long long p = sh[i], q = sh[ix];
                            bool asc = (i & k) == 0;
                            if (asc ? p > q : p < q) {
                                sh[i] = q;
                                sh[ix] = p;
                            }
                        }
                    }
                    __syncthreads();
                }
            for (uint32_t i = threadIdx.x; i < m; i += blockDim.x) seg[cs + i] = sh[i];
            __syncthreads();
        }
        unsigned long long* src = seg;
        unsigned long long* dst = scr + lo;
        for (uint32_t w = EV_CH; w < len; w <<= 1) {
            for (uint32_t i = threadIdx.x; i < len; i += blockDim.x) {
                uint32_t run = i / w, rs = run * w, pb = (run & ~1u) * w;
                uint32_t os = (run & 1u) ? rs - w : rs + w;
                if (os > len) os = len;
                uint32_t oe = min(os + w, len);
                unsigned long long key = src[i];
                uint32_t l2 = os, h2 = oe;
                while (l2 < h2) {
                    uint32_t mid = (l2 + h2) >> 1;
                    if (src[mid] < key) l2 = mid + 1;
                    else h2 = mid;
                }
                dst[pb + (i - rs) + (l2 - os)] = key;
            }
            __syncthreads();
            unsigned long long* t = src;
            src = dst;
            dst = t;
        }
        if (src != seg)
            for (uint32_t i = threadIdx.x; i < len; i += blockDim.x) seg[i] = src[i];
        __syncthreads();
    }
}

struct RevArgs {
    const float* x;
    uint32_t dp;
    int metric;
    uint32_t N, C, maxM;
    const uint32_t *g1id, *g1len;
    const float* g1dist;
    const uint64_t* eoff;
    const unsigned long long* ev;
    const uint32_t *sid, *slen;   // guessed snapshots
    uint32_t *tid, *tlen;         // recorded snapshots
    float* tdist;
    uint32_t *gid, *glen;         // final lists
    float* gdist;
    DpgCtr* ctr;
};

__global__ void k_dpg_reverse(RevArgs a) {
    __shared__ uint32_t sid[WPB][MAXC];
    __shared__ float sd[WPB][MAXC];
    __shared__ uint32_t slen[WPB];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t x = blockIdx.x * WPB + w;
    if (x >= a.N) return;
    if (lane == 0) slen[w] = a.g1len[x];
    __syncwarp();
    for (uint32_t l = lane; l < slen[w]; l += 32) {
        sid[w][l] = a.g1id[(size_t)x * a.C + l];
        sd[w][l] = a.g1dist[(size_t)x * a.C + l];
    }
    __syncwarp();
    bool snapped = false;
    const uint64_t lo = a.eoff[x], hi = a.eoff[x + 1];
    for (uint64_t e = lo; e <= hi; e++) {
        const bool end = e == hi;
        unsigned long long v = end ? 0ull : a.ev[e];
        const uint32_t s = (uint32_t)(v >> 32);
        if (!snapped && (end || s >= x)) {  // list of row x when the walk reaches row x
            snapped = true;
            const uint32_t L = __shfl_sync(FULL, slen[w], 0);
            for (uint32_t l = lane; l < L; l += 32) {
                a.tid[(size_t)x * a.C + l] = sid[w][l];
                a.tdist[(size_t)x * a.C + l] = sd[w][l];
            }
            bool diff = L != a.slen[x];
            for (uint32_t l = lane; l < L && !diff; l += 32)
                if (a.sid[(size_t)x * a.C + l] != sid[w][l]) diff = true;
            diff = __any_sync(FULL, diff);
            if (lane == 0) {
                a.tlen[x] = L;
                if (diff) atomicAdd(&a.ctr->changed, 1u);
            }
        }
        if (end) break;
        const float dd = __uint_as_float((uint32_t)(v & 0xffffffffu));
        const uint32_t len = __shfl_sync(FULL, slen[w], 0);
        bool ok = true;
        if (len >= a.maxM) ok = !occluded(a.x, a.dp, a.metric, sid[w], len, s, dd);
        __syncwarp();  // every lane has read the list before lane 0 changes it
        if (ok && lane == 0) list_insert(sid[w], sd[w], &slen[w], s, dd, a.maxM);
        __syncwarp();
    }
    for (uint32_t l = lane; l < slen[w]; l += 32) {
        a.gid[(size_t)x * a.C + l] = sid[w][l];
        a.gdist[(size_t)x * a.C + l] = sd[w][l];
    }
    if (lane == 0) a.glen[x] = slen[w];
}

unsigned nblk(size_t n, unsigned per) { return (unsigned)((n + per - 1) / per); }
}  // namespace

int dpg_init(Ctx& ctx, DpgState& s, uint32_t n_cap, uint32_t K, uint32_t M) {
    s.K = K;
    s.M = M;
    s.n_cap = n_cap;
    s.cap = std::max(K / 2, M) + 1;
    if (s.cap > (uint32_t)MAXC) {
        ctx.last_error = "DPG list capacity exceeds the device limit";
        return 1;
    }
    const size_t nc = (size_t)n_cap * s.cap;
    DevBuf* lists[] = {&s.gid, &s.gdist, &s.g1id, &s.g1dist, &s.sid, &s.sdist, &s.tid, &s.tdist};
    for (auto* b : lists) NNM_CUDA_TRY(b->ensure(nc * 4));
    DevBuf* lens[] = {&s.glen, &s.g1len, &s.slen, &s.tlen, &s.ecnt, &s.ecur, &s.bigseg};
    for (auto* b : lens) NNM_CUDA_TRY(b->ensure(((size_t)n_cap + 1) * 4));
    NNM_CUDA_TRY(s.eoff.ensure(((size_t)n_cap + 1) * 8));
    NNM_CUDA_TRY(s.ev.ensure(nc * 8 + 64));
    NNM_CUDA_TRY(s.escr.ensure(nc * 8 + 64));
    NNM_CUDA_TRY(s.counters.ensure(sizeof(DpgCtr) + 64));
    NNM_CUDA_TRY(s.tmp.ensure(scan_temp_elems((size_t)n_cap + 1) * 8 + 64));
    NNM_CUDA_TRY(cudaMemsetAsync(s.glen.p, 0, ((size_t)n_cap + 1) * 4, ctx.stream));
    s.rows = 0;
    return 0;
}

int dpg_layer(Ctx& ctx, DpgState& s, GraphDev& g, nnm_layers* out) {
    cudaStream_t st = ctx.stream;
    const uint32_t N = g.n, C = s.cap;
    const uint32_t Mo = g.K / 2;                               // lynndescent.cpp:520
    const uint32_t maxM = (N == g.n_cap) ? s.M : s.M / 2;      // lynndescent.cpp:523-534
    DpgCtr* ctr = s.counters.as<DpgCtr>();
    FwdArgs fa{g.x, g.dp, g.metric, g.pid, g.pdist, g.K, N, C, Mo, s.gid.as<uint32_t>(), s.glen.as<uint32_t>(),
               s.gdist.as<float>(), s.g1id.as<uint32_t>(), s.g1len.as<uint32_t>(), s.g1dist.as<float>()};
    k_dpg_forward<<<nblk(N, WPB), WPB * 32, 0, st>>>(fa); count_launch();
    // initial guess: snapshots = forward lists
    NNM_CUDA_TRY(cudaMemcpyAsync(s.sid.p, s.g1id.p, (size_t)N * C * 4, cudaMemcpyDeviceToDevice, st));
    NNM_CUDA_TRY(cudaMemcpyAsync(s.sdist.p, s.g1dist.p, (size_t)N * C * 4, cudaMemcpyDeviceToDevice, st));
    NNM_CUDA_TRY(cudaMemcpyAsync(s.slen.p, s.g1len.p, (size_t)N * 4, cudaMemcpyDeviceToDevice, st));
    DpgCtr h;
    uint32_t rounds = 0;
    for (;;) {
        rounds++;
        NNM_CUDA_TRY(cudaMemsetAsync(ctr, 0, sizeof(DpgCtr), st));
        NNM_CUDA_TRY(cudaMemsetAsync(s.ecnt.p, 0, (size_t)N * 4, st));
        NNM_CUDA_TRY(cudaMemsetAsync(s.ecur.p, 0, (size_t)N * 4, st));
        k_ev_count<<<nblk(N, WPB), WPB * 32, 0, st>>>(s.sid.as<uint32_t>(), s.slen.as<uint32_t>(), N, C,
                                                         s.ecnt.as<uint32_t>()); count_launch();
        NNM_CUDA_TRY(exclusive_scan(s.ecnt.as<uint32_t>(), s.eoff.as<uint64_t>(), N, s.tmp.as<uint64_t>(), nullptr, st));
        k_ev_fill<<<nblk(N, WPB), WPB * 32, 0, st>>>(s.sid.as<uint32_t>(), s.sdist.as<float>(), s.slen.as<uint32_t>(),
                                                        N, C, s.eoff.as<uint64_t>(), s.ecur.as<uint32_t>(),
                                                        s.ev.as<unsigned long long>()); count_launch();
        k_ev_sort_small<<<nblk(N, 8), 256, 0, st>>>(s.eoff.as<uint64_t>(), s.ev.as<unsigned long long>(), N,
                                                    s.bigseg.as<uint32_t>(), ctr); count_launch();
        k_ev_sort_big<<<296, 512, 0, st>>>(s.eoff.as<uint64_t>(), s.ev.as<unsigned long long>(),
                                           s.escr.as<unsigned long long>(), s.bigseg.as<uint32_t>(), ctr); count_launch();
        RevArgs ra{g.x, g.dp, g.metric, N, C, maxM, s.g1id.as<uint32_t>(), s.g1len.as<uint32_t>(),
                   s.g1dist.as<float>(), s.eoff.as<uint64_t>(), s.ev.as<unsigned long long>(),
                   s.sid.as<uint32_t>(), s.slen.as<uint32_t>(), s.tid.as<uint32_t>(), s.tlen.as<uint32_t>(),
                   s.tdist.as<float>(), s.gid.as<uint32_t>(), s.glen.as<uint32_t>(), s.gdist.as<float>(), ctr};
        k_dpg_reverse<<<nblk(N, WPB), WPB * 32, 0, st>>>(ra); count_launch();
        NNM_CUDA_TRY(cudaMemcpyAsync(&h, ctr, sizeof(DpgCtr), cudaMemcpyDeviceToHost, st));
        NNM_CUDA_TRY(cudaStreamSynchronize(st));
        NNM_CUDA_TRY(cudaGetLastError());
        if (h.changed == 0) break;
        if (rounds > N + 1) {
            ctx.last_error = "DPG reverse pass did not reach its fixed point";
            return 6;
        }
        std::swap(s.sid, s.tid);
        std::swap(s.sdist, s.tdist);
        std::swap(s.slen, s.tlen);
    }
    s.last_rounds = rounds;
    s.rows = N;
    if (out && out->nlayers < 16) {
        std::vector<uint32_t> len(N), ids((size_t)N * C);
        NNM_CUDA_TRY(cudaStreamSynchronize(ctx.stream));  // the plain copies below do not order with it
        NNM_CUDA_TRY(cudaMemcpy(len.data(), s.glen.p, (size_t)N * 4, cudaMemcpyDeviceToHost));
        NNM_CUDA_TRY(cudaMemcpy(ids.data(), s.gid.p, (size_t)N * C * 4, cudaMemcpyDeviceToHost));
        uint32_t L = out->nlayers;
        uint64_t* off = static_cast<uint64_t*>(std::malloc(sizeof(uint64_t) * ((size_t)N + 1)));
        off[0] = 0;
        for (uint32_t i = 0; i < N; i++) off[i + 1] = off[i] + len[i];
        uint32_t* adj = static_cast<uint32_t*>(std::malloc(sizeof(uint32_t) * std::max<uint64_t>(off[N], 1)));
        for (uint32_t i = 0; i < N; i++)
            for (uint32_t j = 0; j < len[i]; j++) adj[off[i] + j] = ids[(size_t)i * C + j];
        out->nrows[L] = N;
        out->off[L] = off;
        out->adj[L] = adj;
        out->nlayers = L + 1;
    }
    return 0;
}

}  // namespace nnm
