// Batched LySearch for callers that cannot allocate device memory.
//
// Who needs it: code that runs where cudaMalloc is unavailable or not
// allowed -- inside a memory pool owned by another framework, a serving
// process with a fixed memory budget checked at start-up, or a caller that
// must not trigger the implicit synchronisation of cudaMalloc/cudaFree on
// its latency path.  Such callers already hold the vectors, the hierarchy,
// the queries and the output arrays in device memory and pass them in.
//
// The kernel is the search of search.cu (same greedy descent, same exact
// libstdc++ heap steps, same results), with its per-warp scratch -- visited
// bitmaps, visited lists, candidate heaps and the call's counters -- in
// `g_noalloc_scratch`, a file-scope __device__ array of NA_SCRATCH_BYTES
// (about 16 MiB) that every GPU which loads the library keeps until the
// process exits.  Host code never passes that name to a kernel: on the host
// it only stands for the symbol, so the device address is fetched once per
// device with cudaGetSymbolAddress and cached.
//
// Limits (rejected with NNM_ERR_INVALID): the last layer has at most
// NA_MAX_ROWS rows, topk <= NA_MAX_TOPK, d <= NA_MAX_DIM.  A query whose
// candidate heap would exceed NA_CCAP entries fails the call with
// NNM_ERR_CAPACITY.  All calls share the one array, so calls that overlap on
// the GPU (two streams, two host threads) race and must not be issued.
#include <cstdint>
#include <cstring>
#include <mutex>

#include "../../include/nnm.h"
#include "nnm_common.cuh"
#include "nnm_launch.h"

namespace nnm {
namespace {

constexpr unsigned FULL = 0xffffffffu;
constexpr uint32_t NA_WARPS = 4;              // warps per block
constexpr uint32_t NA_SLOTS = 64;             // concurrent queries (warp slots)
constexpr uint32_t NA_MAX_ROWS = 1u << 20;    // visited-bitmap capacity of a slot
constexpr uint32_t NA_VCAP = 8192;            // visited-list capacity of a slot
constexpr uint32_t NA_CCAP = 12288;           // candidate-heap capacity of a slot
constexpr uint32_t NA_MAX_TOPK = 1024;
constexpr uint32_t NA_MAX_DIM = 4096;
constexpr uint32_t NA_WORDS = NA_MAX_ROWS / 32;
constexpr size_t NA_HEADER = 256;

struct NaHP {
    float f;
    uint32_t id;
};

struct NaSlot {
    uint32_t visited[NA_WORDS];
    uint32_t vlist[NA_VCAP];
    NaHP cand[NA_CCAP];
};

struct NaHeader {
    unsigned next_q;
    unsigned err;
    unsigned long long ncmps;
};

constexpr size_t NA_SCRATCH_BYTES = NA_HEADER + (size_t)NA_SLOTS * sizeof(NaSlot);

__device__ __align__(256) unsigned char g_noalloc_scratch[NA_SCRATCH_BYTES];

enum : unsigned { NA_ERR_HEAP = 1u, NA_ERR_LOOP = 2u, NA_ERR_ID = 4u };

__device__ __forceinline__ void na_push(NaHP* h, uint32_t& n, NaHP v) {
    int hole = (int)n++;
    int parent = (hole - 1) / 2;
    while (hole > 0 && h[parent].f < v.f) {
        h[hole] = h[parent];
        hole = parent;
        parent = (hole - 1) / 2;
    }
    h[hole] = v;
}

__device__ __forceinline__ void na_pop(NaHP* h, uint32_t& n) {
    if (n == 0) return;
    if (n > 1) {
        const int len = (int)n - 1;
        NaHP v = h[len];
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

struct NaArgs {
    const float* x;
    uint32_t dp, d;
    int metric;
    uint32_t L;
    const uint64_t* off[16];
    const uint32_t* adj[16];
    uint32_t nrows[16];
    const float* q;
    uint32_t nq, topk, entry;
    uint32_t* out_ids;
    float* out_d;
    unsigned char* scratch;  // device address of g_noalloc_scratch
};

__device__ __forceinline__ float na_dist(int metric, const float* qv, const float* xr, uint32_t d) {
    float acc = 0.f;
    if (metric == L2) {
        for (uint32_t t = 0; t < d; t++) acc = dist_step<L2>(acc, qv[t], xr[t]);
    } else if (metric == L1) {
        for (uint32_t t = 0; t < d; t++) acc = dist_step<L1>(acc, qv[t], xr[t]);
    } else {
        for (uint32_t t = 0; t < d; t++) acc = dist_step<CHI2>(acc, qv[t], xr[t]);
    }
    return acc;
}

__global__ void k_search_noalloc(NaArgs a) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t slot = blockIdx.x * NA_WARPS + w;
    NaHeader* hdr = reinterpret_cast<NaHeader*>(a.scratch);
    NaSlot* sl = reinterpret_cast<NaSlot*>(a.scratch + NA_HEADER) + slot;
    const size_t wbytes = (((size_t)a.d * 4 + 15) & ~(size_t)15) + (size_t)(a.topk + 1) * 8 + 32 * 8;
    unsigned char* base = smem + (size_t)w * ((wbytes + 15) & ~(size_t)15);
    float* qv = reinterpret_cast<float*>(base);
    NaHP* top = reinterpret_cast<NaHP*>(base + (((size_t)a.d * 4 + 15) & ~(size_t)15));
    float* stage_d = reinterpret_cast<float*>(top + a.topk + 1);
    uint32_t* stage_i = reinterpret_cast<uint32_t*>(stage_d + 32);
    unsigned long long cmps = 0;
    const uint32_t nlast = a.nrows[a.L - 1];
    for (;;) {
        unsigned qi = 0;
        if (lane == 0) qi = atomicAdd(&hdr->next_q, 1u);
        qi = __shfl_sync(FULL, qi, 0);
        if (qi >= a.nq) break;
        for (uint32_t t = lane; t < a.d; t += 32) qv[t] = a.q[(size_t)qi * a.d + t];
        __syncwarp();
        uint32_t cur = a.entry;
        float cur_d = na_dist(a.metric, qv, a.x + (size_t)cur * a.dp, a.d);
        cmps++;
        bool ok = true;
        for (uint32_t g = 0; g + 1 < a.L && ok; g++) {
            const uint64_t* off = a.off[g];
            const uint32_t* adj = a.adj[g];
            bool moved = true;
            uint32_t moves = 0;
            while (moved) {
                moved = false;
                if (cur >= a.nrows[g] || ++moves > a.nrows[g]) {
                    if (lane == 0) atomicOr(&hdr->err, cur >= a.nrows[g] ? NA_ERR_ID : NA_ERR_LOOP);
                    ok = false;
                    break;
                }
                const uint64_t b = off[cur], e = off[cur + 1];
                for (uint64_t c0 = b; c0 < e; c0 += 32) {
                    uint32_t nn = 0;
                    float dd = 0.f;
                    if (c0 + lane < e) {
                        nn = adj[c0 + lane];
                        if (nn < a.nrows[g]) dd = na_dist(a.metric, qv, a.x + (size_t)nn * a.dp, a.d);
                        else {
                            atomicOr(&hdr->err, NA_ERR_ID);
                            dd = __int_as_float(0x7f800000);  // never taken
                        }
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
        const uint64_t* off = a.off[a.L - 1];
        const uint32_t* adj = a.adj[a.L - 1];
        ok = ok && cur < nlast;
        uint32_t ntop = 0, ncand = 0, nvis = ok ? 1u : 0u;
        bool vis_overflow = false;
        if (lane == 0 && ok) {
            na_push(sl->cand, ncand, NaHP{-cur_d, cur});
            na_push(top, ntop, NaHP{cur_d, cur});
            atomicOr(&sl->visited[cur >> 5], 1u << (cur & 31));
            sl->vlist[0] = cur;
        }
        ncand = __shfl_sync(FULL, ncand, 0);
        ntop = __shfl_sync(FULL, ntop, 0);
        __syncwarp();
        float lwbnd = 0.f;
        if (lane == 0 && ok) lwbnd = top[0].f;
        lwbnd = __shfl_sync(FULL, lwbnd, 0);
        uint32_t expansions = 0;
        while (ncand > 0) {
            NaHP c{0.f, 0u};
            if (lane == 0) c = sl->cand[0];
            c.f = __shfl_sync(FULL, c.f, 0);
            c.id = __shfl_sync(FULL, c.id, 0);
            if (-c.f > lwbnd) break;
            if (c.id >= nlast || ++expansions > nlast + 1) {
                if (lane == 0) atomicOr(&hdr->err, c.id >= nlast ? NA_ERR_ID : NA_ERR_LOOP);
                break;
            }
            if (lane == 0) na_pop(sl->cand, ncand);
            ncand = __shfl_sync(FULL, ncand, 0);
            const uint64_t b = off[c.id], e = off[c.id + 1];
            for (uint64_t c0 = b; c0 < e; c0 += 32) {
                uint32_t nn = 0;
                bool fresh = false;
                if (c0 + lane < e) {
                    nn = adj[c0 + lane];
                    if (nn < nlast) {
                        const uint32_t old = atomicOr(&sl->visited[nn >> 5], 1u << (nn & 31));
                        fresh = !(old & (1u << (nn & 31)));
                    } else {
                        atomicOr(&hdr->err, NA_ERR_ID);
                    }
                }
                const unsigned fb = __ballot_sync(FULL, fresh);
                if (fresh) {
                    const uint32_t r = __popc(fb & ((1u << lane) - 1u));
                    if (nvis + r < NA_VCAP) sl->vlist[nvis + r] = nn;
                    stage_d[r] = na_dist(a.metric, qv, a.x + (size_t)nn * a.dp, a.d);
                    stage_i[r] = nn;
                }
                const uint32_t nf = __popc(fb);
                nvis += nf;
                if (nvis > NA_VCAP) vis_overflow = true;
                cmps += nf;
                __syncwarp();
                if (lane == 0) {
                    for (uint32_t r = 0; r < nf; r++) {
                        const float dj = stage_d[r];
                        if (top[0].f > dj || ntop < a.topk) {
                            if (ncand >= NA_CCAP) {
                                atomicOr(&hdr->err, NA_ERR_HEAP);
                                continue;
                            }
                            na_push(sl->cand, ncand, NaHP{-dj, stage_i[r]});
                            na_push(top, ntop, NaHP{dj, stage_i[r]});
                            if (ntop > a.topk) na_pop(top, ntop);
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
        if (lane == 0) {
            for (uint32_t t = ntop; t < a.topk; t++) {
                a.out_ids[(size_t)qi * a.topk + t] = 0xffffffffu;
                if (a.out_d) a.out_d[(size_t)qi * a.topk + t] = 0.f;
            }
            for (int loc = (int)ntop - 1; loc >= 0; loc--) {
                a.out_ids[(size_t)qi * a.topk + loc] = top[0].id;
                if (a.out_d) a.out_d[(size_t)qi * a.topk + loc] = top[0].f;
                na_pop(top, ntop);
            }
        }
        // leave this slot's visited bits clear for the next query
        if (!vis_overflow) {
            for (uint32_t t = lane; t < nvis; t += 32) {
                const uint32_t id = sl->vlist[t];
                atomicAnd(&sl->visited[id >> 5], ~(1u << (id & 31)));
            }
        } else {
            for (uint32_t t = lane; t < (nlast + 31) / 32; t += 32) sl->visited[t] = 0;
        }
        __syncwarp();
    }
    for (int o = 16; o > 0; o >>= 1) cmps += __shfl_xor_sync(FULL, cmps, o);
    if (lane == 0) atomicAdd(&hdr->ncmps, cmps / 32);
}

// Device address of g_noalloc_scratch, fetched once per device.
std::mutex g_addr_mu;
unsigned char* g_addr[64] = {};
// Whether a device's visited bitmaps are known to be all zero.  Every query clears
// the bits it set before its warp takes the next one (error paths included),
// so a call whose kernel ran to completion leaves them all zero; they are
// cleared on the first call on a device and after a call that did not reach
// its final synchronize.
bool g_bits_clean[64] = {};

cudaError_t scratch_address(int dev, unsigned char** out) {
    std::lock_guard<std::mutex> lk(g_addr_mu);
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    if (!g_addr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        g_addr[dev] = static_cast<unsigned char*>(p);
    }
    *out = g_addr[dev];
    return cudaSuccess;
}

// rand() % m for the first rand() after srand(seed) (lysearch.cpp:382),
// without heap allocation: r[0..30] from srand, r[31..33] = r[0..2],
// r[i] = r[i-31] + r[i-3], first output r[344] >> 1.
uint32_t first_rand(uint32_t seed) {
    if (seed == 0) seed = 1;
    uint32_t r[345];
    int32_t word = (int32_t)seed;
    r[0] = (uint32_t)word;
    for (int i = 1; i < 31; i++) {
        long hi = word / 127773, lo = word % 127773;
        word = (int32_t)(16807 * lo - 2836 * hi);
        if (word < 0) word += 2147483647;
        r[i] = (uint32_t)word;
    }
    for (int i = 31; i < 34; i++) r[i] = r[i - 31];
    for (int i = 34; i < 345; i++) r[i] = r[i - 3] + r[i - 31];
    return r[344] >> 1;
}

}  // namespace
}  // namespace nnm

extern "C" int nnm_search_noalloc(const float* x_dev, uint64_t n, uint32_t d, const nnm_dev_layers* layers,
                                  const float* q_dev, uint64_t nq, uint32_t topk, uint32_t seed, uint32_t metric,
                                  uint32_t* out_ids_dev, float* out_dists_dev, uint64_t* ncmps, void* stream) {
    using namespace nnm;
    if (!x_dev || !q_dev || !layers || !out_ids_dev) return NNM_ERR_INVALID;
    if (layers->nlayers < 1 || layers->nlayers > 16) return NNM_ERR_INVALID;
    if (metric > NNM_METRIC_CHI2) return NNM_ERR_UNSUPPORTED_METRIC;
    if (topk == 0 || topk > NA_MAX_TOPK || d == 0 || d > NA_MAX_DIM || nq >= (1ull << 32))
        return NNM_ERR_INVALID;
    const uint32_t L = layers->nlayers;
    for (uint32_t g = 0; g < L; g++) {
        const uint32_t nr = layers->nrows[g];
        if (nr == 0 || nr > n || (g + 1 < L && nr > layers->nrows[g + 1]) || !layers->off[g] || !layers->adj[g])
            return NNM_ERR_INVALID;
    }
    if (layers->nrows[L - 1] > NA_MAX_ROWS) return NNM_ERR_INVALID;  // visited-bitmap capacity
    if (nq == 0) {
        if (ncmps) *ncmps = 0;
        return NNM_OK;
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return NNM_ERR_NO_DEVICE;
    unsigned char* scratch = nullptr;
    if (scratch_address(dev, &scratch) != cudaSuccess) return NNM_ERR_CUDA;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // clear what must start at zero: the counters on every call, the visited
    // bitmaps (64 slots x 128 KiB) only when an earlier call may have left bits
    if (cudaMemsetAsync(scratch, 0, NA_HEADER, st) != cudaSuccess) return NNM_ERR_CUDA;
    if (!g_bits_clean[dev]) {
        if (cudaMemset2DAsync(scratch + NA_HEADER, sizeof(NaSlot), 0, sizeof(uint32_t) * NA_WORDS, NA_SLOTS, st) !=
            cudaSuccess)
            return NNM_ERR_CUDA;
    }
    g_bits_clean[dev] = false;
    NaArgs a{};
    a.x = x_dev;
    a.dp = d;
    a.d = d;
    a.metric = (int)metric;
    a.L = L;
    for (uint32_t g = 0; g < L; g++) {
        a.off[g] = layers->off[g];
        a.adj[g] = layers->adj[g];
        a.nrows[g] = layers->nrows[g];
    }
    a.q = q_dev;
    a.nq = (uint32_t)nq;
    a.topk = topk;
    a.entry = first_rand(seed) % layers->nrows[0];
    a.out_ids = out_ids_dev;
    a.out_d = out_dists_dev;
    a.scratch = scratch;
    const size_t wbytes = (((size_t)d * 4 + 15) & ~(size_t)15) + (size_t)(topk + 1) * 8 + 32 * 8;
    const size_t smem = (size_t)NA_WARPS * ((wbytes + 15) & ~(size_t)15);
    if (smem > 200 * 1024) return NNM_ERR_INVALID;
    if (cudaFuncSetAttribute(k_search_noalloc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return NNM_ERR_CUDA;
    k_search_noalloc<<<NA_SLOTS / NA_WARPS, NA_WARPS * 32, smem, st>>>(a); count_launch();
    if (cudaGetLastError() != cudaSuccess) return NNM_ERR_CUDA;
    NaHeader h;
    if (cudaMemcpyAsync(&h, scratch, sizeof(h), cudaMemcpyDeviceToHost, st) != cudaSuccess) return NNM_ERR_CUDA;
    if (cudaStreamSynchronize(st) != cudaSuccess) return NNM_ERR_CUDA;
    g_bits_clean[dev] = true;  // the kernel finished: every query cleared its bits
    if (ncmps) *ncmps = h.ncmps;
    if (h.err) return NNM_ERR_CAPACITY;
    return NNM_OK;
}
