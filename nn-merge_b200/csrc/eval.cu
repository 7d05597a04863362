// Recall of a k-NN graph on the device (the reference's Evaluator,
// evaluator.cpp:258-295, with the ground truth computed here instead of read
// from a file).
//
// For each evaluated row r: t_r = the atop-th smallest distance from r to
// every other row (exact brute force, the reference's sequential FP32 sum);
// a hit is one of the graph's first atop ids of r whose distance is <= t_r.
// recall = hits / (rows x atop).  Where no two rows tie at the atop-th
// distance this is the size of the intersection of the graph's first atop
// ids with the exact atop nearest ids (getKGraphRecall); tied rows count as
// hits either way.
//
// k_kth: 8 warps per block, one evaluated row per warp; the block streams
// the data set through shared memory in tiles of 64 rows (each tile read
// once per 8 evaluated rows); lane l measures tile rows l and l + 32 and
// keeps its 16 smallest distances sorted in registers; the warp then merges
// the 32 lists to the atop-th value.
#include <algorithm>
#include <cmath>
#include <vector>

#include "nnm_common.cuh"
#include "nnm_eval.h"
#include "nnm_launch.h"

namespace nnm {
namespace {
constexpr unsigned FULL = 0xffffffffu;
constexpr uint32_t EW = 8;   // evaluated rows (warps) per block
constexpr uint32_t ET = 64;  // data rows per shared-memory tile
constexpr int EA = EVAL_MAX_ATOP;

__global__ void __launch_bounds__(EW * 32) k_kth(const float* __restrict__ x, uint32_t n, uint32_t dp, int metric,
                                                 const uint32_t* __restrict__ rows, uint32_t nrows, uint32_t atop,
                                                 float* __restrict__ kth) {
    extern __shared__ __align__(16) float sm[];
    const uint32_t st = dp + 4;  // row stride: a quarter-warp's float4 reads fall in distinct banks
    float* tile = sm;
    float* qs = sm + ET * st;
    const uint32_t w = threadIdx.x >> 5, lane = threadIdx.x & 31, r0 = blockIdx.x * EW;
    const bool active = r0 + w < nrows;
    const uint32_t self = active ? rows[r0 + w] : 0xffffffffu;
    for (uint32_t i = threadIdx.x; i < EW * dp; i += blockDim.x) {
        const uint32_t e = i / dp, c = i - e * dp;
        qs[e * st + c] = r0 + e < nrows ? x[(size_t)rows[r0 + e] * dp + c] : 0.f;
    }
    float best[EA];
#pragma unroll
    for (int q = 0; q < EA; q++) best[q] = INFINITY;
    for (uint32_t t0 = 0; t0 < n; t0 += ET) {
        __syncthreads();
        const uint32_t nt = min(ET, n - t0);
        for (uint32_t i = threadIdx.x; i < nt * (dp / 4); i += blockDim.x) {
            const uint32_t rr = i / (dp / 4), c4 = i - rr * (dp / 4);
            *reinterpret_cast<float4*>(tile + rr * st + 4 * c4) =
                *reinterpret_cast<const float4*>(x + (size_t)(t0 + rr) * dp + 4 * c4);
        }
        __syncthreads();
        if (!active) continue;
#pragma unroll
        for (uint32_t h = 0; h < 2; h++) {
            const uint32_t j = lane + 32 * h;
            if (j < nt && t0 + j != self) {
                const float d = dist_seq_rt(metric, qs + w * st, tile + j * st, (int)dp);
                if (d < best[EA - 1]) {
                    best[EA - 1] = d;
#pragma unroll
                    for (int q = EA - 1; q > 0; q--)
                        if (best[q] < best[q - 1]) {
                            const float tv = best[q];
                            best[q] = best[q - 1];
                            best[q - 1] = tv;
                        }
                }
            }
        }
    }
    if (!active) return;
    // the atop-th smallest of the 32 sorted lists: atop rounds of taking the
    // smallest list head
    float v = INFINITY;
    for (uint32_t t = 0; t < atop; t++) {
        float m = best[0];
        uint32_t ml = lane;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const float om = __shfl_xor_sync(FULL, m, o);
            const uint32_t ol = __shfl_xor_sync(FULL, ml, o);
            if (om < m || (om == m && ol < ml)) {
                m = om;
                ml = ol;
            }
        }
        v = m;
        if (lane == ml) {
#pragma unroll
            for (int q = 0; q < EA - 1; q++) best[q] = best[q + 1];
            best[EA - 1] = INFINITY;
        }
    }
    if (lane == 0) kth[r0 + w] = v;
}

// Warp per evaluated row: hits among the graph's first atop ids.
__global__ void k_hits(const float* __restrict__ x, uint32_t dp, int metric, const uint32_t* __restrict__ ids,
                       uint32_t k, const uint32_t* __restrict__ rows, uint32_t nrows, uint32_t atop, uint32_t n,
                       const float* __restrict__ kth, unsigned long long* __restrict__ hits) {
    const uint32_t w = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (w >= nrows) return;
    const uint32_t row = rows[w];
    bool hit = false;
    if (lane < atop) {
        const uint32_t id = ids[(size_t)row * k + lane] & ID_MASK;
        if (id < n && id != row)
            hit = dist_seq_rt(metric, x + (size_t)row * dp, x + (size_t)id * dp, (int)dp) <= kth[w];
    }
    const uint32_t c = __popc(__ballot_sync(FULL, hit));
    if (lane == 0 && c) atomicAdd(hits, (unsigned long long)c);
}
}  // namespace

int graph_recall_dev(Ctx& ctx, const float* x, uint32_t n, uint32_t dp, int metric, const uint32_t* ids, uint32_t k,
                     const uint32_t* rows, uint32_t nrows, uint32_t atop, double* recall) {
    if (!nrows) {
        *recall = 0.0;
        return 0;
    }
    DevBuf kb, hb;
    auto done = [&](int rc) {
        kb.release();
        hb.release();
        return rc;
    };
    const size_t smem = ((size_t)ET + EW) * (dp + 4) * 4;
    if (cudaFuncSetAttribute(k_kth, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess ||
        kb.ensure((size_t)nrows * 4) != cudaSuccess || hb.ensure(8) != cudaSuccess) {
        ctx.last_error = "recall: device setup failed";
        return done(4);
    }
    cudaStream_t st = ctx.stream;
    cudaMemsetAsync(hb.p, 0, 8, st);
    k_kth<<<(nrows + EW - 1) / EW, EW * 32, smem, st>>>(x, n, dp, metric, rows, nrows, atop, kb.as<float>());
    k_hits<<<(nrows + 7) / 8, 256, 0, st>>>(x, dp, metric, ids, k, rows, nrows, atop, n, kb.as<float>(),
                                            hb.as<unsigned long long>());
    count_launch(2);
    unsigned long long h = 0;
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h, hb.p, 8, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        ctx.last_error = std::string("recall: ") + cudaGetErrorString(e);
        return done(3);
    }
    *recall = (double)h / ((double)nrows * (double)atop);
    return done(0);
}

}  // namespace nnm
