// Entry-point network of the serving path (NNM_ENTRY_LEARNED): inference,
// brute-force training labels, and training with hand-written kernels.
//
//   u = x * scale + shift            (d inputs, d <= 256)
//   h = relu(W1 u + b1)              (256)
//   s = W2 h + b2                    (C scores; class c = row c of the entry layer)
//   loss = mean_b [ log sum_c exp(s_bc) - s_b,label_b ]
//
// The label of a training row is its nearest class row (squared L2).  A
// query's probes are the classes of its P largest scores; the search then
// measures those rows and starts its greedy descent at the nearest one, on
// the entry layer, instead of descending from the top of the hierarchy.
//
// Weights are BF16 on the device (rounded from FP32 master copies that Adam
// updates); every product is accumulated in FP32; gradients are taken with
// respect to the BF16 weights.  One training step (sampling, forward, loss,
// backward, Adam, BF16 refresh, step counter) is captured as a CUDA graph and
// replayed, as the code network's training is.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "nnm_common.cuh"
#include "nnm_entry.h"
#include "nnm_launch.h"
#include "nnm_learned.h"
#include "nnm_tc.cuh"

namespace nnm {
namespace {
using bf16 = __nv_bfloat16;
constexpr uint32_t EH = ENTRY_H;
constexpr uint32_t ERB = 32;          // rows per block
constexpr uint64_t STEP_KERNELS = 11; // kernels of one captured training step

struct EView {
    const bf16* w1t;  // d x 256
    const float* b1;
    const bf16* w2t;  // 256 x C
    const bf16* w2r;  // C x 256
    const float* b2;
    uint32_t d, C;
    float scale, shift;
};

__device__ __forceinline__ float bf(bf16 v) { return __bfloat162float(v); }

size_t hidden_smem(uint32_t d) { return (size_t)ERB * ((d + 3) & ~3u) * 4; }

__device__ __forceinline__ void put(float* p, float v) { *p = v; }
__device__ __forceinline__ void put(bf16* p, float v) { *p = __float2bfloat16_rn(v); }

// h = relu(W1 u + b1) of ERB rows per block; row r is x row idx[r] (or r).
// Training keeps h in FP32; inference rounds it to BF16, the tensor-core
// operand of the score kernel.
template <typename OutT>
__global__ void __launch_bounds__(256) k_ent_hidden(EView v, const float* __restrict__ x, uint32_t dp,
                                                    const uint32_t* __restrict__ idx, uint32_t nrows,
                                                    OutT* __restrict__ h) {
    extern __shared__ __align__(16) float us[];
    const uint32_t d = v.d, dpad = (d + 3) & ~3u, tid = threadIdx.x, r0 = blockIdx.x * ERB;
    for (uint32_t i = tid; i < ERB * dpad; i += 256) {
        const uint32_t r = i / dpad, k = i - r * dpad, gr = r0 + r;
        float val = 0.f;
        if (gr < nrows && k < d) {
            const size_t row = idx ? idx[gr] : gr;
            val = fmaf(x[row * dp + k], v.scale, v.shift);
        }
        us[i] = val;
    }
    __syncthreads();
    const uint32_t j = tid;
    float acc[ERB];
    const float bj = v.b1[j];
#pragma unroll
    for (uint32_t r = 0; r < ERB; r++) acc[r] = bj;
    for (uint32_t k = 0; k < dpad; k += 4) {
        float w[4];
#pragma unroll
        for (int q = 0; q < 4; q++) w[q] = k + q < d ? bf(v.w1t[(size_t)(k + q) * EH + j]) : 0.f;
#pragma unroll
        for (uint32_t r = 0; r < ERB; r++) {
            const float4 u = *reinterpret_cast<const float4*>(us + r * dpad + k);
            acc[r] = fmaf(u.x, w[0], acc[r]);
            acc[r] = fmaf(u.y, w[1], acc[r]);
            acc[r] = fmaf(u.z, w[2], acc[r]);
            acc[r] = fmaf(u.w, w[3], acc[r]);
        }
    }
#pragma unroll
    for (uint32_t r = 0; r < ERB; r++)
        if (r0 + r < nrows) put(h + (size_t)(r0 + r) * EH + j, fmaxf(acc[r], 0.f));
}

// s = W2 h + b2: block (row tile, 256-class tile), thread = class.
__global__ void __launch_bounds__(256) k_ent_scores(EView v, const float* __restrict__ h, uint32_t nrows,
                                                    float* __restrict__ s) {
    __shared__ __align__(16) float hs[ERB * EH];
    const uint32_t tid = threadIdx.x, r0 = blockIdx.x * ERB, c = blockIdx.y * 256 + tid;
    for (uint32_t i = tid; i < ERB * EH; i += 256) {
        const uint32_t r = i / EH;
        hs[i] = r0 + r < nrows ? h[(size_t)(r0 + r) * EH + (i - r * EH)] : 0.f;
    }
    __syncthreads();
    if (c >= v.C) return;
    float acc[ERB];
    const float b = v.b2[c];
#pragma unroll
    for (uint32_t r = 0; r < ERB; r++) acc[r] = b;
    for (uint32_t j = 0; j < EH; j += 4) {
        float w[4];
#pragma unroll
        for (int q = 0; q < 4; q++) w[q] = bf(v.w2t[(size_t)(j + q) * v.C + c]);
#pragma unroll
        for (uint32_t r = 0; r < ERB; r++) {
            const float4 hv = *reinterpret_cast<const float4*>(hs + r * EH + j);
            acc[r] = fmaf(hv.x, w[0], acc[r]);
            acc[r] = fmaf(hv.y, w[1], acc[r]);
            acc[r] = fmaf(hv.z, w[2], acc[r]);
            acc[r] = fmaf(hv.w, w[3], acc[r]);
        }
    }
#pragma unroll
    for (uint32_t r = 0; r < ERB; r++)
        if (r0 + r < nrows) s[(size_t)(r0 + r) * v.C + c] = acc[r];
}

// Warp per row: the loss term, and dL/ds = (softmax(s) - onehot) / B written
// over s.  Per-block loss partial sums in a fixed order (deterministic).
__global__ void k_ent_ce(float* __restrict__ s, const uint32_t* __restrict__ lab, uint32_t B, uint32_t C,
                         float* __restrict__ partial) {
    __shared__ float wl[8];
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t b = blockIdx.x * 8 + warp;
    float l = 0.f;
    if (b < B) {
        float* row = s + (size_t)b * C;
        float mx = -INFINITY;
        for (uint32_t c = lane; c < C; c += 32) mx = fmaxf(mx, row[c]);
        for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        float se = 0.f;
        for (uint32_t c = lane; c < C; c += 32) se += expf(row[c] - mx);
        for (int o = 16; o > 0; o >>= 1) se += __shfl_xor_sync(0xffffffffu, se, o);
        const uint32_t y = lab[b];
        l = logf(se) + mx - row[y];
        __syncwarp();
        const float inv = 1.f / (se * (float)B), oneb = 1.f / (float)B;
        for (uint32_t c = lane; c < C; c += 32) row[c] = expf(row[c] - mx) * inv - (c == y ? oneb : 0.f);
    }
    if (lane == 0) wl[warp] = l;
    __syncthreads();
    if (threadIdx.x == 0) {
        float t = 0.f;
        for (int w = 0; w < 8; w++) t += wl[w];
        partial[blockIdx.x] = t;
    }
}

__global__ void k_ent_loss_final(const float* partial, uint32_t nblk, uint32_t B, float* loss, const uint32_t* step) {
    float t = 0.f;
    for (uint32_t i = 0; i < nblk; i++) t += partial[i];
    loss[step ? *step : 0] = t / (float)B;
}

// dL/d(pre-activation of h) = (h > 0) * sum_c g[r][c] W2[c][j]: block of
// ERB rows, thread j, classes in tiles of 32 staged in shared memory.
__global__ void __launch_bounds__(256) k_ent_dh(const float* __restrict__ g, const float* __restrict__ h, EView v,
                                                uint32_t B, float* __restrict__ dh) {
    __shared__ __align__(16) float gs[ERB * 32];
    const uint32_t j = threadIdx.x, r0 = blockIdx.x * ERB, C = v.C;
    float acc[ERB];
#pragma unroll
    for (uint32_t r = 0; r < ERB; r++) acc[r] = 0.f;
    for (uint32_t c0 = 0; c0 < C; c0 += 32) {
        __syncthreads();
        for (uint32_t i = j; i < ERB * 32; i += 256) {
            const uint32_t r = i >> 5, cc = i & 31;
            gs[i] = (r0 + r < B && c0 + cc < C) ? g[(size_t)(r0 + r) * C + c0 + cc] : 0.f;
        }
        __syncthreads();
        for (uint32_t cc = 0; cc < 32; cc += 4) {
            float w[4];
#pragma unroll
            for (int q = 0; q < 4; q++) w[q] = c0 + cc + q < C ? bf(v.w2r[(size_t)(c0 + cc + q) * EH + j]) : 0.f;
#pragma unroll
            for (uint32_t r = 0; r < ERB; r++) {
                const float4 gv = *reinterpret_cast<const float4*>(gs + r * 32 + cc);
                acc[r] = fmaf(gv.x, w[0], acc[r]);
                acc[r] = fmaf(gv.y, w[1], acc[r]);
                acc[r] = fmaf(gv.z, w[2], acc[r]);
                acc[r] = fmaf(gv.w, w[3], acc[r]);
            }
        }
    }
#pragma unroll
    for (uint32_t r = 0; r < ERB; r++)
        if (r0 + r < B) {
            const size_t o = (size_t)(r0 + r) * EH + j;
            dh[o] = h[o] > 0.f ? acc[r] : 0.f;
        }
}

// dW2[c][j] = sum_r g[r][c] h[r][j] and db2[c]: block of 16 classes, thread j.
constexpr uint32_t GC = 16;
__global__ void __launch_bounds__(256) k_ent_gw2(const float* __restrict__ g, const float* __restrict__ h, uint32_t B,
                                                 uint32_t C, float* __restrict__ gw2, float* __restrict__ gb2) {
    __shared__ __align__(16) float gs[32 * GC];
    const uint32_t j = threadIdx.x, c0 = blockIdx.x * GC;
    float acc[GC];
#pragma unroll
    for (uint32_t q = 0; q < GC; q++) acc[q] = 0.f;
    float sb = 0.f;
    for (uint32_t r0 = 0; r0 < B; r0 += 32) {
        __syncthreads();
        for (uint32_t i = j; i < 32 * GC; i += 256) {
            const uint32_t r = i / GC, cc = i % GC;
            gs[i] = (r0 + r < B && c0 + cc < C) ? g[(size_t)(r0 + r) * C + c0 + cc] : 0.f;
        }
        __syncthreads();
        const uint32_t rn = min(32u, B - r0);
        for (uint32_t r = 0; r < rn; r++) {
            const float hv = h[(size_t)(r0 + r) * EH + j];
#pragma unroll
            for (uint32_t q = 0; q < GC; q += 4) {
                const float4 gv = *reinterpret_cast<const float4*>(gs + r * GC + q);
                acc[q] = fmaf(gv.x, hv, acc[q]);
                acc[q + 1] = fmaf(gv.y, hv, acc[q + 1]);
                acc[q + 2] = fmaf(gv.z, hv, acc[q + 2]);
                acc[q + 3] = fmaf(gv.w, hv, acc[q + 3]);
            }
        }
        if (j < GC)
            for (uint32_t r = 0; r < rn; r++) sb += gs[r * GC + j];
    }
#pragma unroll
    for (uint32_t q = 0; q < GC; q++)
        if (c0 + q < C) gw2[(size_t)(c0 + q) * EH + j] = acc[q];
    if (j < GC && c0 + j < C) gb2[c0 + j] = sb;
}

// BF16 copies of the master weights: W1 transposed, W2 both ways.
__global__ void k_ent_refresh(const float* __restrict__ w1, const float* __restrict__ w2, uint32_t d, uint32_t C,
                              bf16* __restrict__ w1t, bf16* __restrict__ w2t, bf16* __restrict__ w2r) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < EH * d) {
        const uint32_t j = i / d, k = i - j * d;
        w1t[(size_t)k * EH + j] = __float2bfloat16_rn(w1[i]);
    }
    if (i < C * EH) {
        const uint32_t c = i / EH, j = i - c * EH;
        const bf16 b = __float2bfloat16_rn(w2[i]);
        w2r[i] = b;
        w2t[(size_t)j * C + c] = b;
    }
}

// Nearest class row (rows 0..C-1 of x) of every pool row, squared L2 in
// FP32, ties to the lower class.  Block: 32 pool rows x class tiles of 64;
// thread (row t/8, classes t%8 + 8q).
constexpr uint32_t LR = 32, LC = 64;
__global__ void __launch_bounds__(256) k_ent_labels(const float* __restrict__ x, uint32_t dp, uint32_t d,
                                                    const uint32_t* __restrict__ rows, uint32_t npool, uint32_t C,
                                                    uint32_t* __restrict__ lab) {
    extern __shared__ float sm[];
    const uint32_t st = d + 1;  // odd stride: rows of one warp fall in different banks
    float* ps = sm;
    float* cs = sm + LR * st;
    const uint32_t tid = threadIdx.x, r0 = blockIdx.x * LR, r = tid >> 3, sub = tid & 7;
    for (uint32_t i = tid; i < LR * d; i += 256) {
        const uint32_t rr = i / d, k = i - rr * d;
        ps[rr * st + k] = r0 + rr < npool ? x[(size_t)rows[r0 + rr] * dp + k] : 0.f;
    }
    float bd = INFINITY;
    uint32_t bc = 0xffffffffu;
    for (uint32_t c0 = 0; c0 < C; c0 += LC) {
        __syncthreads();
        for (uint32_t i = tid; i < LC * d; i += 256) {
            const uint32_t cc = i / d, k = i - cc * d;
            cs[cc * st + k] = c0 + cc < C ? x[(size_t)(c0 + cc) * dp + k] : 0.f;
        }
        __syncthreads();
        float acc[LC / 8];
#pragma unroll
        for (uint32_t q = 0; q < LC / 8; q++) acc[q] = 0.f;
        for (uint32_t k = 0; k < d; k++) {
            const float pv = ps[r * st + k];
#pragma unroll
            for (uint32_t q = 0; q < LC / 8; q++) {
                const float t = pv - cs[(sub + 8 * q) * st + k];
                acc[q] = fmaf(t, t, acc[q]);
            }
        }
#pragma unroll
        for (uint32_t q = 0; q < LC / 8; q++) {
            const uint32_t c = c0 + sub + 8 * q;
            if (c < C && (acc[q] < bd || (acc[q] == bd && c < bc))) {
                bd = acc[q];
                bc = c;
            }
        }
    }
#pragma unroll
    for (int o = 1; o < 8; o <<= 1) {
        const float od = __shfl_xor_sync(0xffffffffu, bd, o);
        const uint32_t oc = __shfl_xor_sync(0xffffffffu, bc, o);
        if (od < bd || (od == bd && oc < bc)) {
            bd = od;
            bc = oc;
        }
    }
    if (sub == 0 && r0 + r < npool) lab[r0 + r] = bc < C ? bc : 0u;
}

__global__ void k_ent_pool(uint32_t* rows, uint32_t npool, uint32_t n, uint32_t seed) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= npool) return;
    if (npool == n) {
        rows[i] = i;
    } else {
        const Philox ph{seed, 0x6e6e6d30u};
        rows[i] = bounded(ph(i, 0, 0, 0).x, n);
    }
}

__global__ void k_ent_sample(uint32_t* idx, uint32_t* lab, uint32_t B, const uint32_t* prow, const uint32_t* plab,
                             uint32_t npool, uint32_t seed, const uint32_t* step) {
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= B) return;
    const Philox ph{seed, 0x6e6e6d31u};
    const uint32_t t = bounded(ph(b, *step, 0, 0).x, npool);
    idx[b] = prow[t];
    lab[b] = plab[t];
}

__global__ void k_ent_step_inc(uint32_t* step) { *step += 1; }

// ---- inference on the tensor cores ----
// Scores of 128 rows per CTA against the C classes in tiles of 128 classes:
// D (128 x 128, FP32 in TMEM) = A (BF16 h, 128 x 256, K-major, resident in
// shared memory) x B^T (BF16 W2 rows of the tile, 128 x 256, K-major), one
// tcgen05.mma chain of 16 instructions (K = 16 each) per tile, issued by one
// thread and committed to an mbarrier.  Two B buffers and two 128-column
// accumulators: the MMA of tile j+1 runs while the epilogue reads tile j and
// tile j+2 loads.  The epilogue (thread = row = TMEM lane) reads 32 scores
// at a time with tcgen05.ld, adds the biases (all C of them staged in shared
// memory, padded with -inf), and either writes the scores (MODE 0) or keeps
// the row's ENTRY_MAX_PROBES largest in registers (MODE 1, ties to the lower
// class; a chunk whose maximum cannot enter the list is skipped) -- the
// probes, with no score written to HBM.  Operand layout: no swizzle, 8-row
// groups of 32 K-chunks of 16 bytes (4096 bytes per group).
constexpr uint32_t PT = 128;                  // rows (M) and classes (N) per tile
constexpr uint32_t PROW = EH * 2;             // 512 bytes of K per row
constexpr uint32_t PGRP = (PROW / 16) * 128;  // 4096 bytes per 8-row group
constexpr uint32_t PTILE = PT * PROW;         // 64 KB per operand tile
constexpr size_t PROBE_SMEM = 3 * (size_t)PTILE + (size_t)ENTRY_MAX_C * 4;
constexpr uint32_t IDESC_E = (1u << 4) | (1u << 7) | (1u << 10) | ((PT >> 3) << 17) | ((PT >> 4) << 24);
constexpr unsigned EERR_WAIT = 64u;           // an mbarrier wait ran out (search self-check code)

__device__ __forceinline__ void st_shared_zero16(uint32_t addr) {
    asm volatile("st.shared.v4.u32 [%0], {%1, %1, %1, %1};" ::"r"(addr), "r"(0u) : "memory");
}

// Rows [r0, r0 + 128) of a (rows x 256 BF16, row-major) into the operand
// layout at dst; rows past `rows` are zero.  Thread t copies chunk t % 32 of
// rows t / 32 + 4i: 32 consecutive threads read one 512-byte row.
__device__ __forceinline__ void load_tile(uint32_t dst, const bf16* __restrict__ src, uint32_t r0, uint32_t rows,
                                          uint32_t tid) {
    const uint32_t c = tid & 31, rt = tid >> 5;
    const char* s0 = reinterpret_cast<const char*>(src) + (size_t)r0 * PROW + c * 16;
#pragma unroll 8
    for (uint32_t i = 0; i < PT / 4; i++) {
        const uint32_t r = rt + 4 * i;
        const uint32_t addr = dst + (r >> 3) * PGRP + c * 128 + (r & 7) * 16;
        if (r0 + r < rows) cp_async16(addr, s0 + (size_t)r * PROW);
        else st_shared_zero16(addr);
    }
}

__device__ __forceinline__ void mma_tile(uint32_t tmem_acc, uint32_t a_s, uint32_t b_s, uint32_t bar) {
    asm volatile("tcgen05.fence::after_thread_sync;");
#pragma unroll 1
    for (uint32_t kk = 0; kk < PROW / 32; kk++) {  // 32 bytes of K per instruction
        const uint64_t da = smem_desc(a_s + kk * 256, 128, PGRP);
        const uint64_t db = smem_desc(b_s + kk * 256, 128, PGRP);
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_acc),
            "l"(da), "l"(db), "r"(IDESC_E), "r"(kk));
    }
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

template <int MODE>
__global__ void __launch_bounds__(128, 1) k_ent_tc(const bf16* __restrict__ h, uint32_t nrows,
                                                   const bf16* __restrict__ w2r, const float* __restrict__ b2,
                                                   uint32_t C, float* __restrict__ scores, uint32_t P,
                                                   uint32_t* __restrict__ probes, unsigned* __restrict__ err) {
    extern __shared__ __align__(1024) unsigned char smem[];
    __shared__ uint64_t mma_bar[2];
    __shared__ uint32_t tmem_base;
    const uint32_t tid = threadIdx.x, warp = tid >> 5;
    const uint32_t a_s = smem_u32(smem), r0 = blockIdx.x * PT;
    const uint32_t b_s0 = a_s + PTILE;  // B buffer x at b_s0 + x * PTILE
    float* sbias = reinterpret_cast<float*>(smem + 3 * (size_t)PTILE);
    const uint32_t nt = (C + PT - 1) / PT, row = r0 + tid;
    if (tid == 0) {
        for (int b = 0; b < 2; b++) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mma_bar[b])));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)),
                     "r"(2 * PT));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    for (uint32_t c = tid; c < nt * PT; c += 128) sbias[c] = c < C ? b2[c] : -INFINITY;
    load_tile(a_s, h, r0, nrows, tid);
    load_tile(b_s0, w2r, 0, C, tid);
    if (nt > 1) load_tile(b_s0 + PTILE, w2r, PT, C, tid);
    asm volatile("cp.async.wait_all;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // cp.async writes -> tensor core reads
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = tmem_base;
    const uint32_t bar0 = smem_u32(&mma_bar[0]);  // barrier x at bar0 + 8x
    if (tid == 0) mma_tile(tmem, a_s, b_s0, bar0);
    constexpr int Q = ENTRY_MAX_PROBES;
    float lv[Q];
    uint32_t li[Q];
#pragma unroll
    for (int q = 0; q < Q; q++) {
        lv[q] = -INFINITY;
        li[q] = 0xffffffffu;
    }
    uint32_t phase = 0u, pending = 1u;  // bit x: accumulator x's next phase / MMA in flight
    bool failed = false;
    for (uint32_t j = 0; j < nt; j++) {
        const uint32_t b = j & 1;
        // MMA j+1: its B buffer was loaded before the last barrier, and its
        // accumulator was last read by epilogue j-1, before that barrier
        if (j + 1 < nt) {
            if (tid == 0) mma_tile(tmem + (b ^ 1) * PT, a_s, b_s0 + (b ^ 1) * PTILE, bar0 + 8 * (b ^ 1));
            pending |= 1u << (b ^ 1);
        }
        const bool ok = mbar_wait_bounded(bar0 + 8 * b, (phase >> b) & 1u);
        if (__syncthreads_or(!ok)) {
            failed = true;
            break;
        }
        pending &= ~(1u << b);
        phase ^= 1u << b;
        asm volatile("tcgen05.fence::after_thread_sync;");
        if (j + 2 < nt) load_tile(b_s0 + b * PTILE, w2r, (j + 2) * PT, C, tid);  // MMA j, its last reader, is complete
        const uint32_t c0 = j * PT;
#pragma unroll 1
        for (uint32_t cc = 0; cc < PT; cc += 32) {
            uint32_t v[32];
            tmem_ld32(tmem + ((warp * 32u) << 16) + b * PT + cc, v);
            float sc[32];
#pragma unroll
            for (int i = 0; i < 32; i += 4) {
                const float4 bv = *reinterpret_cast<const float4*>(sbias + c0 + cc + i);
                sc[i] = __uint_as_float(v[i]) + bv.x;
                sc[i + 1] = __uint_as_float(v[i + 1]) + bv.y;
                sc[i + 2] = __uint_as_float(v[i + 2]) + bv.z;
                sc[i + 3] = __uint_as_float(v[i + 3]) + bv.w;
            }
            if (MODE == 0) {
                if (row < nrows)
#pragma unroll
                    for (int i = 0; i < 32; i++)
                        if (c0 + cc + i < C) scores[(size_t)row * C + c0 + cc + i] = sc[i];
            } else {
                float mx = sc[0];
#pragma unroll
                for (int i = 1; i < 32; i++) mx = fmaxf(mx, sc[i]);
                if (mx > lv[Q - 1]) {
#pragma unroll
                    for (int i = 0; i < 32; i++) {
                        if (sc[i] > lv[Q - 1]) {
                            lv[Q - 1] = sc[i];
                            li[Q - 1] = c0 + cc + i;
#pragma unroll
                            for (int q = Q - 1; q > 0; q--)
                                if (lv[q] > lv[q - 1]) {
                                    const float tv = lv[q];
                                    lv[q] = lv[q - 1];
                                    lv[q - 1] = tv;
                                    const uint32_t ti = li[q];
                                    li[q] = li[q - 1];
                                    li[q - 1] = ti;
                                }
                        }
                    }
                }
            }
        }
        asm volatile("cp.async.wait_all;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;");
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;");
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
    if (failed) {
        if (tid == 0) atomicOr(err, EERR_WAIT);
        for (uint32_t b = 0; b < 2; b++)
            if ((pending >> b) & 1u) mbar_wait_bounded(bar0 + 8 * b, (phase >> b) & 1u);  // an MMA may still write TMEM
    } else if (MODE == 1 && row < nrows) {
        for (uint32_t t = 0; t < P; t++) probes[(size_t)row * P + t] = li[t] < C ? li[t] : 0u;
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * PT));
    }
}

// Flat parameter layout: W1 (256 x d), b1, W2 (C x 256), b2.
struct ELayout {
    size_t w1, b1, w2, b2, total;
    ELayout(uint32_t d, uint32_t C)
        : w1(0), b1((size_t)EH * d), w2(b1 + EH), b2(w2 + (size_t)C * EH), total(b2 + C) {}
};

std::vector<float> eflatten(const nnm_entry_mlp& m, const ELayout& L) {
    std::vector<float> f(L.total);
    std::memcpy(f.data() + L.w1, m.w1, (size_t)EH * m.d_in * 4);
    std::memcpy(f.data() + L.b1, m.b1, EH * 4);
    std::memcpy(f.data() + L.w2, m.w2, (size_t)m.n_classes * EH * 4);
    std::memcpy(f.data() + L.b2, m.b2, (size_t)m.n_classes * 4);
    return f;
}

void eunflatten(const std::vector<float>& f, const ELayout& L, nnm_entry_mlp& m) {
    std::memcpy(m.w1, f.data() + L.w1, (size_t)EH * m.d_in * 4);
    std::memcpy(m.b1, f.data() + L.b1, EH * 4);
    std::memcpy(m.w2, f.data() + L.w2, (size_t)m.n_classes * EH * 4);
    std::memcpy(m.b2, f.data() + L.b2, (size_t)m.n_classes * 4);
}

EView view_of(const DevEntry& m) {
    return EView{m.w1t.as<bf16>(), m.b1.as<float>(), m.w2t.as<bf16>(), m.w2r.as<bf16>(), m.b2.as<float>(),
                 m.d, m.C, m.scale, m.shift};
}

cudaError_t set_attrs(uint32_t d) {
    const int hs = (int)hidden_smem(d);
    cudaError_t e = cudaFuncSetAttribute(k_ent_hidden<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, hs);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_ent_hidden<bf16>, cudaFuncAttributeMaxDynamicSharedMemorySize, hs);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_ent_tc<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)PROBE_SMEM);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_ent_tc<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)PROBE_SMEM);
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(k_ent_labels, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)((LR + LC) * (d + 1) * 4));
}

// Device model whose BF16 weights are refreshed from the flat FP32 vector f.
void refresh(const float* f, const ELayout& L, DevEntry& m, cudaStream_t st) {
    const uint32_t cnt = std::max<uint32_t>(EH * m.d, m.C * EH);
    k_ent_refresh<<<(cnt + 255) / 256, 256, 0, st>>>(f + L.w1, f + L.w2, m.d, m.C, m.w1t.as<bf16>(), m.w2t.as<bf16>(),
                                                     m.w2r.as<bf16>());
}

int alloc_model(Ctx& ctx, DevEntry& m, uint32_t d, uint32_t C, float scale, float shift) {
    NNM_CUDA_TRY(m.w1t.ensure((size_t)d * EH * 2));
    NNM_CUDA_TRY(m.w2t.ensure((size_t)EH * C * 2));
    NNM_CUDA_TRY(m.w2r.ensure((size_t)EH * C * 2));
    NNM_CUDA_TRY(m.b1.ensure(EH * 4));
    NNM_CUDA_TRY(m.b2.ensure((size_t)C * 4));
    m.d = d;
    m.C = C;
    m.scale = scale;
    m.shift = shift;
    return 0;
}

// Forward + loss + backward of B rows (p_idx, p_lab) with the device model
// m whose biases are the flat vector's; gradients into grad.
struct EPass {
    DevBuf idx, lab, h, s, dh, partial, flat, grad, mom, vel, loss, step;
    ~EPass() {
        for (DevBuf* b : {&idx, &lab, &h, &s, &dh, &partial, &flat, &grad, &mom, &vel, &loss, &step}) b->release();
    }
};

int alloc_pass(Ctx& ctx, EPass& p, uint32_t B, uint32_t C, const ELayout& L) {
    NNM_CUDA_TRY(p.idx.ensure((size_t)B * 4));
    NNM_CUDA_TRY(p.lab.ensure((size_t)B * 4));
    NNM_CUDA_TRY(p.h.ensure((size_t)B * EH * 4));
    NNM_CUDA_TRY(p.s.ensure((size_t)B * C * 4));
    NNM_CUDA_TRY(p.dh.ensure((size_t)B * EH * 4));
    NNM_CUDA_TRY(p.partial.ensure(((B + 7) / 8) * 4 + 64));
    NNM_CUDA_TRY(p.flat.ensure(L.total * 4));
    NNM_CUDA_TRY(p.grad.ensure(L.total * 4));
    NNM_CUDA_TRY(p.step.ensure(64));
    return 0;
}

EView pass_view(const EPass& p, const ELayout& L, const DevEntry& m) {
    EView v = view_of(m);
    v.b1 = p.flat.as<float>() + L.b1;
    v.b2 = p.flat.as<float>() + L.b2;
    return v;
}

void enqueue_pass(const EView& v, const float* x, uint32_t dp, uint32_t B, EPass& p, const ELayout& L,
                  const uint32_t* step, cudaStream_t st) {
    k_ent_hidden<float><<<(B + ERB - 1) / ERB, 256, hidden_smem(v.d), st>>>(v, x, dp, p.idx.as<uint32_t>(), B,
                                                                    p.h.as<float>());
    k_ent_scores<<<dim3((B + ERB - 1) / ERB, (v.C + 255) / 256), 256, 0, st>>>(v, p.h.as<float>(), B, p.s.as<float>());
    const uint32_t nblk = (B + 7) / 8;
    k_ent_ce<<<nblk, 256, 0, st>>>(p.s.as<float>(), p.lab.as<uint32_t>(), B, v.C, p.partial.as<float>());
    k_ent_loss_final<<<1, 1, 0, st>>>(p.partial.as<float>(), nblk, B, p.loss.as<float>(), step);
    k_ent_dh<<<(B + ERB - 1) / ERB, 256, 0, st>>>(p.s.as<float>(), p.h.as<float>(), v, B, p.dh.as<float>());
    float* g = p.grad.as<float>();
    k_ent_gw2<<<(v.C + GC - 1) / GC, 256, 0, st>>>(p.s.as<float>(), p.h.as<float>(), B, v.C, g + L.w2, g + L.b2);
    launch_grad_w1(p.dh.as<float>(), x, dp, p.idx.as<uint32_t>(), B, v.d, v.scale, v.shift, g + L.w1, g + L.b1, st);
}
constexpr uint64_t PASS_KERNELS = 7;

}  // namespace

void DevEntry::release() {
    w1t.release();
    b1.release();
    w2t.release();
    w2r.release();
    b2.release();
}

int entry_upload(Ctx& ctx, DevEntry& m, const nnm_entry_mlp& h) {
    const ELayout L(h.d_in, h.n_classes);
    int rc = alloc_model(ctx, m, h.d_in, h.n_classes, h.in_scale, h.in_shift);
    if (rc) return rc;
    std::vector<float> f = eflatten(h, L);
    DevBuf tmp;
    NNM_CUDA_TRY(tmp.ensure(L.total * 4));
    NNM_CUDA_TRY(cudaMemcpyAsync(tmp.p, f.data(), L.total * 4, cudaMemcpyHostToDevice, ctx.stream));
    const float* t = tmp.as<float>();
    refresh(t, L, m, ctx.stream);
    count_launch();
    NNM_CUDA_TRY(cudaMemcpyAsync(m.b1.p, t + L.b1, EH * 4, cudaMemcpyDeviceToDevice, ctx.stream));
    NNM_CUDA_TRY(cudaMemcpyAsync(m.b2.p, t + L.b2, (size_t)h.n_classes * 4, cudaMemcpyDeviceToDevice, ctx.stream));
    NNM_CUDA_TRY(cudaStreamSynchronize(ctx.stream));
    tmp.release();
    return 0;
}

int entry_infer(Ctx& ctx, const DevEntry& m, const float* x, uint32_t n, uint32_t dp, void* hbuf, float* scores,
                uint32_t P, uint32_t* probes, unsigned* err) {
    NNM_CUDA_TRY(set_attrs(m.d));
    if (!n) return 0;
    bf16* hb = static_cast<bf16*>(hbuf);
    k_ent_hidden<bf16><<<(n + ERB - 1) / ERB, 256, hidden_smem(m.d), ctx.stream>>>(view_of(m), x, dp, nullptr, n,
                                                                                  hb);
    const uint32_t grid = (n + PT - 1) / PT;
    if (scores)
        k_ent_tc<0><<<grid, 128, PROBE_SMEM, ctx.stream>>>(hb, n, m.w2r.as<bf16>(), m.b2.as<float>(), m.C, scores, 0,
                                                          nullptr, err);
    else
        k_ent_tc<1><<<grid, 128, PROBE_SMEM, ctx.stream>>>(hb, n, m.w2r.as<bf16>(), m.b2.as<float>(), m.C, nullptr, P,
                                                          probes, err);
    count_launch(2);
    NNM_CUDA_TRY(cudaGetLastError());
    return 0;
}

int entry_predict(Ctx& ctx, IndexDev& ix, const float* q, uint32_t nq, uint32_t* probes, unsigned* err) {
    NNM_CUDA_TRY(ix.hid.ensure((size_t)nq * EH * 2));
    return entry_infer(ctx, *ix.net, q, nq, ix.dp, ix.hid.p, nullptr, ix.nprobe, probes, err);
}

int entry_grad(Ctx& ctx, const nnm_entry_mlp& model, const float* x_dev, uint32_t n, uint32_t dp,
               const uint32_t* lab_host, float* loss, nnm_entry_mlp& grad) {
    const uint32_t d = model.d_in, C = model.n_classes, B = n;
    const ELayout L(d, C);
    EPass p;
    DevEntry m;
    int rc = alloc_pass(ctx, p, B, C, L);
    if (!rc) rc = alloc_model(ctx, m, d, C, model.in_scale, model.in_shift);
    if (rc) {
        m.release();
        return rc;
    }
    NNM_CUDA_TRY(p.loss.ensure(64));
    NNM_CUDA_TRY(set_attrs(d));
    std::vector<uint32_t> idx(B);
    for (uint32_t i = 0; i < B; i++) idx[i] = i;
    NNM_CUDA_TRY(cudaMemcpyAsync(p.idx.p, idx.data(), (size_t)B * 4, cudaMemcpyHostToDevice, ctx.stream));
    NNM_CUDA_TRY(cudaMemcpyAsync(p.lab.p, lab_host, (size_t)B * 4, cudaMemcpyHostToDevice, ctx.stream));
    std::vector<float> f = eflatten(model, L);
    NNM_CUDA_TRY(cudaMemcpyAsync(p.flat.p, f.data(), L.total * 4, cudaMemcpyHostToDevice, ctx.stream));
    refresh(p.flat.as<float>(), L, m, ctx.stream);
    enqueue_pass(pass_view(p, L, m), x_dev, dp, B, p, L, nullptr, ctx.stream);
    count_launch(1 + PASS_KERNELS);
    cudaError_t ce = cudaGetLastError();
    std::vector<float> g(L.total);
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(g.data(), p.grad.p, L.total * 4, cudaMemcpyDeviceToHost, ctx.stream);
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(loss, p.loss.p, 4, cudaMemcpyDeviceToHost, ctx.stream);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(ctx.stream);
    m.release();
    if (ce != cudaSuccess) {
        ctx.last_error = std::string("entry gradient: ") + cudaGetErrorString(ce);
        return 3;
    }
    eunflatten(g, L, grad);
    return 0;
}

int entry_train(Ctx& ctx, IndexDev& ix, uint32_t layer, const nnm_train_opts& o, nnm_entry_mlp& model,
                float* loss_trace) {
    const uint32_t d = model.d_in, C = model.n_classes, B = o.batch;
    const uint32_t npool = std::min<uint32_t>(ix.n, ENTRY_POOL);
    (void)layer;  // classes are rows 0..C-1, a prefix of every lower layer
    const ELayout L(d, C);
    EPass p;
    DevEntry m;
    DevBuf prow, plab;
    auto done = [&](int rc) {
        m.release();
        prow.release();
        plab.release();
        return rc;
    };
    int rc = alloc_pass(ctx, p, B, C, L);
    if (!rc) rc = alloc_model(ctx, m, d, C, model.in_scale, model.in_shift);
    if (rc) return done(rc);
    cudaStream_t st = ctx.stream;
    cudaError_t ce = cudaSuccess;
    auto chk = [&](cudaError_t e) {
        if (ce == cudaSuccess && e != cudaSuccess) ce = e;
    };
    chk(p.mom.ensure(L.total * 4));
    chk(p.vel.ensure(L.total * 4));
    chk(p.loss.ensure((size_t)o.steps * 4 + 64));
    chk(prow.ensure((size_t)npool * 4));
    chk(plab.ensure((size_t)npool * 4));
    chk(set_attrs(d));
    std::vector<float> f = eflatten(model, L);
    chk(cudaMemcpyAsync(p.flat.p, f.data(), L.total * 4, cudaMemcpyHostToDevice, st));
    chk(cudaMemsetAsync(p.mom.p, 0, L.total * 4, st));
    chk(cudaMemsetAsync(p.vel.p, 0, L.total * 4, st));
    chk(cudaMemsetAsync(p.step.p, 0, 4, st));
    if (ce != cudaSuccess) {
        ctx.last_error = std::string("entry training setup: ") + cudaGetErrorString(ce);
        return done(ce == cudaErrorMemoryAllocation ? 4 : 3);
    }
    // training pool and its labels
    k_ent_pool<<<(npool + 255) / 256, 256, 0, st>>>(prow.as<uint32_t>(), npool, ix.n, o.seed);
    k_ent_labels<<<(npool + LR - 1) / LR, 256, (LR + LC) * (d + 1) * 4, st>>>(
        ix.x.as<float>(), ix.dp, d, prow.as<uint32_t>(), npool, C, plab.as<uint32_t>());
    float* fl = p.flat.as<float>();
    refresh(fl, L, m, st);
    count_launch(3);
    chk(cudaGetLastError());
    chk(cudaStreamSynchronize(st));
    if (ce != cudaSuccess) {
        ctx.last_error = std::string("entry training labels: ") + cudaGetErrorString(ce);
        return done(3);
    }
    const EView v = pass_view(p, L, m);
    uint32_t* step = p.step.as<uint32_t>();
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    ce = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
    if (ce != cudaSuccess) {
        ctx.last_error = std::string("entry training capture: ") + cudaGetErrorString(ce);
        return done(3);
    }
    k_ent_sample<<<(B + 255) / 256, 256, 0, st>>>(p.idx.as<uint32_t>(), p.lab.as<uint32_t>(), B, prow.as<uint32_t>(),
                                                 plab.as<uint32_t>(), npool, o.seed, step);
    enqueue_pass(v, ix.x.as<float>(), ix.dp, B, p, L, step, st);
    launch_adam(fl, p.mom.as<float>(), p.vel.as<float>(), p.grad.as<float>(), (uint32_t)L.total, o.lr, step, st);
    refresh(fl, L, m, st);
    k_ent_step_inc<<<1, 1, 0, st>>>(step);
    ce = cudaStreamEndCapture(st, &graph);
    if (ce != cudaSuccess) {
        ctx.last_error = std::string("entry training capture: ") + cudaGetErrorString(ce);
        return done(3);
    }
    ce = cudaGraphInstantiate(&exec, graph, 0);
    for (uint32_t s = 0; s < o.steps && ce == cudaSuccess; s++) {
        ce = cudaGraphLaunch(exec, st);
        count_launch(STEP_KERNELS);
    }
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
    if (exec) cudaGraphExecDestroy(exec);
    cudaGraphDestroy(graph);
    if (ce == cudaSuccess) ce = cudaMemcpy(f.data(), p.flat.p, L.total * 4, cudaMemcpyDeviceToHost);
    if (ce == cudaSuccess && loss_trace)
        ce = cudaMemcpy(loss_trace, p.loss.p, (size_t)o.steps * 4, cudaMemcpyDeviceToHost);
    if (ce != cudaSuccess) {
        ctx.last_error = std::string("entry training: ") + cudaGetErrorString(ce);
        return done(3);
    }
    eunflatten(f, L, model);
    return done(0);
}

}  // namespace nnm
