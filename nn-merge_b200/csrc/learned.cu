// The code MLP of the learned initialisation: inference (32-bit sign codes)
// and training (triplet loss, backward, Adam) with hand-written kernels.
//
//   u = x * scale + shift            (d inputs, d <= 256)
//   h = relu(W1 u + b1)              (256)
//   z = W2 h + b2                    (32); code bit o = z_o > 0
//   t = tanh(z)
//   loss = mean_b max(0, margin + |t_a - t_p|^2 - |t_a - t_n|^2)
//
// Weights are BF16 on the device (rounded from FP32 master copies that Adam
// updates), every product is accumulated in FP32.  Gradients are taken with
// respect to the BF16 weights (the master copy is updated with them).
//
// One training step -- triplet sampling (Philox), forward, loss, backward,
// Adam, BF16 refresh, step counter -- is captured once as a CUDA graph and
// replayed `steps` times; the step counter lives on the device so that the
// replays draw new triplets and apply the right Adam bias correction.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "nnm_launch.h"
#include "nnm_learned.h"
#include "nnm_tc.cuh"

namespace nnm {
namespace {

constexpr uint32_t RB = 32;  // rows per forward block
constexpr int FWD_THREADS = 256;
constexpr uint64_t STEP_KERNELS = 10;  // kernels of one captured training step

__device__ __forceinline__ float bf(__nv_bfloat16 v) { return __bfloat162float(v); }

MlpView view_of(const DevMlp& m) {
    return MlpView{m.w1t.as<__nv_bfloat16>(), m.b1.as<float>(), m.w2t.as<__nv_bfloat16>(), m.b2.as<float>(), m.d,
                   m.scale, m.shift};
}

size_t fwd_smem(uint32_t d) { return ((size_t)RB * ((d + 3) & ~3u) + (size_t)RB * MLP_H) * 4; }

// Forward of RB rows per block.  Row r of the block is x row idx[r0 + r]
// (training) or r0 + r (inference).  Training writes h (rows x 256) and
// t = tanh(z) (rows x 32); inference writes the codes and, optionally, z.
template <bool TRAIN>
__global__ void __launch_bounds__(FWD_THREADS) k_mlp_fwd(MlpView m, const float* __restrict__ x, uint32_t dp,
                                                         const uint32_t* __restrict__ idx, uint32_t nrows,
                                                         float* __restrict__ h_out, float* __restrict__ t_out,
                                                         uint32_t* __restrict__ codes, float* __restrict__ z_out) {
    extern __shared__ float sm[];
    const uint32_t d = m.d, dpad = (d + 3) & ~3u;
    float* us = sm;
    float* hs = sm + RB * dpad;
    const uint32_t tid = threadIdx.x, r0 = blockIdx.x * RB;
    for (uint32_t i = tid; i < RB * dpad; i += FWD_THREADS) {
        const uint32_t r = i / dpad, k = i - r * dpad, gr = r0 + r;
        float v = 0.f;
        if (gr < nrows && k < d) {
            const size_t row = TRAIN ? idx[gr] : gr;
            v = fmaf(x[row * dp + k], m.scale, m.shift);
        }
        us[i] = v;
    }
    __syncthreads();
    {
        const uint32_t j = tid;  // hidden unit
        float acc[RB];
        const float bj = m.b1[j];
#pragma unroll
        for (uint32_t r = 0; r < RB; r++) acc[r] = bj;
        for (uint32_t k = 0; k < dpad; k += 4) {
            float w[4];
#pragma unroll
            for (int q = 0; q < 4; q++) w[q] = k + q < d ? bf(m.w1t[(size_t)(k + q) * MLP_H + j]) : 0.f;
#pragma unroll
            for (uint32_t r = 0; r < RB; r++) {
                const float4 u = *reinterpret_cast<const float4*>(us + r * dpad + k);
                acc[r] = fmaf(u.x, w[0], acc[r]);
                acc[r] = fmaf(u.y, w[1], acc[r]);
                acc[r] = fmaf(u.z, w[2], acc[r]);
                acc[r] = fmaf(u.w, w[3], acc[r]);
            }
        }
#pragma unroll
        for (uint32_t r = 0; r < RB; r++) {
            const float h = fmaxf(acc[r], 0.f);
            hs[r * MLP_H + j] = h;
            if (TRAIN && r0 + r < nrows) h_out[(size_t)(r0 + r) * MLP_H + j] = h;
        }
    }
    __syncthreads();
    const uint32_t warp = tid >> 5, o = tid & 31;  // output unit = lane
    constexpr uint32_t RPW = RB / (FWD_THREADS / 32);
    float acc[RPW];
    const float bo = m.b2[o];
#pragma unroll
    for (uint32_t q = 0; q < RPW; q++) acc[q] = bo;
    for (uint32_t j = 0; j < MLP_H; j++) {
        const float w = bf(m.w2t[j * MLP_O + o]);
#pragma unroll
        for (uint32_t q = 0; q < RPW; q++) acc[q] = fmaf(hs[(warp * RPW + q) * MLP_H + j], w, acc[q]);
    }
#pragma unroll
    for (uint32_t q = 0; q < RPW; q++) {
        const uint32_t gr = r0 + warp * RPW + q;
        const float z = acc[q];
        const unsigned code = __ballot_sync(0xffffffffu, z > 0.f);
        if (gr < nrows) {
            if (TRAIN) {
                t_out[(size_t)gr * MLP_O + o] = tanhf(z);
            } else {
                if (o == 0) codes[gr] = code;
                if (z_out) z_out[(size_t)gr * MLP_O + o] = z;
            }
        }
    }
}

// Inference on the tensor cores (d <= 128): a CTA per SM, 128 rows per
// tile.  Layer 1 is one tcgen05 kind::f16 MMA chain D = U W1^T (M = 128
// rows, N = 256 hidden units, FP32 accumulators in 256 TMEM columns) over
// u = x * scale + shift split into three BF16 parts u = hi + mid + lo
// (successive rounding residuals; a float's 24 significant bits in three
// 8-bit parts): W1 is BF16 and every product of BF16 values is exact in
// FP32, so layer 1 is the FP32 dot product of the CUDA-core kernel up to
// the order of its sums.  The epilogue reads the row's hidden accumulators
// (TMEM lane = row), adds b1, applies relu and accumulates layer 2 in FP32
// on the CUDA cores (W2 in shared memory, read as broadcasts); the two warps
// of a TMEM lane quarter take 128 hidden units each and add their partial
// outputs through shared memory.  Operands in the 128-byte swizzle K-major
// layout: W1 (256 rows) staged once per CTA, the three parts of U per tile.
// The MMA wait is bounded; when it runs out the CTA records the failure,
// waits (bounded) once more, frees its TMEM and returns.
constexpr uint32_t MT_ROWS = 128, MT_THREADS = 256, MT_MAX_D = 128;
// Instruction descriptor of kind::f16: D = F32 (bits 4-5 = 1), A = B = BF16
// (bits 7-9 = 1, 10-12 = 1), both K-major, N = 256 (N >> 3 at bit 17),
// M = 128 (M >> 4 at bit 24).
constexpr uint32_t MT_IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((MLP_H >> 3) << 17) | ((MT_ROWS >> 4) << 24);

__host__ __device__ constexpr uint32_t mt_dk(uint32_t d) { return (d + 15) & ~15u; }    // K: 16 per MMA
__host__ __device__ constexpr uint32_t mt_cols(uint32_t d) { return (mt_dk(d) + 63) / 64; }  // 128-B columns
__host__ __device__ constexpr size_t mt_w1_bytes(uint32_t d) { return (size_t)mt_cols(d) * MLP_H * 128; }
__host__ __device__ constexpr size_t mt_part_bytes(uint32_t d) { return (size_t)mt_cols(d) * MT_ROWS * 128; }
// W1, the three parts of U, W2 (FP32), b1, b2, the partial outputs (128 rows
// of 33 floats)
__host__ __device__ constexpr size_t mt_smem_bytes(uint32_t d) {
    return mt_w1_bytes(d) + 3 * mt_part_bytes(d) + (size_t)MLP_H * MLP_O * 4 + MLP_H * 4 + MLP_O * 4 +
           (size_t)MT_ROWS * 33 * 4;
}

// Byte offset of 16-byte chunk `kc` (elements 8 kc .. 8 kc + 7) of row r in
// a swizzled K-major operand of `rows` rows.
__device__ __forceinline__ uint32_t mt_chunk(uint32_t r, uint32_t kc, uint32_t rows) {
    return (kc >> 3) * rows * 128 + r * 128 + (((kc & 7) ^ (r & 7)) << 4);
}

__device__ __forceinline__ uint32_t pack_bf16(float a, float b) {
    const __nv_bfloat162 v = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<const uint32_t*>(&v);
}

__global__ void __launch_bounds__(MT_THREADS, 1) k_mlp_tc(MlpView m, const float* __restrict__ x, uint32_t dp,
                                                          uint32_t nrows, uint32_t* __restrict__ codes,
                                                          float* __restrict__ z_out, unsigned* err) {
    extern __shared__ __align__(1024) unsigned char smem[];
    __shared__ uint64_t mma_bar_s;
    __shared__ uint32_t tmem_s;
    const uint32_t tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t d = m.d, dk = mt_dk(d), nkc = dk / 8;
    unsigned char* w1s = smem;
    unsigned char* us = w1s + mt_w1_bytes(d);
    float* w2s = reinterpret_cast<float*>(us + 3 * mt_part_bytes(d));
    float* b1s = w2s + MLP_H * MLP_O;
    float* b2s = b1s + MLP_H;
    float* zp = b2s + MLP_O;
    const uint32_t mma_bar = smem_u32(&mma_bar_s);
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mma_bar));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_s)),
                     "r"(MLP_H));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    // the weights, once: W1 row j (hidden unit) = column j of w1t, zero past d
    for (uint32_t i = tid; i < MLP_H * nkc; i += MT_THREADS) {
        const uint32_t j = i % MLP_H, kc = i / MLP_H;
        uint32_t w[4];
#pragma unroll
        for (int t = 0; t < 4; t++) {
            const uint32_t k = kc * 8 + 2 * t;
            const float a = k < d ? bf(m.w1t[(size_t)k * MLP_H + j]) : 0.f;
            const float b = k + 1 < d ? bf(m.w1t[(size_t)(k + 1) * MLP_H + j]) : 0.f;
            w[t] = pack_bf16(a, b);  // exact: the values are BF16
        }
        *reinterpret_cast<uint4*>(w1s + mt_chunk(j, kc, MLP_H)) = make_uint4(w[0], w[1], w[2], w[3]);
    }
    for (uint32_t i = tid; i < MLP_H * MLP_O; i += MT_THREADS) w2s[i] = bf(m.w2t[i]);
    for (uint32_t i = tid; i < MLP_H; i += MT_THREADS) b1s[i] = m.b1[i];
    if (tid < MLP_O) b2s[tid] = m.b2[tid];
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // generic writes -> tensor core reads
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = tmem_s;
    uint32_t phase = 0;
    bool failed = false;
    const uint32_t ntiles = (nrows + MT_ROWS - 1) / MT_ROWS;
    for (uint32_t t = blockIdx.x; t < ntiles && !failed; t += gridDim.x) {
        const uint32_t r0 = t * MT_ROWS;
        // U's three parts: chunk kc of row r from two float4 of x (zero past d
        // and past the last row)
        for (uint32_t i = tid; i < MT_ROWS * nkc; i += MT_THREADS) {
            const uint32_t r = i / nkc, kc = i - r * nkc, k0 = kc * 8;
            float u[8];
#pragma unroll
            for (int h = 0; h < 2; h++) {
                float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
                if (r0 + r < nrows && k0 + 4 * h < d)
                    v = __ldg(reinterpret_cast<const float4*>(x + (size_t)(r0 + r) * dp + k0 + 4 * h));
                const float e[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
                for (int c = 0; c < 4; c++) {
                    const uint32_t k = k0 + 4 * h + c;
                    u[4 * h + c] = (r0 + r < nrows && k < d) ? fmaf(e[c], m.scale, m.shift) : 0.f;
                }
            }
            uint32_t ph[4], pm[4], pl[4];
#pragma unroll
            for (int c = 0; c < 4; c++) {
                float hi[2], mi[2], lo[2];
#pragma unroll
                for (int s = 0; s < 2; s++) {
                    const float v = u[2 * c + s];
                    hi[s] = __bfloat162float(__float2bfloat16_rn(v));
                    const float r1 = v - hi[s];
                    mi[s] = __bfloat162float(__float2bfloat16_rn(r1));
                    lo[s] = r1 - mi[s];
                }
                ph[c] = pack_bf16(hi[0], hi[1]);
                pm[c] = pack_bf16(mi[0], mi[1]);
                pl[c] = pack_bf16(lo[0], lo[1]);
            }
            const uint32_t off = mt_chunk(r, kc, MT_ROWS);
            *reinterpret_cast<uint4*>(us + off) = make_uint4(ph[0], ph[1], ph[2], ph[3]);
            *reinterpret_cast<uint4*>(us + mt_part_bytes(d) + off) = make_uint4(pm[0], pm[1], pm[2], pm[3]);
            *reinterpret_cast<uint4*>(us + 2 * mt_part_bytes(d) + off) = make_uint4(pl[0], pl[1], pl[2], pl[3]);
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // generic writes -> tensor core reads
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;");
            const uint32_t wb = smem_u32(w1s), ub = smem_u32(us);
            for (uint32_t part = 0; part < 3; part++)
                for (uint32_t kk = 0; kk < dk / 16; kk++) {
                    const uint32_t koff = kk * 32;  // bytes into the operand row
                    const uint64_t da = smem_desc_sw128(ub + part * (uint32_t)mt_part_bytes(d) +
                                                        (koff >> 7) * MT_ROWS * 128 + (koff & 127));
                    const uint64_t db = smem_desc_sw128(wb + (koff >> 7) * MLP_H * 128 + (koff & 127));
                    asm volatile(
                        "{\n\t.reg .pred p;\n\t"
                        "setp.ne.b32 p, %4, 0;\n\t"
                        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem),
                        "l"(da), "l"(db), "r"(MT_IDESC), "r"(part | kk), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
                }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mma_bar)
                         : "memory");
        }
        const bool ok = mbar_wait_bounded(mma_bar, phase);
        if (__syncthreads_or(!ok)) {
            failed = true;
            break;
        }
        phase ^= 1u;
        asm volatile("tcgen05.fence::after_thread_sync;");
        // epilogue: row r0 + 32 quarter + lane, hidden units [128 half, + 128)
        const uint32_t quarter = warp & 3, half = warp >> 2, rl = quarter * 32 + lane;
        float z[MLP_O];
#pragma unroll
        for (uint32_t o = 0; o < MLP_O; o++) z[o] = 0.f;
        for (uint32_t c0 = 0; c0 < MLP_H / 2; c0 += 8) {
            const uint32_t j0 = half * (MLP_H / 2) + c0;
            uint32_t v[8];
            tmem_ld8(tmem + ((quarter * 32) << 16) + j0, v);
#pragma unroll
            for (uint32_t jj = 0; jj < 8; jj++) {
                const float h = fmaxf(__uint_as_float(v[jj]) + b1s[j0 + jj], 0.f);
                const float4* w = reinterpret_cast<const float4*>(w2s + (j0 + jj) * MLP_O);
#pragma unroll
                for (uint32_t o4 = 0; o4 < MLP_O / 4; o4++) {
                    const float4 wv = w[o4];
                    z[4 * o4] = fmaf(h, wv.x, z[4 * o4]);
                    z[4 * o4 + 1] = fmaf(h, wv.y, z[4 * o4 + 1]);
                    z[4 * o4 + 2] = fmaf(h, wv.z, z[4 * o4 + 2]);
                    z[4 * o4 + 3] = fmaf(h, wv.w, z[4 * o4 + 3]);
                }
            }
        }
        if (half == 1)
#pragma unroll
            for (uint32_t o = 0; o < MLP_O; o++) zp[rl * 33 + o] = z[o];
        asm volatile("tcgen05.fence::before_thread_sync;");
        __syncthreads();  // partial outputs written; TMEM and U read before the next tile's MMA
        if (half == 0 && r0 + rl < nrows) {
            uint32_t code = 0;
#pragma unroll
            for (uint32_t o = 0; o < MLP_O; o++) {
                const float zo = z[o] + zp[rl * 33 + o] + b2s[o];
                code |= (zo > 0.f ? 1u : 0u) << o;
                if (z_out) z_out[(size_t)(r0 + rl) * MLP_O + o] = zo;
            }
            codes[r0 + rl] = code;
        }
    }
    if (failed) {
        if (tid == 0) atomicOr(err, 1u);
        mbar_wait_bounded(mma_bar, phase);  // the MMA may still write TMEM
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(MLP_H));
    }
}

// Warp per triplet: loss term and dL/dz of its three rows.  Per-block loss
// partial sums in a fixed order (deterministic).
__global__ void k_triplet(const float* __restrict__ t, uint32_t B, float margin, float* __restrict__ dz,
                          float* __restrict__ partial) {
    __shared__ float wl[8];
    const uint32_t warp = threadIdx.x >> 5, o = threadIdx.x & 31;
    const uint32_t b = blockIdx.x * 8 + warp;
    float l = 0.f;
    if (b < B) {
        const float ta = t[(size_t)b * MLP_O + o], tp = t[(size_t)(B + b) * MLP_O + o],
                    tn = t[(size_t)(2 * B + b) * MLP_O + o];
        float dp = (ta - tp) * (ta - tp), dn = (ta - tn) * (ta - tn);
        for (int s = 16; s > 0; s >>= 1) {
            dp += __shfl_xor_sync(0xffffffffu, dp, s);
            dn += __shfl_xor_sync(0xffffffffu, dn, s);
        }
        l = fmaxf(margin + dp - dn, 0.f);
        const float sc = l > 0.f ? 2.f / (float)B : 0.f;
        const float ga = sc * (tn - tp), gp = -sc * (ta - tp), gn = sc * (ta - tn);
        dz[(size_t)b * MLP_O + o] = ga * (1.f - ta * ta);
        dz[(size_t)(B + b) * MLP_O + o] = gp * (1.f - tp * tp);
        dz[(size_t)(2 * B + b) * MLP_O + o] = gn * (1.f - tn * tn);
    }
    if (o == 0) wl[warp] = l;
    __syncthreads();
    if (threadIdx.x == 0) {
        float s = 0.f;
        for (int w = 0; w < 8; w++) s += wl[w];
        partial[blockIdx.x] = s;
    }
}

__global__ void k_loss_final(const float* partial, uint32_t nblk, uint32_t B, float* loss, const uint32_t* step) {
    float s = 0.f;
    for (uint32_t i = 0; i < nblk; i++) s += partial[i];
    loss[step ? *step : 0] = s / (float)B;
}

// dL/d(pre-activation of h): (h > 0) * sum_o dz_o W2[o][j].
__global__ void k_bwd_h(const float* __restrict__ dz, const float* __restrict__ h, MlpView m, uint32_t R,
                        float* __restrict__ dh) {
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (size_t)R * MLP_H) return;
    const uint32_t r = (uint32_t)(t / MLP_H), j = (uint32_t)(t - (size_t)r * MLP_H);
    float acc = 0.f;
#pragma unroll 8
    for (uint32_t o = 0; o < MLP_O; o++) acc = fmaf(dz[(size_t)r * MLP_O + o], bf(m.w2t[j * MLP_O + o]), acc);
    dh[t] = h[t] > 0.f ? acc : 0.f;
}

// Block o: dW2[o][j] = sum_r dz[r][o] h[r][j] (thread j), db2[o].
__global__ void k_grad_w2(const float* __restrict__ dz, const float* __restrict__ h, uint32_t R,
                          float* __restrict__ gw2, float* __restrict__ gb2) {
    __shared__ float red[MLP_H];
    const uint32_t o = blockIdx.x, j = threadIdx.x;
    float acc = 0.f, sb = 0.f;
    for (uint32_t r = 0; r < R; r++) acc = fmaf(dz[(size_t)r * MLP_O + o], h[(size_t)r * MLP_H + j], acc);
    for (uint32_t r = j; r < R; r += MLP_H) sb += dz[(size_t)r * MLP_O + o];
    gw2[(size_t)o * MLP_H + j] = acc;
    red[j] = sb;
    __syncthreads();
    for (uint32_t s = MLP_H / 2; s > 0; s >>= 1) {
        if (j < s) red[j] += red[j + s];
        __syncthreads();
    }
    if (j == 0) gb2[o] = red[0];
}

// Block j: dW1[j][k] = sum_r dh[r][j] u[r][k] (thread k), db1[j].
__global__ void k_grad_w1(const float* __restrict__ dh, const float* __restrict__ x, uint32_t dp,
                          const uint32_t* __restrict__ idx, uint32_t R, MlpView m, float* __restrict__ gw1,
                          float* __restrict__ gb1) {
    __shared__ float red[256];
    const uint32_t j = blockIdx.x, k = threadIdx.x;
    float acc = 0.f, sb = 0.f;
    if (k < m.d)
        for (uint32_t r = 0; r < R; r++)
            acc = fmaf(dh[(size_t)r * MLP_H + j], fmaf(x[(size_t)idx[r] * dp + k], m.scale, m.shift), acc);
    for (uint32_t r = k; r < R; r += blockDim.x) sb += dh[(size_t)r * MLP_H + j];
    if (k < m.d) gw1[(size_t)j * m.d + k] = acc;
    red[k] = sb;
    __syncthreads();
    for (uint32_t s = blockDim.x / 2; s > 0; s >>= 1) {
        if (k < s) red[k] += red[k + s];
        __syncthreads();
    }
    if (k == 0) gb1[j] = red[0];
}

// Adam (Kingma & Ba, 2015) on the flat parameter vector, step t = *step + 1.
__global__ void k_adam(float* __restrict__ p, float* __restrict__ mo, float* __restrict__ ve,
                       const float* __restrict__ g, uint32_t cnt, float lr, const uint32_t* step) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= cnt) return;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    const float t = (float)(*step + 1);
    const float m = b1 * mo[i] + (1.f - b1) * g[i];
    const float v = b2 * ve[i] + (1.f - b2) * g[i] * g[i];
    mo[i] = m;
    ve[i] = v;
    const float mh = m / (1.f - powf(b1, t)), vh = v / (1.f - powf(b2, t));
    p[i] -= lr * mh / (sqrtf(vh) + eps);
}

// BF16 transposed copies of the master weights.
__global__ void k_refresh(const float* __restrict__ w1, const float* __restrict__ w2, uint32_t d,
                          __nv_bfloat16* __restrict__ w1t, __nv_bfloat16* __restrict__ w2t) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < MLP_H * d) {
        const uint32_t j = i / d, k = i - j * d;
        w1t[(size_t)k * MLP_H + j] = __float2bfloat16_rn(w1[i]);
    }
    if (i < MLP_O * MLP_H) {
        const uint32_t o = i / MLP_H, j = i - o * MLP_H;
        w2t[j * MLP_O + o] = __float2bfloat16_rn(w2[i]);
    }
}

__global__ void k_sample_triplets(uint32_t* idx, uint32_t B, uint32_t n, const uint32_t* graph, uint32_t K,
                                  uint32_t seed, const uint32_t* step) {
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= B) return;
    const Philox ph{seed, 0x6e6e6d10u};
    const uint4 r = ph(b, *step, 0, 0);
    const uint32_t a = bounded(r.x, n);
    idx[b] = a;
    idx[B + b] = graph[(size_t)a * K + bounded(r.y, K)] & ID_MASK;
    idx[2 * B + b] = bounded(r.z, n);
}

__global__ void k_step_inc(uint32_t* step) { *step += 1; }

// Parameter layout of the flat training vectors: W1 (256 x d), b1, W2 (32 x 256), b2.
struct Layout {
    size_t w1, b1, w2, b2, total;
    explicit Layout(uint32_t d)
        : w1(0), b1((size_t)MLP_H * d), w2(b1 + MLP_H), b2(w2 + (size_t)MLP_O * MLP_H), total(b2 + MLP_O) {}
};

cudaError_t set_fwd_attrs(uint32_t d) {
    cudaError_t e = cudaFuncSetAttribute(k_mlp_fwd<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fwd_smem(d));
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(k_mlp_fwd<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fwd_smem(d));
}

// Scratch of one training/gradient pass over B triplets.
struct Pass {
    DevBuf idx, h, t, dz, dh, partial, flat, grad, mom, vel, w1t, w2t, loss, step;
    ~Pass() {
        for (DevBuf* b : {&idx, &h, &t, &dz, &dh, &partial, &flat, &grad, &mom, &vel, &w1t, &w2t, &loss, &step})
            b->release();
    }
};

// Forward + loss + backward over the triplets in p.idx; gradients into p.grad.
void enqueue_pass(const MlpView& mv, const float* x, uint32_t dp, uint32_t B, float margin, Pass& p,
                  const Layout& L, const uint32_t* step, cudaStream_t st) {
    const uint32_t R = 3 * B;
    k_mlp_fwd<true><<<(R + RB - 1) / RB, FWD_THREADS, fwd_smem(mv.d), st>>>(mv, x, dp, p.idx.as<uint32_t>(), R,
                                                                           p.h.as<float>(), p.t.as<float>(),
                                                                           nullptr, nullptr);
    const uint32_t nblk = (B + 7) / 8;
    k_triplet<<<nblk, 256, 0, st>>>(p.t.as<float>(), B, margin, p.dz.as<float>(), p.partial.as<float>());
    k_loss_final<<<1, 1, 0, st>>>(p.partial.as<float>(), nblk, B, p.loss.as<float>(), step);
    k_bwd_h<<<(unsigned)(((size_t)R * MLP_H + 255) / 256), 256, 0, st>>>(p.dz.as<float>(), p.h.as<float>(), mv, R,
                                                                        p.dh.as<float>());
    float* g = p.grad.as<float>();
    k_grad_w2<<<MLP_O, MLP_H, 0, st>>>(p.dz.as<float>(), p.h.as<float>(), R, g + L.w2, g + L.b2);
    k_grad_w1<<<MLP_H, 256, 0, st>>>(p.dh.as<float>(), x, dp, p.idx.as<uint32_t>(), R, mv, g + L.w1, g + L.b1);
}

int alloc_pass(Ctx& ctx, Pass& p, uint32_t B, const Layout& L, uint32_t d) {
    const size_t R = 3 * (size_t)B;
    NNM_CUDA_TRY(p.idx.ensure(R * 4));
    NNM_CUDA_TRY(p.h.ensure(R * MLP_H * 4));
    NNM_CUDA_TRY(p.t.ensure(R * MLP_O * 4));
    NNM_CUDA_TRY(p.dz.ensure(R * MLP_O * 4));
    NNM_CUDA_TRY(p.dh.ensure(R * MLP_H * 4));
    NNM_CUDA_TRY(p.partial.ensure(((B + 7) / 8) * 4 + 64));
    NNM_CUDA_TRY(p.flat.ensure(L.total * 4));
    NNM_CUDA_TRY(p.grad.ensure(L.total * 4));
    NNM_CUDA_TRY(p.w1t.ensure((size_t)d * MLP_H * 2));
    NNM_CUDA_TRY(p.w2t.ensure((size_t)MLP_H * MLP_O * 2));
    NNM_CUDA_TRY(p.step.ensure(64));
    return 0;
}

// Host model -> flat FP32 vector.
std::vector<float> flatten(const nnm_mlp& m, const Layout& L) {
    std::vector<float> f(L.total);
    std::memcpy(f.data() + L.w1, m.w1, (size_t)MLP_H * m.d_in * 4);
    std::memcpy(f.data() + L.b1, m.b1, MLP_H * 4);
    std::memcpy(f.data() + L.w2, m.w2, (size_t)MLP_O * MLP_H * 4);
    std::memcpy(f.data() + L.b2, m.b2, MLP_O * 4);
    return f;
}

void unflatten(const std::vector<float>& f, const Layout& L, nnm_mlp& m) {
    std::memcpy(m.w1, f.data() + L.w1, (size_t)MLP_H * m.d_in * 4);
    std::memcpy(m.b1, f.data() + L.b1, MLP_H * 4);
    std::memcpy(m.w2, f.data() + L.w2, (size_t)MLP_O * MLP_H * 4);
    std::memcpy(m.b2, f.data() + L.b2, MLP_O * 4);
}

MlpView pass_view(const Pass& p, const Layout& L, const nnm_mlp& m) {
    const float* f = p.flat.as<float>();
    return MlpView{p.w1t.as<__nv_bfloat16>(), f + L.b1, p.w2t.as<__nv_bfloat16>(), f + L.b2, m.d_in, m.in_scale,
                   m.in_shift};
}

}  // namespace

void launch_grad_w1(const float* dh, const float* x, uint32_t dp, const uint32_t* idx, uint32_t R, uint32_t d,
                    float scale, float shift, float* gw1, float* gb1, cudaStream_t st) {
    MlpView m{};
    m.d = d;
    m.scale = scale;
    m.shift = shift;
    k_grad_w1<<<MLP_H, 256, 0, st>>>(dh, x, dp, idx, R, m, gw1, gb1);
}

void launch_adam(float* p, float* mo, float* ve, const float* g, uint32_t cnt, float lr, const uint32_t* step,
                 cudaStream_t st) {
    k_adam<<<(cnt + 255) / 256, 256, 0, st>>>(p, mo, ve, g, cnt, lr, step);
}

int mlp_upload(Ctx& ctx, DevMlp& m, const nnm_mlp& h) {
    const uint32_t d = h.d_in;
    const Layout L(d);
    std::vector<float> f = flatten(h, L);
    DevBuf tmp;
    NNM_CUDA_TRY(tmp.ensure(L.total * 4));
    NNM_CUDA_TRY(m.w1t.ensure((size_t)d * MLP_H * 2));
    NNM_CUDA_TRY(m.w2t.ensure((size_t)MLP_H * MLP_O * 2));
    NNM_CUDA_TRY(m.b1.ensure(MLP_H * 4));
    NNM_CUDA_TRY(m.b2.ensure(MLP_O * 4));
    NNM_CUDA_TRY(cudaMemcpyAsync(tmp.p, f.data(), L.total * 4, cudaMemcpyHostToDevice, ctx.stream));
    const float* t = tmp.as<float>();
    k_refresh<<<(MLP_H * d + 255) / 256, 256, 0, ctx.stream>>>(t + L.w1, t + L.w2, d, m.w1t.as<__nv_bfloat16>(),
                                                             m.w2t.as<__nv_bfloat16>()); count_launch();
    NNM_CUDA_TRY(cudaMemcpyAsync(m.b1.p, t + L.b1, MLP_H * 4, cudaMemcpyDeviceToDevice, ctx.stream));
    NNM_CUDA_TRY(cudaMemcpyAsync(m.b2.p, t + L.b2, MLP_O * 4, cudaMemcpyDeviceToDevice, ctx.stream));
    NNM_CUDA_TRY(cudaStreamSynchronize(ctx.stream));
    tmp.release();
    m.d = d;
    m.scale = h.in_scale;
    m.shift = h.in_shift;
    return 0;
}

// Inference: on the tensor cores (k_mlp_tc) for d <= 128 when its shared
// memory fits, else the CUDA-core forward.
int mlp_codes_dev(Ctx& ctx, const DevMlp& m, const float* x, uint32_t n, uint32_t dp, uint32_t* codes, float* z) {
    NNM_CUDA_TRY(set_fwd_attrs(m.d));
    if (!n) return 0;
    int optin = 0, nsm = 148;
    NNM_CUDA_TRY(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, ctx.device));
    NNM_CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, ctx.device));
    if (m.d <= MT_MAX_D && mt_smem_bytes(m.d) <= (size_t)optin) {
        NNM_CUDA_TRY(cudaFuncSetAttribute(k_mlp_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)mt_smem_bytes(m.d)));
        NNM_CUDA_TRY(ctx.ws.mlp_err.ensure(64));
        NNM_CUDA_TRY(cudaMemsetAsync(ctx.ws.mlp_err.p, 0, 4, ctx.stream));
        const uint32_t tiles = (n + MT_ROWS - 1) / MT_ROWS;
        k_mlp_tc<<<std::min<uint32_t>(tiles, (uint32_t)nsm), MT_THREADS, mt_smem_bytes(m.d), ctx.stream>>>(
            view_of(m), x, dp, n, codes, z, ctx.ws.mlp_err.as<unsigned>()); count_launch();
        NNM_CUDA_TRY(cudaGetLastError());
        unsigned err = 0;
        NNM_CUDA_TRY(cudaMemcpyAsync(&err, ctx.ws.mlp_err.p, 4, cudaMemcpyDeviceToHost, ctx.stream));
        NNM_CUDA_TRY(cudaStreamSynchronize(ctx.stream));
        if (err) {
            ctx.last_error = "the code network's tensor-core wait ran out";
            return 6;
        }
        return 0;
    }
    k_mlp_fwd<false><<<(n + RB - 1) / RB, FWD_THREADS, fwd_smem(m.d), ctx.stream>>>(view_of(m), x, dp, nullptr, n,
                                                                                  nullptr, nullptr, codes, z); count_launch();
    NNM_CUDA_TRY(cudaGetLastError());
    return 0;
}

int mlp_grad(Ctx& ctx, const nnm_mlp& model, const float* x_dev, uint32_t n, uint32_t dp, const uint32_t* trip_host,
             uint32_t ntrip, float margin, float* loss, nnm_mlp& grad) {
    (void)n;
    const uint32_t d = model.d_in, B = ntrip;
    const Layout L(d);
    Pass p;
    int rc = alloc_pass(ctx, p, B, L, d);
    if (rc) return rc;
    NNM_CUDA_TRY(p.loss.ensure(64));
    NNM_CUDA_TRY(set_fwd_attrs(d));
    // triplets (anchor, positive, negative) -> idx = anchors | positives | negatives
    std::vector<uint32_t> h(3 * (size_t)B);
    for (uint32_t b = 0; b < B; b++)
        for (int c = 0; c < 3; c++) h[(size_t)c * B + b] = trip_host[(size_t)b * 3 + c];
    NNM_CUDA_TRY(cudaMemcpyAsync(p.idx.p, h.data(), h.size() * 4, cudaMemcpyHostToDevice, ctx.stream));
    std::vector<float> f = flatten(model, L);
    NNM_CUDA_TRY(cudaMemcpyAsync(p.flat.p, f.data(), L.total * 4, cudaMemcpyHostToDevice, ctx.stream));
    const float* fl = p.flat.as<float>();
    k_refresh<<<(MLP_H * d + 255) / 256, 256, 0, ctx.stream>>>(fl + L.w1, fl + L.w2, d, p.w1t.as<__nv_bfloat16>(),
                                                             p.w2t.as<__nv_bfloat16>()); count_launch();
    enqueue_pass(pass_view(p, L, model), x_dev, dp, B, margin, p, L, nullptr, ctx.stream);
    count_launch(6);
    NNM_CUDA_TRY(cudaGetLastError());
    std::vector<float> g(L.total);
    NNM_CUDA_TRY(cudaMemcpyAsync(g.data(), p.grad.p, L.total * 4, cudaMemcpyDeviceToHost, ctx.stream));
    NNM_CUDA_TRY(cudaMemcpyAsync(loss, p.loss.p, 4, cudaMemcpyDeviceToHost, ctx.stream));
    NNM_CUDA_TRY(cudaStreamSynchronize(ctx.stream));
    unflatten(g, L, grad);
    return 0;
}

int mlp_train(Ctx& ctx, const float* x_dev, uint32_t n, uint32_t dp, const uint32_t* graph_dev, uint32_t K,
              const nnm_train_opts& o, nnm_mlp& model, float* loss_trace) {
    const uint32_t d = model.d_in, B = o.batch;
    const Layout L(d);
    Pass p;
    int rc = alloc_pass(ctx, p, B, L, d);
    if (rc) return rc;
    NNM_CUDA_TRY(p.mom.ensure(L.total * 4));
    NNM_CUDA_TRY(p.vel.ensure(L.total * 4));
    NNM_CUDA_TRY(p.loss.ensure((size_t)o.steps * 4 + 64));
    NNM_CUDA_TRY(set_fwd_attrs(d));
    std::vector<float> f = flatten(model, L);
    cudaStream_t st = ctx.stream;
    NNM_CUDA_TRY(cudaMemcpyAsync(p.flat.p, f.data(), L.total * 4, cudaMemcpyHostToDevice, st));
    NNM_CUDA_TRY(cudaMemsetAsync(p.mom.p, 0, L.total * 4, st));
    NNM_CUDA_TRY(cudaMemsetAsync(p.vel.p, 0, L.total * 4, st));
    NNM_CUDA_TRY(cudaMemsetAsync(p.step.p, 0, 4, st));
    float* fl = p.flat.as<float>();
    k_refresh<<<(MLP_H * d + 255) / 256, 256, 0, st>>>(fl + L.w1, fl + L.w2, d, p.w1t.as<__nv_bfloat16>(),
                                                     p.w2t.as<__nv_bfloat16>()); count_launch();
    NNM_CUDA_TRY(cudaStreamSynchronize(st));
    const MlpView mv = pass_view(p, L, model);
    uint32_t* step = p.step.as<uint32_t>();
    // capture one step
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    NNM_CUDA_TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    k_sample_triplets<<<(B + 255) / 256, 256, 0, st>>>(p.idx.as<uint32_t>(), B, n, graph_dev, K, o.seed, step);
    enqueue_pass(mv, x_dev, dp, B, o.margin, p, L, step, st);
    k_adam<<<(unsigned)((L.total + 255) / 256), 256, 0, st>>>(fl, p.mom.as<float>(), p.vel.as<float>(),
                                                              p.grad.as<float>(), (uint32_t)L.total, o.lr, step);
    k_refresh<<<(MLP_H * d + 255) / 256, 256, 0, st>>>(fl + L.w1, fl + L.w2, d, p.w1t.as<__nv_bfloat16>(),
                                                     p.w2t.as<__nv_bfloat16>());
    k_step_inc<<<1, 1, 0, st>>>(step);
    cudaError_t ce = cudaStreamEndCapture(st, &graph);
    if (ce != cudaSuccess) {
        ctx.last_error = std::string("training step capture: ") + cudaGetErrorString(ce);
        return 3;
    }
    ce = cudaGraphInstantiate(&exec, graph, 0);
    if (ce == cudaSuccess) {
        for (uint32_t s = 0; s < o.steps && ce == cudaSuccess; s++) {
            ce = cudaGraphLaunch(exec, st);
            count_launch(STEP_KERNELS);
        }
    }
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
    if (exec) cudaGraphExecDestroy(exec);
    cudaGraphDestroy(graph);
    if (ce != cudaSuccess) {
        ctx.last_error = std::string("training: ") + cudaGetErrorString(ce);
        return 3;
    }
    NNM_CUDA_TRY(cudaMemcpy(f.data(), p.flat.p, L.total * 4, cudaMemcpyDeviceToHost));
    unflatten(f, L, model);
    if (loss_trace) NNM_CUDA_TRY(cudaMemcpy(loss_trace, p.loss.p, (size_t)o.steps * 4, cudaMemcpyDeviceToHost));
    return 0;
}

}  // namespace nnm
