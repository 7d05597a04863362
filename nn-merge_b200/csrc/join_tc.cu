// Local join on the 5th-generation tensor cores (tcgen05, TMEM accumulators).
//
// The join evaluates d(a, b) for every pair of a row's sample lists.  For the
// squared L2 metric d(a, b) = |a|^2 + |b|^2 - 2 a.b, so the distances of a
// row are its Gram matrix plus norms.  When every vector component is an
// integer in [0, 255] (checked on upload, k_quantize), the vectors are kept
// as u8 and the Gram matrix is computed by tcgen05.mma kind::i8 with S32
// accumulation: every product and sum is an exact integer, every distance is
// below 2^24, and the reference's sequential float sum (vmath.cpp:56-88) of
// the same integer terms is exact too -- the two agree bit for bit, so the
// graphs are identical to the FP32 path's.
//
// Tiles.  Rows of list size S <= 16, 32, 64, 128 (tiers 0-3) are packed 8,
// 4, 2, 1 to a tile of 128 slots; slot s holds list entry s % B of the
// tile's row s / B (B = 16 << tier).  One MMA chain (M = N = 128, K = 32 per
// instruction) computes the 128 x 128 slot Gram matrix into 128 TMEM
// columns; only its diagonal blocks are read.  The epilogue reads TMEM lane
// b (slot b) with tcgen05.ld; by symmetry column a of that lane is G(a, b),
// so lane b evaluates the pairs (a, b), a < b, of its row: a thread per
// "inner" slot, all lanes of a warp on the same "outer" column at a time.
//
// Two passes, as the FP32 path: pass 0 counts, per list slot, the proposals
// that pass the K-th-distance filter (the bucket sizes); pass 1 recomputes
// the distances and writes the proposals.  Nothing per pair is stored.
//
// Synchronisation: persistent CTAs of 256 threads, at most four per SM (the
// TMEM columns and the shared memory request both allow four), each holding
// 128 TMEM columns for its lifetime.  Producer warps load tile k+1 into one
// buffer while the consumer warps run tile k from the other (full/empty
// mbarriers per buffer); consumer thread 0 issues the MMAs and commits them
// to an mbarrier.  Every mbarrier wait is bounded in time; when a bound runs
// out the group stops (decided by a barrier-OR over its threads), the CTA
// records DERR_TC_WAIT, waits (bounded) once more for its MMA, frees its
// TMEM and returns.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <type_traits>

#include <cuda_bf16.h>

#include "../../include/nnm.h"
#include "nnm_engine.h"
#include "nnm_join.h"
#include "nnm_launch.h"
#include "nnm_tc.cuh"

namespace nnm {
namespace {

constexpr int TC_THREADS = 256;                // consumers (warps 0-3) + producers (warps 4-7)
constexpr uint32_t TC_SLOTS = 128;             // M = N = 128: one TMEM lane and one column per slot
constexpr uint32_t TC_COLS = 128;              // TMEM columns held by a CTA
constexpr uint32_t TC_SMEM_FLOOR = 50 * 1024;  // keeps residency at <= 4 CTAs per SM (4 x 128 columns)
constexpr uint32_t TC_MAX_KQ = 768;              // two tile buffers of 128 x kq bytes fit in shared memory
constexpr uint32_t NO_SLOT = 0xffffffffu;

// Instruction descriptor of kind::i8: D = S32 (bits 4-5 = 2), A = B = u8
// (bits 7-9 = 0, 10-12 = 0), both K-major, N >> 3 at bit 17, M >> 4 at bit 24.
constexpr uint32_t IDESC_U8 = (2u << 4) | ((TC_SLOTS >> 3) << 17) | ((TC_SLOTS >> 4) << 24);
// Instruction descriptor of kind::f16: D = F32 (bits 4-5 = 1), A = B = BF16
// (bits 7-9 = 1, 10-12 = 1), both K-major.
constexpr uint32_t IDESC_BF16 = (1u << 4) | (1u << 7) | (1u << 10) | ((TC_SLOTS >> 3) << 17) | ((TC_SLOTS >> 4) << 24);

// The reference's sequential FP32 distance of rows i and j: the BF16 tier's
// recheck, one non-inlined copy for every call site.
__device__ __noinline__ float exact_l2(const float* x, uint32_t dp, uint32_t i, uint32_t j) {
    return dist_seq<L2>(x + (size_t)i * dp, x + (size_t)j * dp, (int)dp);
}

// Tile header of one buffer, written by the producers, read by the consumers.
struct TileHdr {
    uint32_t t, lgB, nrows, pad;
    uint32_t row[8], nn[8], S[8], any[8];
};

struct TcShared {
    uint64_t mma_bar;           // MMA completion (tcgen05.commit)
    uint64_t full[2], empty[2];  // tile buffer b loaded / released
    uint32_t tmem;
    TileHdr hdr[2];
};

// Shared memory of one tile buffer: the slot vectors (128 x kq bytes,
// canonical K-major layout: 8-slot groups of kq/16 core matrices), then the
// per-slot arrays.  Two buffers.
__host__ __device__ constexpr size_t tc_vec_bytes(uint32_t kq) { return (size_t)TC_SLOTS * kq; }
__host__ __device__ constexpr size_t tc_buf_bytes(uint32_t kq) {
    return (tc_vec_bytes(kq) + (size_t)TC_SLOTS * (5 * 4 + 8) + 1023) & ~(size_t)1023;
}
__host__ __device__ constexpr size_t tc_smem_bytes(uint32_t kq) { return 2 * tc_buf_bytes(kq) + 1024; }

struct SlotBuf {
    unsigned char* vec;
    uint32_t* ids;
    float* kth;
    uint32_t* nrm;
    uint32_t* cnt;  // pass 0: counts; pass 1: bucket cursors
    uint32_t* grp;
    unsigned long long* base;
};

__device__ __forceinline__ SlotBuf slot_buf(unsigned char* smem, uint32_t kq, uint32_t b) {
    unsigned char* p = smem + b * tc_buf_bytes(kq);
    SlotBuf s;
    s.vec = p;
    s.ids = reinterpret_cast<uint32_t*>(p + tc_vec_bytes(kq));
    s.kth = reinterpret_cast<float*>(s.ids + TC_SLOTS);
    s.nrm = reinterpret_cast<uint32_t*>(s.kth + TC_SLOTS);
    s.cnt = s.nrm + TC_SLOTS;
    s.grp = s.cnt + TC_SLOTS;
    s.base = reinterpret_cast<unsigned long long*>(s.grp + TC_SLOTS);
    return s;
}

// Barriers of one 128-thread group (producers: 1, consumers: 2).
constexpr uint32_t BAR_PROD = 1, BAR_CONS = 2;

__device__ __forceinline__ void group_sync(uint32_t id) {
    asm volatile("bar.sync %0, 128;" ::"r"(id) : "memory");
}

// Barrier of the group that also ORs a predicate over its 128 threads, so
// that a decision taken after per-thread bounded waits is the same in every
// thread of the group.
__device__ __forceinline__ bool group_any(uint32_t id, bool p) {
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\t"
        "setp.ne.u32 p, %1, 0;\n\t"
        "bar.red.or.pred q, %2, 128, p;\n\t"
        "selp.u32 %0, 1, 0, q;\n\t}\n"
        : "=r"(r)
        : "r"((uint32_t)p), "r"(id)
        : "memory");
    return r != 0;
}

// Persistent CTAs of 256 threads in two groups over two tile buffers:
//   producers (warps 4-7): for tile k, wait until buffer k%2 is released,
//     write its header and slot metadata, gather the slot vectors with
//     cp.async, then arrive on full[k%2];
//   consumers (warps 0-3, TMEM lanes 0-127): wait for full[k%2], run the
//     MMA chain (thread 0) and the epilogue, write the counts, then arrive on
//     empty[k%2].
// So the loads of tile k+1 overlap the MMA and epilogue of tile k.  Every
// mbarrier wait is bounded; a group decides to stop with a barrier-OR over
// its threads, and the other group then times out on its next wait.
// PASS 0 counts, PASS 1 writes the proposals (FAST: the fast tier's 8-byte
// form); KIND 0: u8 operands, 1: BF16 with the exact recheck.
template <int PASS, int KIND, bool FAST>
__global__ void __launch_bounds__(TC_THREADS, 4) k_join_tc(JoinArgs a) {
    extern __shared__ __align__(1024) unsigned char smem[];
    __shared__ TcShared sh;
    const uint32_t tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t kq = a.kq, nchunk = kq >> 4, gbytes = nchunk * 128;
    const uint32_t mma_bar = smem_u32(&sh.mma_bar);

    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mma_bar));
        for (int b = 0; b < 2; b++) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 128;" ::"r"(smem_u32(&sh.full[b])));
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 128;" ::"r"(smem_u32(&sh.empty[b])));
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&sh.tmem)),
                     "r"(TC_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = sh.tmem;

    // pass 0 joins every row of tiers 0-3; pass 1 only the rows that pass 0
    // found to have proposals
    const uint32_t* rcount = PASS == 0 ? a.ctr->ntier : a.ctr->nemit;
    const uint32_t* rlist = PASS == 0 ? a.tier_rows : a.emit_rows;
    uint32_t nt[4];
    uint32_t total = 0;
#pragma unroll
    for (int t = 0; t < 4; t++) {
        nt[t] = (rcount[t] + (8u >> t) - 1) >> (3 - t);
        total += nt[t];
    }
    bool failed = false, mma_pending = false;
    uint32_t mma_phase = 0;

    if (warp >= 4) {
        // ---------------- producers ----------------
        const uint32_t ptid = tid - 128;
        unsigned long long sum_s = 0;
        for (uint32_t k = 0;; k++) {
            const uint32_t tile = blockIdx.x + k * gridDim.x;
            if (tile >= total) break;
            const uint32_t b = k & 1, use = k >> 1;
            if (use > 0) {
                const bool ok = mbar_wait_bounded(smem_u32(&sh.empty[b]), (use - 1) & 1);
                if (group_any(BAR_PROD, !ok)) {
                    failed = true;
                    break;
                }
            }
            uint32_t t = 0, lt = tile;
            while (t < 3 && lt >= nt[t]) {
                lt -= nt[t];
                t++;
            }
            const uint32_t lgB = 4 + t, B = 1u << lgB, RT = 8u >> t;
            const uint32_t first = lt * RT, nrows = min(RT, rcount[t] - first);
            TileHdr& H = sh.hdr[b];
            const SlotBuf S = slot_buf(smem, kq, b);
            if (ptid == 0) {
                H.t = t;
                H.lgB = lgB;
                H.nrows = nrows;
            }
            if (ptid < 8) H.any[ptid] = 0;
            if (ptid < nrows) {
                const uint32_t row = rlist[(size_t)t * a.n + first + ptid];
                const uint32_t nn = a.newlen[row], Sr = nn + a.oldlen[row];
                H.row[ptid] = row;
                H.nn[ptid] = nn;
                H.S[ptid] = Sr;
                sum_s += Sr;
            }
            group_sync(BAR_PROD);
            {  // slot metadata, ptid = slot
                const uint32_t r = ptid >> lgB, q = ptid & (B - 1);
                uint32_t e = NO_SLOT;
                if (r < nrows && q < H.S[r]) {
                    const uint32_t row = H.row[r], nn = H.nn[r];
                    e = q < nn ? a.newL[(size_t)row * a.capn + q] : a.oldL[(size_t)row * a.capo + q - nn];
                    const uint32_t id = e & LID_MASK;
                    S.kth[ptid] = a.pdist[(size_t)id * a.K + a.K - 1];
                    S.nrm[ptid] = a.nrm[id];
                    S.grp[ptid] = a.mode == MODE_SMERGE ? leaf_of(id, a.leaf_off, a.nleaf) : (e >> 31);
                    S.cnt[ptid] = 0;
                    if (PASS == 1) {
                        const uint32_t c = a.cntpos[(size_t)row * a.caps + q];
                        S.base[ptid] = c ? a.boff[id] + atomicAdd(&a.bcur[id], c) : 0ull;
                    }
                }
                S.ids[ptid] = e;
            }
            group_sync(BAR_PROD);
            // gather: 16-byte chunk c of slot s -> group s/8, core matrix c, row s%8
            const uint32_t vbase = smem_u32(S.vec);
            for (uint32_t i = ptid; i < TC_SLOTS * nchunk; i += 128) {
                const uint32_t r8 = i & 7, rest = i >> 3, c = rest % nchunk, g = rest / nchunk, sl = g * 8 + r8;
                const uint32_t e = S.ids[sl];
                if (e != NO_SLOT)
                    cp_async16(vbase + g * gbytes + c * 128 + r8 * 16, a.xq + (size_t)(e & LID_MASK) * kq + c * 16);
            }
            asm volatile("cp.async.wait_all;" ::: "memory");
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // cp.async writes -> tensor core reads
            mbar_arrive(smem_u32(&sh.full[b]));
        }
        if (PASS == 0) {
            for (int o = 16; o > 0; o >>= 1) sum_s += __shfl_xor_sync(0xffffffffu, sum_s, o);
            if (lane == 0 && sum_s) {
                atomicAdd(&a.ctr->sum_s, sum_s);
                atomicAdd(&a.ctr->sum_s_tc, sum_s);
            }
        }
    } else {
        // ---------------- consumers ----------------
        uint32_t cmps = 0;
        for (uint32_t k = 0;; k++) {
            const uint32_t tile = blockIdx.x + k * gridDim.x;
            if (tile >= total) break;
            const uint32_t b = k & 1, use = k >> 1;
            const bool okf = mbar_wait_bounded(smem_u32(&sh.full[b]), use & 1);
            if (group_any(BAR_CONS, !okf)) {
                failed = true;
                break;
            }
            const TileHdr& H = sh.hdr[b];
            const SlotBuf S = slot_buf(smem, kq, b);
            const uint32_t t = H.t, lgB = H.lgB, nrows = H.nrows, B = 1u << lgB;
            if (tid == 0) {
                asm volatile("tcgen05.fence::after_thread_sync;");
                const uint32_t vbase = smem_u32(S.vec);
                for (uint32_t kk = 0; kk < nchunk / 2; kk++) {  // 32 bytes of K per instruction
                    const uint64_t desc = smem_desc(vbase + kk * 256, 128, gbytes);
                    if (KIND == 0)
                        asm volatile(
                            "{\n\t.reg .pred p;\n\t"
                            "setp.ne.b32 p, %4, 0;\n\t"
                            "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(
                                tmem),
                            "l"(desc), "l"(desc), "r"(IDESC_U8), "r"(kk), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
                    else
                        asm volatile(
                            "{\n\t.reg .pred p;\n\t"
                            "setp.ne.b32 p, %4, 0;\n\t"
                            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(
                                tmem),
                            "l"(desc), "l"(desc), "r"(IDESC_BF16), "r"(kk), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
                }
                asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                                 mma_bar)
                             : "memory");
            }
            const bool okm = mbar_wait_bounded(mma_bar, mma_phase);
            if (group_any(BAR_CONS, !okm)) {
                failed = true;
                mma_pending = true;
                break;
            }
            mma_phase ^= 1u;
            asm volatile("tcgen05.fence::after_thread_sync;");

            // epilogue: this thread is slot b = tid (TMEM lane tid)
            const uint32_t e_b = S.ids[tid];
            const bool valid_b = e_b != NO_SLOT;
            const uint32_t r_b = tid >> lgB, q_b = tid & (B - 1);
            const uint32_t nn_b = valid_b ? H.nn[r_b] : 0u, S_b = valid_b ? H.S[r_b] : 0u;
            const uint32_t row_b = valid_b ? H.row[r_b] : 0u;
            const float kth_b = S.kth[tid];
            const uint32_t nrm_b = S.nrm[tid], grp_b = S.grp[tid];
            const uint32_t blk = tid & ~(B - 1);
            uint32_t cb = 0;
            // Rows of at most 32 slots lie inside one warp, so every proposal
            // to slot s of such a tile comes from the warp holding s: its
            // counter lives in a register of lane s % 32 (read by shuffle)
            // instead of shared memory (an atomic round trip per pair).
            const bool wl_tile = lgB <= 5;
            uint32_t cnt_r = 0;
            const uint32_t c_first = B >= 32 ? ((warp * 32) & ~(B - 1)) : warp * 32;
            // the loop specialised for the tile's counter kind, so that the
            // one running holds no code of the other (the emit pass is
            // bound by instruction fetch)
            auto pairs = [&](auto wl_kind) {
                constexpr bool wl = decltype(wl_kind)::value;
                for (uint32_t c0 = c_first; c0 <= warp * 32; c0 += 32) {
                    // columns a of a pair are new-list entries: a < blk + nn_b; the
                    // bound is made warp-uniform (lanes of different rows take the max)
                    const int lim = valid_b ? (int)(blk + nn_b) - (int)c0 : 0;
                    const uint32_t jend = (uint32_t)__reduce_max_sync(0xffffffffu, lim < 0 ? 0 : (lim > 32 ? 32 : lim));
                    if (jend == 0) continue;
                    // 8 columns per TMEM load: no spills at 64 registers, a short unrolled body
                    for (uint32_t h = 0; h < jend; h += 8) {
                        uint32_t v[8];
                        tmem_ld8(tmem + ((warp * 32) << 16) + c0 + h, v);
#pragma unroll
                        for (uint32_t j8 = 0; j8 < 8; j8++) {
                            const uint32_t jj = h + j8;
                            if (jj >= jend) break;
                            const uint32_t av = c0 + jj;
                            const uint32_t q_a = av & (B - 1);
                            const bool pv = valid_b && (av & ~(B - 1)) == blk && q_a < q_b && q_a < nn_b;
                            const uint32_t e_a = S.ids[av];
                            float dd;
                            if (KIND == 0) {
                                dd = (float)((int)(S.nrm[av] + nrm_b) - 2 * (int)v[j8]);
                            } else {
                                // approximate distance; pairs it cannot rule out get
                                // the reference's exact sum
                                const float ns = __uint_as_float(S.nrm[av]) + __uint_as_float(nrm_b);
                                dd = ns - 2.f * __uint_as_float(v[j8]);
                                if (pv && dd - a.err_c * ns < fmaxf(S.kth[av], kth_b))
                                    dd = exact_l2(a.x, a.dp, e_a & LID_MASK, e_b & LID_MASK);
                            }
                            uint32_t outer = 0, inner = 0;
                            const bool ok = pv && pair_order(a.mode, a.verse, q_a, q_b, nn_b, e_a, e_b, S.grp[av],
                                                             grp_b, outer, inner);
                            const float kth_a = S.kth[av];
                            if (PASS == 0) {
                                cmps += ok;
                                cb += (ok && dd < kth_b);
                                const unsigned m = __ballot_sync(0xffffffffu, ok && dd < kth_a);
                                if (wl) {
                                    if (lane == (av & 31)) cnt_r += __popc(m);
                                } else if (m && lane == 0) {
                                    atomicAdd(&S.cnt[av], (uint32_t)__popc(m));
                                }
                            } else {
                                const uint32_t pidx = outer * S_b + inner;
                                const bool pa = ok && dd < kth_a;
                                const unsigned m = __ballot_sync(0xffffffffu, pa);
                                if (m) {
                                    uint32_t base;
                                    if (wl) {
                                        // the owner of slot av is lane av % 32; its own
                                        // pair with av is not a pair (q_a == q_b), so it
                                        // takes no b-side proposal in this step
                                        base = __shfl_sync(0xffffffffu, cnt_r, av & 31);
                                        if (lane == (av & 31)) cnt_r += __popc(m);
                                    } else {
                                        const uint32_t leader = __ffs(m) - 1;
                                        base = 0;
                                        if (lane == leader) base = atomicAdd(&S.cnt[av], (uint32_t)__popc(m));
                                        base = __shfl_sync(0xffffffffu, base, leader);
                                    }
                                    if (pa) {
                                        const uint32_t before = __popc(m & ((1u << lane) - 1u));
                                        const unsigned long long slot = S.base[av] + base + before;
                                        put_prop<FAST>(a.bucket, slot, dd, e_b, row_b, pidx, outer == q_a ? 0u : 1u);
                                    }
                                }
                                if (ok && dd < kth_b) {
                                    const uint32_t pos = wl ? cnt_r++ : atomicAdd(&S.cnt[tid], 1u);
                                    const unsigned long long slot = S.base[tid] + pos;
                                    put_prop<FAST>(a.bucket, slot, dd, e_a, row_b, pidx, outer == q_b ? 0u : 1u);
                                }
                            }
                        }
                    }
                }
            };
            if (wl_tile) pairs(std::true_type{});
            else pairs(std::false_type{});
            if (PASS == 0) {
                if (wl_tile)
                    S.cnt[tid] = cnt_r + cb;
                else if (cb)
                    atomicAdd(&S.cnt[tid], cb);
            }
            asm volatile("tcgen05.fence::before_thread_sync;");
            group_sync(BAR_CONS);
            if (PASS == 0) {
                if (valid_b) {
                    const uint32_t c = S.cnt[tid];
                    a.cntpos[(size_t)row_b * a.caps + q_b] = (uint16_t)c;
                    if (c) {
                        atomicAdd(&a.bcnt[e_b & LID_MASK], c);
                        sh.hdr[b].any[r_b] = 1;
                    }
                }
                group_sync(BAR_CONS);
                if (warp == 0) {  // rows with proposals go to the emit pass's list
                    const bool has = lane < nrows && H.any[lane];
                    const unsigned m = __ballot_sync(0xffffffffu, has);
                    uint32_t base = 0;
                    if (m && lane == 0) base = atomicAdd(&a.ctr->nemit[t], (uint32_t)__popc(m));
                    base = __shfl_sync(0xffffffffu, base, 0);
                    if (has) a.emit_rows[(size_t)t * a.n + base + __popc(m & ((1u << lane) - 1u))] = H.row[lane];
                }
            }
            mbar_arrive(smem_u32(&sh.empty[b]));
        }
        if (PASS == 0) {
            for (int o = 16; o > 0; o >>= 1) cmps += __shfl_xor_sync(0xffffffffu, cmps, o);
            if (lane == 0 && cmps) atomicAdd(&a.ctr->ncmps, (unsigned long long)cmps);
        }
    }
    if (failed && (tid & 127) == 0) atomicOr(a.tc_err, (unsigned)DERR_TC_WAIT);
    if (mma_pending) mbar_wait_bounded(mma_bar, mma_phase);  // the MMA may still write TMEM
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TC_COLS));
    }
}

// Warp per vector: checks that every component is an integer in [0, 255],
// writes the u8 copy (zero padded to kq bytes) and the squared norm, and
// tracks the largest norm.
__global__ void k_quantize(const float* x, uint32_t n, uint32_t d, uint32_t dp, uint32_t kq, uint8_t* xq,
                           uint32_t* nrm, unsigned* bad, unsigned* maxnrm) {
    const uint32_t row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const uint32_t lane = threadIdx.x & 31;
    if (row >= n) return;
    const float* src = x + (size_t)row * dp;
    uint8_t* dst = xq + (size_t)row * kq;
    uint32_t s = 0;
    bool ok = true;
    for (uint32_t k = lane; k < kq; k += 32) {
        uint32_t u = 0;
        if (k < d) {
            const float v = src[k];
            if (v >= 0.f && v <= 255.f && v == truncf(v)) u = (uint32_t)v;
            else ok = false;
        }
        dst[k] = (uint8_t)u;
        s += u * u;
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    const bool all_ok = __all_sync(0xffffffffu, ok);
    if (lane == 0) {
        nrm[row] = s;
        if (!all_ok) atomicOr(bad, 1u);
        atomicMax(maxnrm, s);
    }
}

// Warp per vector: the BF16 copy (round to nearest even, zero padded to kq
// bytes) and the squared norm (double sum, rounded to float).  Flags rows
// the BF16 bound does not cover: non-finite components, or nonzero ones
// outside [2^-60, 2^50] (products must stay normal and sums finite).
__global__ void k_to_bf16(const float* x, uint32_t n, uint32_t d, uint32_t dp, uint32_t kq, __nv_bfloat16* xb,
                          uint32_t* nrm, unsigned* bad) {
    const uint32_t row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const uint32_t lane = threadIdx.x & 31;
    if (row >= n) return;
    const float* src = x + (size_t)row * dp;
    __nv_bfloat16* dst = xb + (size_t)row * (kq / 2);
    double s = 0.0;
    bool ok = true;
    for (uint32_t k = lane; k < kq / 2; k += 32) {
        float v = 0.f;
        if (k < d) {
            v = src[k];
            const float m = fabsf(v);
            if (!(m <= 0x1p50f) || (m != 0.f && m < 0x1p-60f)) ok = false;
        }
        dst[k] = __float2bfloat16_rn(v);
        s += (double)v * (double)v;
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    const bool all_ok = __all_sync(0xffffffffu, ok);
    if (lane == 0) {
        nrm[row] = __float_as_uint((float)s);
        if (!all_ok) atomicOr(bad, 1u);
    }
}

}  // namespace

int tc_prepare(Ctx& ctx, GraphStore& s, GraphDev& g) {
    g.xq = nullptr;
    g.nrm = nullptr;
    g.kq = 0;
    if (g.join_kernel == NNM_JOIN_FP32) return 0;
    const uint32_t kq = (g.d + 31) & ~31u;
    const char* why = nullptr;
    if (g.metric != L2) why = "the tensor-core join needs the L2 metric";
    else if (kq > TC_MAX_KQ) why = "the tensor-core join takes d <= 768";
    if (!why) {
        NNM_CUDA_TRY(s.xq.ensure((size_t)g.n_cap * kq));
        NNM_CUDA_TRY(s.nrm.ensure((size_t)g.n_cap * 4));
        DevBuf& m = ctx.ws.misc;
        NNM_CUDA_TRY(m.ensure(64));
        NNM_CUDA_TRY(cudaMemsetAsync(m.p, 0, 16, ctx.stream));
        unsigned* flags = m.as<unsigned>();
        k_quantize<<<(g.n_cap + 7) / 8, 256, 0, ctx.stream>>>(g.x, g.n_cap, g.d, g.dp, kq, s.xq.as<uint8_t>(),
                                                              s.nrm.as<uint32_t>(), flags, flags + 1); count_launch();
        unsigned h[2] = {0, 0};
        NNM_CUDA_TRY(cudaMemcpyAsync(h, flags, 8, cudaMemcpyDeviceToHost, ctx.stream));
        NNM_CUDA_TRY(cudaStreamSynchronize(ctx.stream));
        // every squared distance is at most |a|^2 + |b|^2 for non-negative vectors
        if (!h[0] && 2ull * h[1] < (1ull << 24)) {
            g.xq = s.xq.as<uint8_t>();
            g.nrm = s.nrm.as<uint32_t>();
            g.kq = kq;
            g.tc_kind = 0;
            return 0;
        }
        // other data: BF16 Gram matrices with the FP32 recheck, on request
        // only -- the rigorous BF16 bound (about 2^-8 of |a|^2 + |b|^2)
        // leaves most candidate pairs inside the recheck band, and the
        // per-pair exact sums then cost more than the FP32 join (measured
        // 3-4x slower per iteration on unit-norm 96-d data)
        const uint32_t kqb = 2 * ((g.d + 15) & ~15u);
        if (g.join_kernel != NNM_JOIN_TENSOR) {
            why = "auto: FP32 join for non-integer data";
        } else if (kqb > TC_MAX_KQ) {
            why = "the BF16 tensor-core join takes d <= 384";
        } else {
            NNM_CUDA_TRY(s.xq.ensure((size_t)g.n_cap * kqb));
            NNM_CUDA_TRY(cudaMemsetAsync(m.p, 0, 16, ctx.stream));
            k_to_bf16<<<(g.n_cap + 7) / 8, 256, 0, ctx.stream>>>(g.x, g.n_cap, g.d, g.dp, kqb,
                                                                 s.xq.as<__nv_bfloat16>(), s.nrm.as<uint32_t>(), flags); count_launch();
            NNM_CUDA_TRY(cudaMemcpyAsync(h, flags, 4, cudaMemcpyDeviceToHost, ctx.stream));
            NNM_CUDA_TRY(cudaStreamSynchronize(ctx.stream));
            if (h[0]) {
                why = "the BF16 tensor-core join needs finite components with magnitudes in [2^-60, 2^50]";
            } else {
                g.xq = s.xq.as<uint8_t>();
                g.nrm = s.nrm.as<uint32_t>();
                g.kq = kqb;
                g.tc_kind = 1;
                // |computed - reference| <= err_c (|a|^2 + |b|^2): BF16 inputs
                // (2 x 2^-9 relative per product), FP32 accumulation of d
                // terms (d 2^-22, truncating adds allowed), the float norms
                // and the final two operations (2^-21), and the reference's
                // own sequential sum ((d + 2) 2^-23 of a distance <= 2(|a|^2 +
                // |b|^2)); |a||b| <= (|a|^2 + |b|^2) / 2; a 1.25 safety factor
                const double dd = (double)g.d;
                g.err_c = (float)(1.25 * (std::ldexp(1.0, -8) + std::ldexp(1.0, -18) + (2 * dd + 4) * std::ldexp(1.0, -22) +
                                          std::ldexp(1.0, -21)));
                return 0;
            }
        }
    }
    if (why && g.join_kernel == NNM_JOIN_TENSOR) {
        ctx.last_error = why;
        return 1;  // NNM_ERR_INVALID
    }
    return 0;
}

cudaError_t tc_set_attributes(uint32_t kq, uint32_t kind) {
    const int bytes = (int)std::max<size_t>(tc_smem_bytes(kq), TC_SMEM_FLOOR);
    cudaError_t e;
    const void* fns[2][3] = {{(const void*)k_join_tc<0, 0, false>, (const void*)k_join_tc<1, 0, false>,
                              (const void*)k_join_tc<1, 0, true>},
                             {(const void*)k_join_tc<0, 1, false>, (const void*)k_join_tc<1, 1, false>,
                              (const void*)k_join_tc<1, 1, true>}};
    for (const void* f : fns[kind ? 1 : 0])
        if ((e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes)) != cudaSuccess) return e;
    return cudaSuccess;
}

cudaError_t launch_join_tc(int pass, const JoinArgs& ja, const unsigned* ntier, int nsm, cudaStream_t st) {
    unsigned tiles = 0;
    for (int t = 0; t < 4; t++) tiles += (ntier[t] + (8u >> t) - 1) >> (3 - t);
    if (!tiles) return cudaSuccess;
    const unsigned grid = std::min<unsigned>(tiles, (unsigned)nsm * 4);
    const size_t bytes = std::max<size_t>(tc_smem_bytes(ja.kq), TC_SMEM_FLOOR);
    const bool fast = ja.fast_key != 0;
    if (ja.tc_kind == 0) {
        if (pass == 0) k_join_tc<0, 0, false><<<grid, TC_THREADS, bytes, st>>>(ja);
        else if (fast) k_join_tc<1, 0, true><<<grid, TC_THREADS, bytes, st>>>(ja);
        else k_join_tc<1, 0, false><<<grid, TC_THREADS, bytes, st>>>(ja);
    } else {
        if (pass == 0) k_join_tc<0, 1, false><<<grid, TC_THREADS, bytes, st>>>(ja);
        else if (fast) k_join_tc<1, 1, true><<<grid, TC_THREADS, bytes, st>>>(ja);
        else k_join_tc<1, 1, false><<<grid, TC_THREADS, bytes, st>>>(ja);
    }
    count_launch();
    return cudaGetLastError();
}

}  // namespace nnm
