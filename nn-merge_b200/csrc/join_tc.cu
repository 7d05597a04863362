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
// Longer lists (the last tier) take k_pairs_tc below: a row's slots in
// several 128-slot blocks, one MMA chain per pair of blocks.
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
#include <cuda_fp16.h>
#include <cuda_fp8.h>

#include "../../include/nnm.h"
#include "nnm_engine.h"
#include "nnm_join.h"
#include "nnm_launch.h"
#include "nnm_tc.cuh"

namespace nnm {
namespace {

// Consumer threads per CTA: the emit pass runs two warps per TMEM lane
// quarter (warps 0-7), the count pass one (warps 0-3); the producers are
// the next four warps, one thread per tile slot.
constexpr int TC_PROD = 128;
__host__ __device__ constexpr int tc_cons(int pass) { return pass == 1 ? 256 : 128; }
__host__ __device__ constexpr int tc_threads(int pass) { return tc_cons(pass) + TC_PROD; }
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
// Instruction descriptor of kind::f8f6f4: D = F32 (bits 4-5 = 1), A = B =
// E4M3 (bits 7-9 = 0, 10-12 = 0), both K-major.
constexpr uint32_t IDESC_E4M3 = (1u << 4) | ((TC_SLOTS >> 3) << 17) | ((TC_SLOTS >> 4) << 24);

// Operand kinds of the join (JoinArgs::tc_kind):
//   KIND_U8    u8 vectors, kind::i8, exact integer Gram matrices;
//   KIND_BF16  each row as BF16 parts hi + lo (lo = the rounding residual),
//              G = hi.hi + hi.lo + lo.hi in three kind::f16 MMAs per K step;
//   KIND_FP8   each row scaled by a power of two to |x| <= 448 and written as
//              E4M3 parts hi + mid + lo (successive rounding residuals),
//              G = hh + hm + mh + hl + lh + mm in six kind::f8f6f4 MMAs per
//              K step, unscaled exactly by the two powers of two.
// The reduced-precision kinds give d~ with |d~ - d| <= err_c (|a|^2 + |b|^2)
// against the reference's FP32 distance d.
constexpr uint32_t KIND_U8 = 0, KIND_BF16 = 1, KIND_FP8 = 2;

// The reference's sequential FP32 distance of rows i and j (the audit of
// the reduced-precision bound), one non-inlined copy.
__device__ __noinline__ float audit_l2(const float* x, uint32_t dp, uint32_t i, uint32_t j) {
    return dist_seq<L2>(x + (size_t)i * dp, x + (size_t)j * dp, (int)dp);
}

// Tile header of one buffer, written by the producers, read by the consumers.
struct TileHdr {
    uint32_t t, lgB, nrows, done;  // done: no more tiles (the consumers stop)
    uint32_t next;                 // the tile the producers load after this one
    uint32_t row[8], nn[8], S[8], any[8];
};

struct TcShared {
    uint64_t mma_bar;           // MMA completion (tcgen05.commit)
    uint64_t full[2], empty[2];  // tile buffer b loaded / released
    uint32_t tmem;
    TileHdr hdr[2];
};

// Shared memory of one tile buffer: the slot vectors in the 128-byte swizzle
// K-major layout -- per 128-byte column of the operand row (kq rounded up
// to 128), 128 slot rows of 128 bytes (16 KB, 8-row atoms of 1024 bytes) --
// then the per-slot arrays.  Two buffers.
constexpr uint32_t TC_COL_BYTES = TC_SLOTS * 128;  // one 128-byte column of every slot
__host__ __device__ constexpr uint32_t tc_cols(uint32_t kq) { return (kq + 127) / 128; }
__host__ __device__ constexpr size_t tc_vec_bytes(uint32_t kq) { return (size_t)tc_cols(kq) * TC_COL_BYTES; }
__host__ __device__ constexpr size_t tc_buf_bytes(uint32_t kq) {
    return (tc_vec_bytes(kq) + (size_t)TC_SLOTS * (16 + 3 * 4 + 8) + 1023) & ~(size_t)1023;
}
__host__ __device__ constexpr size_t tc_smem_bytes(uint32_t kq) { return 2 * tc_buf_bytes(kq) + 1024; }

struct SlotBuf {
    unsigned char* vec;
    uint4* info;    // per slot: list entry, K-th distance (bits), norm, group -- one 16-byte read
    uint32_t* cnt;  // pass 0: counts; pass 1: bucket cursors
    uint32_t* lim;  // pass 1: the slot's reserved bucket range (its pass-0 count)
    float* scl;     // KIND_FP8: the row's inverse scale 2^-e
    unsigned long long* base;
};

__device__ __forceinline__ SlotBuf slot_buf(unsigned char* smem, uint32_t kq, uint32_t b) {
    unsigned char* p = smem + b * tc_buf_bytes(kq);
    SlotBuf s;
    s.vec = p;
    s.info = reinterpret_cast<uint4*>(p + tc_vec_bytes(kq));
    s.cnt = reinterpret_cast<uint32_t*>(s.info + TC_SLOTS);
    s.lim = s.cnt + TC_SLOTS;
    s.scl = reinterpret_cast<float*>(s.lim + TC_SLOTS);
    s.base = reinterpret_cast<unsigned long long*>(s.scl + TC_SLOTS);
    return s;
}

// Barriers of one thread group (producers: 1, consumers: 2).
constexpr uint32_t BAR_PROD = 1, BAR_CONS = 2;

__device__ __forceinline__ void group_sync(uint32_t id, uint32_t nthreads) {
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}

// Barrier of the group that also ORs a predicate over its 128 threads, so
// that a decision taken after per-thread bounded waits is the same in every
// thread of the group.
__device__ __forceinline__ bool group_any(uint32_t id, bool p, uint32_t nthreads) {
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\t"
        "setp.ne.u32 p, %1, 0;\n\t"
        "bar.red.or.pred q, %2, %3, p;\n\t"
        "selp.u32 %0, 1, 0, q;\n\t}\n"
        : "=r"(r)
        : "r"((uint32_t)p), "r"(id), "r"(nthreads)
        : "memory");
    return r != 0;
}

// Persistent CTAs in two groups over two tile buffers:
//   producers (the last four warps): for tile k, wait until buffer k%2 is released,
//     write its header and slot metadata, gather the slot vectors with
//     cp.async, then arrive on full[k%2];
//   consumers (warps 0-3; in the emit pass warps 0-7, warps w and w + 4
//     reading TMEM lanes 32 (w % 4) .. + 31 and sharing their columns in
//     8-column blocks): wait for full[k%2], run the MMA chain (thread 0) and
//     the epilogue, write the counts, then arrive on empty[k%2].
// The emit pass takes two warps per lane quarter because its epilogue is
// latency-bound (under one eligible warp per scheduler with one): 9 % off
// the pass, at three CTAs per SM instead of four (registers); the count
// pass, with less to do per pair, measured 6 % slower that way.
// So the loads of tile k+1 overlap the MMA and epilogue of tile k.  Every
// mbarrier wait is bounded; a group decides to stop with a barrier-OR over
// its threads, and the other group then times out on its next wait.
// PASS 0 counts, PASS 1 writes the proposals (FAST: the fast tier's 8-byte
// form); KIND: the operand kind (KIND_U8, KIND_BF16, KIND_FP8).
//
// Reduced-precision kinds: a pair side passes when its lower bound
// d~ - err_c (|a|^2 + |b|^2) is below the target's K-th distance -- every
// side the FP32 join passes, and a few more, which the merge drops after
// computing their exact distances.  The proposal carries d~ and APPROX_BIT.
// Both passes then run the same tiles (all joined rows, not only those with
// proposals), so every pair's d~ comes from the same MMA position and the
// two passes decide alike; pass 1 still writes no proposal beyond the range
// pass 0 reserved, and records DERR_TC_RANGE if a slot's count differs.
// AUDIT (pass 0 of the reduced-precision kinds): every pair's d~ is also
// checked against its exact distance.
template <int PASS, int KIND, bool FAST, bool AUDIT = false>
__global__ void __launch_bounds__(tc_threads(PASS), PASS == 0 ? 4 : KIND == KIND_U8 ? 3 : 2) k_join_tc(JoinArgs a) {
    extern __shared__ __align__(1024) unsigned char smem[];
    __shared__ TcShared sh;
    constexpr uint32_t CONS = tc_cons(PASS), HALVES = CONS / 128;
    if (a.ctr->overflow) return;  // a buffer sized ahead was too small: the host reruns
    const uint32_t tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t kq = a.kq, nchunk = kq >> 4;
    const uint32_t mma_bar = smem_u32(&sh.mma_bar);

    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mma_bar));
        for (int b = 0; b < 2; b++) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&sh.full[b])), "r"(TC_PROD));
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&sh.empty[b])), "r"(CONS));
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
    // found to have proposals (reduced-precision kinds: every row again)
    constexpr bool APPROX = KIND != KIND_U8;
    const uint32_t* rcount = (PASS == 0 || APPROX) ? a.ctr->ntier : a.ctr->nemit;
    const uint32_t* rlist = (PASS == 0 || APPROX) ? a.tier_rows : a.emit_rows;
    uint32_t nt[4];
    uint32_t total = 0;
#pragma unroll
    for (int t = 0; t < 4; t++) {
        nt[t] = (rcount[t] + (8u >> t) - 1) >> (3 - t);
        total += nt[t];
    }
    bool failed = false, mma_pending = false;
    uint32_t mma_phase = 0;

    if (warp >= CONS / 32) {
        // ---------------- producers ----------------
        // One thread per slot.  The slot's metadata (its row, list entry,
        // K-th distance, norm, group; pass 1: its bucket range) is a chain
        // of dependent reads; it is fetched into registers for tile k+1
        // while the vector copies of tile k are in flight, and stored into
        // the buffer once that buffer is released.
        const uint32_t ptid = tid - CONS;
        unsigned long long sum_s = 0;
        struct SlotMeta {
            uint32_t t, lgB, nrows, row, nn, S, e, nrm, grp, lim;
            float kth, scl;
            unsigned long long base;
        };
        auto fetch = [&](uint32_t tile, SlotMeta& m) {
            uint32_t t = 0, lt = tile;
            while (t < 3 && lt >= nt[t]) {
                lt -= nt[t];
                t++;
            }
            const uint32_t lgB = 4 + t, B = 1u << lgB, RT = 8u >> t;
            const uint32_t first = lt * RT;
            m.t = t;
            m.lgB = lgB;
            m.nrows = min(RT, rcount[t] - first);
            m.e = NO_SLOT;
            m.row = m.nn = m.S = 0;
            const uint32_t r = ptid >> lgB, q = ptid & (B - 1);
            if (r < m.nrows) {
                const uint32_t row = rlist[(size_t)t * a.n + first + r];
                const uint32_t nn = a.newlen[row], Sr = nn + a.oldlen[row];
                m.row = row;
                m.nn = nn;
                m.S = Sr;
                if (q < Sr) {
                    const uint32_t e =
                        q < nn ? a.newL[(size_t)row * a.capn + q] : a.oldL[(size_t)row * a.capo + q - nn];
                    const uint32_t id = e & LID_MASK;
                    m.e = e;
                    m.kth = a.kthv[id];
                    m.nrm = a.nrm[id];
                    m.scl = KIND == KIND_FP8 ? a.scl[id] : 1.f;
                    m.grp = a.mode == MODE_SMERGE ? leaf_of(id, a.leaf_off, a.nleaf) : (e >> 31);
                    if (PASS == 1) {
                        const uint32_t c = a.cntpos[(size_t)row * a.caps + q];
                        m.lim = c;
                        m.base = c ? a.boff[id] + atomicAdd(&a.bcur[id], c) : 0ull;
                    }
                }
            }
        };
        // Tiles: a CTA's first is its block index, every later one is
        // claimed from the launch's counter (tiles differ in cost; the CTAs
        // that finish early take more).  After the last tile the producers
        // hand the consumers a buffer marked done.
        SlotMeta cur{};
        uint32_t tile = blockIdx.x;
        if (tile < total) fetch(tile, cur);
        for (uint32_t k = 0;; k++) {
            const uint32_t b = k & 1, use = k >> 1;
            if (use > 0) {
                const bool ok = mbar_wait_bounded(smem_u32(&sh.empty[b]), (use - 1) & 1);
                if (group_any(BAR_PROD, !ok, TC_PROD)) {
                    failed = true;
                    break;
                }
            }
            TileHdr& H = sh.hdr[b];
            if (tile >= total) {
                if (ptid == 0) H.done = 1;
                mbar_arrive(smem_u32(&sh.full[b]));  // the arrive releases the header write
                break;
            }
            if (ptid == 0) {
                H.done = 0;
                H.next = gridDim.x + atomicAdd(&a.ctr->tc_next[PASS], 1u);
            }
            const SlotBuf S = slot_buf(smem, kq, b);
            const uint32_t B = 1u << cur.lgB, r = ptid >> cur.lgB, q = ptid & (B - 1);
            if (ptid == 0) {
                H.t = cur.t;
                H.lgB = cur.lgB;
                H.nrows = cur.nrows;
            }
            if (ptid < 8) H.any[ptid] = 0;
            if (q == 0 && r < cur.nrows) {
                H.row[r] = cur.row;
                H.nn[r] = cur.nn;
                H.S[r] = cur.S;
                sum_s += cur.S;
            }
            S.info[ptid] = cur.e != NO_SLOT ? make_uint4(cur.e, __float_as_uint(cur.kth), cur.nrm, cur.grp)
                                            : make_uint4(NO_SLOT, 0u, 0u, 0u);
            if (cur.e != NO_SLOT) {
                if (KIND == KIND_FP8) S.scl[ptid] = cur.scl;
                S.cnt[ptid] = 0;
                if (PASS == 1) {
                    S.lim[ptid] = cur.lim;
                    S.base[ptid] = cur.base;
                }
            }
            group_sync(BAR_PROD, TC_PROD);
            // gather: 16-byte chunk c of slot s -> column c / 8, row s, chunk
            // (c % 8) ^ (s % 8) (the 128-byte swizzle); a row's chunks by
            // consecutive threads
            const uint32_t vbase = smem_u32(S.vec);
            for (uint32_t i = ptid; i < TC_SLOTS * nchunk; i += 128) {
                const uint32_t sl = i / nchunk, c = i - sl * nchunk;
                const uint32_t e = S.info[sl].x;
                if (e != NO_SLOT)
                    cp_async16(vbase + (c >> 3) * TC_COL_BYTES + sl * 128 + (((c & 7) ^ (sl & 7)) << 4),
                               a.xq + (size_t)(e & LID_MASK) * kq + c * 16);
            }
            // the next tile's metadata while these copies land
            const uint32_t nxt = H.next;
            if (nxt < total) fetch(nxt, cur);
            asm volatile("cp.async.wait_all;" ::: "memory");
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // cp.async writes -> tensor core reads
            mbar_arrive(smem_u32(&sh.full[b]));
            tile = nxt;
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
            const uint32_t b = k & 1, use = k >> 1;
            const bool okf = mbar_wait_bounded(smem_u32(&sh.full[b]), use & 1);
            if (group_any(BAR_CONS, !okf, CONS)) {
                failed = true;
                break;
            }
            const TileHdr& H = sh.hdr[b];
            if (H.done) break;
            const SlotBuf S = slot_buf(smem, kq, b);
            const uint32_t t = H.t, lgB = H.lgB, nrows = H.nrows, B = 1u << lgB;
            if (tid == 0) {
                asm volatile("tcgen05.fence::after_thread_sync;");
                const uint32_t vbase = smem_u32(S.vec);
                // 32 bytes of K per instruction; the parts of a row lie one
                // after another along K (cpp chunks of 16 bytes each)
                const uint32_t nparts = KIND == KIND_U8 ? 1u : KIND == KIND_BF16 ? 2u : 3u;
                const uint32_t cpp = nchunk / nparts;
                auto desc_of = [&](uint32_t part, uint32_t kk) {
                    const uint32_t koff = (part * cpp + 2 * kk) * 16;  // bytes into the operand row
                    return smem_desc_sw128(vbase + (koff >> 7) * TC_COL_BYTES + (koff & 127));
                };
                for (uint32_t kk = 0; kk < cpp / 2; kk++) {
                    if (KIND == KIND_U8) {
                        const uint64_t desc = desc_of(0, kk);
                        asm volatile(
                            "{\n\t.reg .pred p;\n\t"
                            "setp.ne.b32 p, %4, 0;\n\t"
                            "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(
                                tmem),
                            "l"(desc), "l"(desc), "r"(IDESC_U8), "r"(kk), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
                    } else {
                        // (A part, B part) products: BF16 hi.hi, hi.lo, lo.hi;
                        // FP8 hh, hm, mh, hl, lh, mm
                        constexpr uint32_t NPROD = KIND == KIND_BF16 ? 3u : 6u;
                        constexpr uint32_t PA[6] = {0, 0, 1, 0, 2, 1}, PB[6] = {0, 1, 0, 2, 0, 1};
#pragma unroll
                        for (uint32_t pr = 0; pr < NPROD; pr++) {
                            const uint64_t da = desc_of(PA[pr], kk), db = desc_of(PB[pr], kk);
                            const uint32_t acc = (kk | pr) != 0;
                            if (KIND == KIND_BF16)
                                asm volatile(
                                    "{\n\t.reg .pred p;\n\t"
                                    "setp.ne.b32 p, %4, 0;\n\t"
                                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(
                                        tmem),
                                    "l"(da), "l"(db), "r"(IDESC_BF16), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
                            else
                                asm volatile(
                                    "{\n\t.reg .pred p;\n\t"
                                    "setp.ne.b32 p, %4, 0;\n\t"
                                    "tcgen05.mma.cta_group::1.kind::f8f6f4 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(
                                        tmem),
                                    "l"(da), "l"(db), "r"(IDESC_E4M3), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
                        }
                    }
                }
                asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                                 mma_bar)
                             : "memory");
            }
            const bool okm = mbar_wait_bounded(mma_bar, mma_phase);
            if (group_any(BAR_CONS, !okm, CONS)) {
                failed = true;
                mma_pending = true;
                break;
            }
            mma_phase ^= 1u;
            asm volatile("tcgen05.fence::after_thread_sync;");

            // epilogue: this thread is slot b = tid % 128 (TMEM lane b); warps
            // w and w + 4 (half 0 and 1) read the same lanes and take
            // alternate 8-column blocks
            const uint32_t slot = tid & (TC_SLOTS - 1), quarter = warp & 3, half = warp >> 2;
            const uint4 info_b = S.info[slot];
            const uint32_t e_b = info_b.x;
            const bool valid_b = e_b != NO_SLOT;
            const uint32_t r_b = slot >> lgB, q_b = slot & (B - 1);
            const uint32_t nn_b = valid_b ? H.nn[r_b] : 0u, S_b = valid_b ? H.S[r_b] : 0u;
            const uint32_t row_b = valid_b ? H.row[r_b] : 0u;
            const float kth_b = __uint_as_float(info_b.y);
            const uint32_t nrm_b = info_b.z, grp_b = info_b.w;
            const float scl_b = KIND == KIND_FP8 ? S.scl[slot] : 1.f;
            const uint32_t lim_b = PASS == 1 ? S.lim[slot] : 0u;
            // this slot's bucket range start, read once (the proposal stores
            // are generic and would make the compiler reload it)
            const unsigned long long base_b = PASS == 1 ? S.base[slot] : 0ull;
            bool over = false;  // pass 1, reduced precision: a write beyond a reserved range
            const uint32_t blk = slot & ~(B - 1);
            uint32_t cb = 0;
            // Rows of at most 32 slots lie inside one lane quarter, so every
            // proposal to slot s of such a tile comes from the two warps
            // holding s: each keeps its counter in a register of lane s % 32
            // (read by shuffle) instead of shared memory (an atomic round trip
            // per pair).  In the emit pass half 0 fills the slot's reserved
            // range from its start, half 1 from its end.
            const bool wl_tile = lgB <= 5;
            uint32_t cnt_r = 0;
            const uint32_t c_first = B >= 32 ? ((quarter * 32) & ~(B - 1)) : quarter * 32;
            // the loop specialised for the tile's counter kind, so that the
            // one running holds no code of the other (the emit pass is
            // bound by instruction fetch)
            auto pairs = [&](auto wl_kind) {
                constexpr bool wl = decltype(wl_kind)::value;
                uint32_t blocks = 0;  // 8-column blocks of this lane quarter so far
                for (uint32_t c0 = c_first; c0 <= quarter * 32; c0 += 32) {
                    // columns a of a pair are new-list entries: a < blk + nn_b; the
                    // bound is made warp-uniform (lanes of different rows take the max)
                    const int lim = valid_b ? (int)(blk + nn_b) - (int)c0 : 0;
                    const uint32_t jend = (uint32_t)__reduce_max_sync(0xffffffffu, lim < 0 ? 0 : (lim > 32 ? 32 : lim));
                    if (jend == 0) continue;
                    // 8 columns per TMEM load: no spills at 64 registers, a short unrolled body
                    for (uint32_t h = 0; h < jend; h += 8) {
                        // blocks 0, 3, 4, 7, ... to half 0 and 1, 2, 5, 6, ... to
                        // half 1: early columns hold more pairs (a < b)
                        const uint32_t bi = blocks++;
                        if (HALVES == 2 && ((bi + (bi >> 1)) & 1u) != half) continue;
                        uint32_t v[8];
                        tmem_ld8(tmem + ((quarter * 32) << 16) + c0 + h, v);
#pragma unroll
                        for (uint32_t j8 = 0; j8 < 8; j8++) {
                            const uint32_t jj = h + j8;
                            if (jj >= jend) break;
                            const uint32_t av = c0 + jj;
                            const uint32_t q_a = av & (B - 1);
                            const bool pv = valid_b && (av & ~(B - 1)) == blk && q_a < q_b && q_a < nn_b;
                            const uint4 info_a = S.info[av];
                            const uint32_t e_a = info_a.x;
                            float dd, lb;
                            if (KIND == KIND_U8) {
                                dd = (float)((int)(info_a.z + nrm_b) - 2 * (int)v[j8]);
                                lb = dd;
                            } else {
                                // d~ and its lower bound (distances are >= 0)
                                const float ns = __uint_as_float(info_a.z) + __uint_as_float(nrm_b);
                                float gd = __uint_as_float(v[j8]);
                                if (KIND == KIND_FP8) gd *= S.scl[av] * scl_b;
                                dd = fmaxf(ns - 2.f * gd, 0.f);
                                lb = dd - a.err_c * ns;
                                if (PASS == 0 && AUDIT && pv) {  // the bound against the exact distance
                                    const float ex = audit_l2(a.x, a.dp, e_a & LID_MASK, e_b & LID_MASK);
                                    if (!(ex >= lb && ex <= dd + a.err_c * ns)) atomicOr(a.tc_err, (unsigned)DERR_BOUND);
                                    if (ns > 0.f) atomicMax(&a.ctr->audit_max, __float_as_uint(fabsf(ex - dd) / ns));
                                }
                            }
                            const uint32_t axb = APPROX ? APPROX_BIT : 0u;
                            uint32_t outer = 0, inner = 0;
                            const bool ok = pv && pair_order(a.mode, a.verse, q_a, q_b, nn_b, e_a, e_b, info_a.w,
                                                             grp_b, outer, inner);
                            const float kth_a = __uint_as_float(info_a.y);
                            if (PASS == 0) {
                                cmps += ok;
                                cb += (ok && lb < kth_b);
                                const unsigned m = __ballot_sync(0xffffffffu, ok && lb < kth_a);
                                if (wl) {
                                    if (lane == (av & 31)) cnt_r += __popc(m);
                                } else if (m && lane == 0) {
                                    atomicAdd(&S.cnt[av], (uint32_t)__popc(m));
                                }
                            } else {
                                const uint32_t pidx = outer * S_b + inner;
                                const bool pa = ok && lb < kth_a;
                                const unsigned m = __ballot_sync(0xffffffffu, pa);
                                if (m) {
                                    uint32_t base;
                                    if (wl) {
                                        // the owner of slot av is lane av % 32; its own
                                        // pair with av is not a pair (q_a == q_b), so it
                                        // takes no b-side proposal in this step
                                        base = __shfl_sync(0xffffffffu, cnt_r, av & 31);
                                        if (lane == (av & 31)) cnt_r += __popc(m);
                                        if (half) base = S.lim[av] - base - __popc(m);  // from the range's end
                                    } else {
                                        const uint32_t leader = __ffs(m) - 1;
                                        base = 0;
                                        if (lane == leader) base = atomicAdd(&S.cnt[av], (uint32_t)__popc(m));
                                        base = __shfl_sync(0xffffffffu, base, leader);
                                    }
                                    if (pa) {
                                        const uint32_t before = __popc(m & ((1u << lane) - 1u));
                                        const unsigned long long at = S.base[av] + base + before;
                                        if (!APPROX || base + before < S.lim[av])
                                            put_prop<FAST>(a.bucket, at, dd, e_b | axb, row_b, pidx,
                                                           outer == q_a ? 0u : 1u);
                                        else
                                            over = true;
                                    }
                                }
                                if (ok && lb < kth_b) {
                                    const uint32_t pos =
                                        wl ? (half ? lim_b - 1u - cnt_r++ : cnt_r++) : atomicAdd(&S.cnt[slot], 1u);
                                    const unsigned long long at = base_b + pos;
                                    if (!APPROX || pos < lim_b)
                                        put_prop<FAST>(a.bucket, at, dd, e_a | axb, row_b, pidx, outer == q_b ? 0u : 1u);
                                    else
                                        over = true;
                                }
                            }
                        }
                    }
                }
            };
            if (wl_tile) pairs(std::true_type{});
            else pairs(std::false_type{});
            if (PASS == 0) {
                if (wl_tile ? (cnt_r + cb) != 0 : cb != 0) atomicAdd(&S.cnt[slot], wl_tile ? cnt_r + cb : cb);
            }
            if (PASS == 1 && APPROX && wl_tile && cnt_r) atomicAdd(&S.cnt[slot], cnt_r);
            if (PASS == 1 && APPROX && over) atomicOr(a.tc_err, (unsigned)DERR_TC_RANGE);
            asm volatile("tcgen05.fence::before_thread_sync;");
            group_sync(BAR_CONS, CONS);
            if (PASS == 1 && APPROX && half == 0) {  // every reserved range filled exactly
                if (valid_b && S.cnt[slot] != lim_b) atomicOr(a.tc_err, (unsigned)DERR_TC_RANGE);
            }
            if (PASS == 0) {
                if (half == 0 && valid_b) {
                    const uint32_t c = S.cnt[slot];
                    a.cntpos[(size_t)row_b * a.caps + q_b] = (uint16_t)c;
                    if (c) {
                        atomicAdd(&a.bcnt[e_b & LID_MASK], c);
                        sh.hdr[b].any[r_b] = 1;
                    }
                }
                group_sync(BAR_CONS, CONS);
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

// Rows of the last tier (S > the tile's list cap) of the u8 join, count
// pass, on the tensor cores.  A row's S slots lie in blocks of 128 (the
// 128-byte swizzle K-major layout of a tile buffer, one block after
// another); per block pair (p, q), p <= q, one kind::i8 MMA chain
// D = X_q X_p^T (M = N = 128) into the CTA's 128 TMEM columns: TMEM lane m
// is slot b = 128 q + m, column c is slot a = 128 p + c.  Consumer lane m
// takes the pairs (a, b), a < b, a in the new list, column by column, so a
// warp's 32 lanes hold 32 consecutive b of one a: each stored pair distance
// (the slots of `pair_slot`, read by k_emit_rows) is one coalesced 128-byte
// write, b's count a register, a's a ballot.  The outputs are k_pairs_u8's:
// the distances (exact integers), the per-slot counts and the bucket
// totals.  Recomputing the MMA in the emit pass instead of storing the
// distances was measured slower (the emit epilogue costs more than reading
// 4 bytes a pair back).
//
// Persistent CTAs of 320 threads over two row buffers, as the tiled join:
// producers (warps 8-9) load a row's members and gather its vectors with
// cp.async into buffer k % 2 while the consumers (warps 0-7, two per TMEM
// lane quarter, alternate 8-column blocks) run the MMAs and the epilogue of
// the other; full / empty mbarriers per buffer, every wait bounded, a
// group's stop decided by a barrier-OR over its threads; a CTA that stops
// records DERR_TC_WAIT, waits (bounded) once more for its MMA, frees its
// TMEM and returns.
constexpr int PT_CONS = 256, PT_PROD = 64, PT_THREADS = PT_CONS + PT_PROD;
__host__ __device__ constexpr uint32_t pt_blocks(uint32_t R) { return (R + TC_SLOTS - 1) / TC_SLOTS; }
// Rows of the last block: R's remainder rounded up to an 8-row swizzle atom.
// Its columns are that many rows apart; an MMA reads 128 rows from a column
// start all the same, the rows past the block's from whatever follows (slots
// >= R, never read back).
__host__ __device__ constexpr uint32_t pt_rows_last(uint32_t R) {
    return ((R - TC_SLOTS * (pt_blocks(R) - 1)) + 7) & ~7u;
}
__host__ __device__ constexpr uint32_t pt_col_stride(uint32_t R, uint32_t blk) {
    return (blk + 1 < pt_blocks(R) ? TC_SLOTS : pt_rows_last(R)) * 128;
}
__host__ __device__ constexpr size_t pt_vec_bytes(uint32_t R, uint32_t kq) {
    return (size_t)((pt_blocks(R) - 1) * TC_SLOTS + pt_rows_last(R)) * 128 * tc_cols(kq);
}
// the members of one row buffer: per slot the 16-byte record {entry, K-th
// distance bits, norm, group} and the count (4 B)
__host__ __device__ constexpr size_t pt_mem_bytes(uint32_t R) { return ((size_t)R * 20 + 15) & ~(size_t)15; }
// both buffers' vector blocks (1024-byte aligned), then both buffers'
// members, and at least the 128 rows an MMA reads from the last column start
__host__ __device__ constexpr size_t pt_smem_bytes(uint32_t R, uint32_t kq) {
    return 2 * pt_vec_bytes(R, kq) + (2 * pt_mem_bytes(R) > (size_t)(TC_SLOTS - pt_rows_last(R)) * 128
                                          ? 2 * pt_mem_bytes(R)
                                          : (size_t)(TC_SLOTS - pt_rows_last(R)) * 128);
}

struct PtHdr {
    uint32_t row, nn, S, done;
    unsigned long long poff;  // the row's stored pair distances
};

__global__ void __launch_bounds__(PT_THREADS, 3) k_pairs_tc(JoinArgs a, uint32_t R) {
    extern __shared__ __align__(1024) unsigned char smem[];
    __shared__ uint64_t mma_bar_s, full_s[2], empty_s[2];
    __shared__ uint32_t tmem_s;
    __shared__ PtHdr hdr[2];
    if (a.ctr->overflow) return;  // a buffer sized ahead was too small: the host reruns
    const uint32_t tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t kq = a.kq, nchunk = kq >> 4, ncol = tc_cols(kq);
    const size_t vbytes = pt_vec_bytes(R, kq), mbytes = pt_mem_bytes(R);
    const uint32_t mma_bar = smem_u32(&mma_bar_s);
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mma_bar));
        for (int b = 0; b < 2; b++) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&full_s[b])), "r"(PT_PROD));
            asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&empty_s[b])), "r"(PT_CONS));
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_s)),
                     "r"(TC_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = tmem_s;
    const uint32_t cnt = a.ctr->ntier[NTIER - 1];
    const uint32_t* rows = a.tier_rows + (size_t)(NTIER - 1) * a.n;
    bool failed = false, mma_pending = false;
    uint32_t mma_phase = 0;

    if (warp >= PT_CONS / 32) {
        // ---------------- producers ----------------
        const uint32_t ptid = tid - PT_CONS;
        uint32_t bi = blockIdx.x;
        uint32_t pf_bi = ~0u, pf_row = 0, pf_nn = 0, pf_S = 0;  // a row header fetched ahead
        unsigned long long sum_s = 0;
        for (uint32_t k = 0;; k++) {
            const uint32_t b = k & 1, use = k >> 1;
            if (use > 0) {
                const bool ok = mbar_wait_bounded(smem_u32(&empty_s[b]), (use - 1) & 1);
                if (group_any(BAR_PROD, !ok, PT_PROD)) {
                    failed = true;
                    break;
                }
            }
            unsigned char* buf = smem + b * vbytes;
            uint4* info = reinterpret_cast<uint4*>(smem + 2 * vbytes + b * mbytes);
            uint32_t* cur = reinterpret_cast<uint32_t*>(info + R);
            // the next row with new entries; its header may have been
            // fetched while the last row's vectors landed
            uint32_t row = 0, nn = 0, S = 0;
            for (; bi < cnt; bi += gridDim.x) {
                if (pf_bi == bi) {
                    row = pf_row;
                    nn = pf_nn;
                    S = pf_S;
                } else {
                    row = rows[bi];
                    nn = a.newlen[row];
                    S = nn + a.oldlen[row];
                }
                if (nn) break;
                for (uint32_t q = ptid; q < S; q += PT_PROD) a.cntpos[(size_t)row * a.caps + q] = 0;  // no pairs
            }
            PtHdr& H = hdr[b];
            if (bi >= cnt) {
                if (ptid == 0) H.done = 1;
                mbar_arrive(smem_u32(&full_s[b]));  // the arrive releases the header write
                break;
            }
            // the members, four slots a thread at a time: each step's loads
            // (entries; then K-th distances and norms; then groups) issued
            // together
            for (uint32_t q0 = ptid; q0 < S; q0 += 4 * PT_PROD) {
                uint32_t e[4], nr[4];
                float kt[4];
#pragma unroll
                for (int i = 0; i < 4; i++) {
                    const uint32_t q = q0 + i * PT_PROD;
                    e[i] = q < nn ? a.newL[(size_t)row * a.capn + q]
                                  : (q < S ? a.oldL[(size_t)row * a.capo + q - nn] : 0u);
                }
#pragma unroll
                for (int i = 0; i < 4; i++) {
                    const uint32_t q = q0 + i * PT_PROD, id = e[i] & LID_MASK;
                    kt[i] = q < S ? a.kthv[id] : 0.f;
                    nr[i] = q < S ? a.nrm[id] : 0u;
                }
#pragma unroll
                for (int i = 0; i < 4; i++) {
                    const uint32_t q = q0 + i * PT_PROD, id = e[i] & LID_MASK;
                    if (q < S) {
                        info[q] = make_uint4(e[i], __float_as_uint(kt[i]), nr[i],
                                             a.mode == MODE_SMERGE ? leaf_of(id, a.leaf_off, a.nleaf) : (e[i] >> 31));
                        cur[q] = 0;
                    }
                }
            }
            sum_s += S;
            if (ptid == 0) {
                H.row = row;
                H.nn = nn;
                H.S = S;
                H.done = 0;
                H.poff = a.poff[row];
            }
            group_sync(BAR_PROD, PT_PROD);  // the members, before the gather reads them
            bi += gridDim.x;
            // gather: chunk c of slot s -> block s / 128, column c / 8, row
            // s % 128, chunk (c % 8) ^ (s % 8)
            const uint32_t vbase = smem_u32(buf);
            for (uint32_t i = ptid; i < S * nchunk; i += PT_PROD) {
                const uint32_t sl = i / nchunk, c = i - sl * nchunk, ls = sl & (TC_SLOTS - 1);
                const uint32_t blk = sl >> 7;
                cp_async16(vbase + blk * ncol * TC_COL_BYTES + (c >> 3) * pt_col_stride(R, blk) + ls * 128 +
                               (((c & 7) ^ (ls & 7)) << 4),
                           a.xq + (size_t)(info[sl].x & LID_MASK) * kq + c * 16);
            }
            if (bi < cnt) {  // the next row's header while these copies land
                pf_bi = bi;
                pf_row = rows[bi];
                pf_nn = a.newlen[pf_row];
                pf_S = pf_nn + a.oldlen[pf_row];
            }
            asm volatile("cp.async.wait_all;" ::: "memory");
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // cp.async writes -> tensor core reads
            mbar_arrive(smem_u32(&full_s[b]));
        }
        if (ptid == 0 && sum_s) atomicAdd(&a.ctr->sum_s, sum_s);  // every producer holds the total
    } else {
        // ---------------- consumers ----------------
        uint32_t cmps = 0;
        const uint32_t quarter = warp & 3, half = warp >> 2;
        const uint32_t tlane = tmem + ((quarter * 32) << 16);
        for (uint32_t k = 0;; k++) {
            const uint32_t b = k & 1, use = k >> 1;
            const bool okf = mbar_wait_bounded(smem_u32(&full_s[b]), use & 1);
            if (group_any(BAR_CONS, !okf, PT_CONS)) {
                failed = true;
                break;
            }
            const PtHdr& H = hdr[b];
            if (H.done) break;
            const uint32_t row = H.row, nn = H.nn, S = H.S, no = S - nn;
            float* pd = a.pd + H.poff;
            const uint4* info = reinterpret_cast<const uint4*>(smem + 2 * vbytes + b * mbytes);
            uint32_t* cur = const_cast<uint32_t*>(reinterpret_cast<const uint32_t*>(info + R));
            const uint32_t vbase = smem_u32(smem + b * vbytes);
            for (uint32_t p = 0; p * TC_SLOTS < nn && !failed; p++) {
                for (uint32_t q = p; q * TC_SLOTS < S; q++) {
                    if (tid == 0) {
                        asm volatile("tcgen05.fence::after_thread_sync;");
                        const uint32_t ab = vbase + q * ncol * TC_COL_BYTES, bb = vbase + p * ncol * TC_COL_BYTES;
                        const uint32_t as = pt_col_stride(R, q), bs = pt_col_stride(R, p);
                        for (uint32_t kk = 0; kk < kq / 32; kk++) {
                            const uint32_t koff = kk * 32;  // bytes into the operand row
                            const uint64_t da = smem_desc_sw128(ab + (koff >> 7) * as + (koff & 127));
                            const uint64_t db = smem_desc_sw128(bb + (koff >> 7) * bs + (koff & 127));
                            asm volatile(
                                "{\n\t.reg .pred p;\n\t"
                                "setp.ne.b32 p, %4, 0;\n\t"
                                "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(
                                    tmem),
                                "l"(da), "l"(db), "r"(IDESC_U8), "r"(kk), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
                        }
                        asm volatile(
                            "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                                mma_bar)
                            : "memory");
                    }
                    const bool okm = mbar_wait_bounded(mma_bar, mma_phase);
                    if (group_any(BAR_CONS, !okm, PT_CONS)) {
                        failed = true;
                        mma_pending = true;
                        break;
                    }
                    mma_phase ^= 1u;
                    asm volatile("tcgen05.fence::after_thread_sync;");
                    // this lane: slot b = 128 q + 32 quarter + lane; columns a = 128 p + c
                    // with a < nn and (diagonal block) a < the quarter's last b
                    const uint32_t bv = q * TC_SLOTS + quarter * 32 + lane;
                    if (q * TC_SLOTS + quarter * 32 < S) {
                        const bool in_b = bv < S;
                        const uint4 ib = info[in_b ? bv : 0];
                        const uint32_t eb = ib.x, gb = ib.w, nb = ib.z;
                        const float kth_b = __uint_as_float(ib.y);
                        uint32_t cnt_b = 0;
                        const uint32_t a0 = p * TC_SLOTS;
                        uint32_t ncols = min(TC_SLOTS, nn - a0);
                        if (p == q) ncols = min(ncols, quarter * 32 + 32);
                        // 8-column blocks 0, 3, 4, 7, ... to half 0, 1, 2, 5, 6, ... to
                        // half 1 (early columns of a diagonal block hold more pairs)
                        for (uint32_t c0 = 0; c0 < ncols; c0 += 8) {
                            const uint32_t bk = c0 >> 3;
                            if (((bk + (bk >> 1)) & 1u) != half) continue;
                            uint32_t v[8];
                            tmem_ld8(tlane + c0, v);
                            const uint32_t jn = min(8u, ncols - c0);
#pragma unroll
                            for (uint32_t j = 0; j < 8; j++) {
                                if (j < jn) {
                                    const uint32_t av = a0 + c0 + j;
                                    const uint4 ia = info[av];
                                    const float dd = (float)((int)(ia.z + nb) - 2 * (int)v[j]);
                                    if (in_b && bv > av)  // lanes: consecutive b of one a
                                        pd[(bv < nn ? av * nn - av * (av + 1) / 2 - av - 1
                                                    : nn * (nn - 1) / 2 + av * no - nn) + bv] = dd;
                                    uint32_t outer, inner;
                                    const bool pr = in_b && bv > av &&
                                                    pair_order(a.mode, a.verse, av, bv, nn, ia.x, eb, ia.w, gb, outer, inner);
                                    cmps += pr;
                                    cnt_b += pr && dd < kth_b;
                                    const unsigned bal = __ballot_sync(0xffffffffu, pr && dd < __uint_as_float(ia.y));
                                    if (lane == 0 && bal) atomicAdd(&cur[av], (uint32_t)__popc(bal));
                                }
                            }
                        }
                        if (cnt_b) atomicAdd(&cur[bv], cnt_b);
                    }
                    asm volatile("tcgen05.fence::before_thread_sync;");
                    group_sync(BAR_CONS, PT_CONS);  // TMEM read and counts done before the next MMA
                }
            }
            if (failed) break;
            for (uint32_t q = tid; q < S; q += PT_CONS) {
                const uint32_t c = cur[q];
                a.cntpos[(size_t)row * a.caps + q] = (uint16_t)c;
                if (c) atomicAdd(&a.bcnt[info[q].x & LID_MASK], c);
            }
            mbar_arrive(smem_u32(&empty_s[b]));
        }
        for (int o = 16; o > 0; o >>= 1) cmps += __shfl_xor_sync(0xffffffffu, cmps, o);
        if (lane == 0 && cmps) atomicAdd(&a.ctr->ncmps, (unsigned long long)cmps);
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
// tracks the largest norm.  Four components per lane and step (rows are
// dp floats, dp a multiple of 4; kq a multiple of 32).  Warps stride over
// the rows; the largest norm and the check go to global memory once per
// block (an atomic per row on one word serialised the kernel).
__global__ void __launch_bounds__(256) k_quantize(const float* x, uint32_t n, uint32_t d, uint32_t dp, uint32_t kq,
                                                  uint8_t* xq, uint32_t* nrm, unsigned* bad, unsigned* maxnrm) {
    __shared__ unsigned bmax, bbad;
    const uint32_t lane = threadIdx.x & 31, wpb = blockDim.x >> 5;
    if (threadIdx.x == 0) bmax = bbad = 0;
    __syncthreads();
    unsigned wmax = 0;
    bool wok = true;
    for (uint32_t row = blockIdx.x * wpb + (threadIdx.x >> 5); row < n; row += gridDim.x * wpb) {
        const float* src = x + (size_t)row * dp;
        uint8_t* dst = xq + (size_t)row * kq;
        uint32_t s = 0;
        bool ok = true;
        for (uint32_t k = lane * 4; k < kq; k += 128) {
            float v[4] = {0.f, 0.f, 0.f, 0.f};
            if (k < dp) {
                const float4 f = *reinterpret_cast<const float4*>(src + k);
                v[0] = f.x;
                v[1] = f.y;
                v[2] = f.z;
                v[3] = f.w;
            }
            uint32_t packed = 0;
#pragma unroll
            for (uint32_t j = 0; j < 4; j++) {
                uint32_t u = 0;
                if (k + j < d) {
                    if (v[j] >= 0.f && v[j] <= 255.f && v[j] == truncf(v[j])) u = (uint32_t)v[j];
                    else ok = false;
                }
                packed |= u << (8 * j);
                s += u * u;
            }
            *reinterpret_cast<uint32_t*>(dst + k) = packed;
        }
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        wok = wok && __all_sync(0xffffffffu, ok);
        if (lane == 0) nrm[row] = s;
        wmax = max(wmax, s);
    }
    if (lane == 0) {
        atomicMax(&bmax, wmax);
        if (!wok) bbad = 1;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        if (bbad) atomicOr(bad, 1u);
        if (bmax) atomicMax(maxnrm, bmax);
    }
}

// Warp per vector: the BF16 parts hi = bf16(x) and lo = bf16(x - hi)
// (round to nearest even), stored one after the other along K (each part
// dpad = d rounded up to 16 elements, zero padded), and the squared norm
// (double sum, rounded to float).  Flags rows the bound does not cover:
// non-finite components, or nonzero ones outside [2^-60, 2^50] (products of
// parts must stay normal and sums finite).
__global__ void k_to_bf16x2(const float* x, uint32_t n, uint32_t d, uint32_t dp, uint32_t dpad, __nv_bfloat16* xb,
                            uint32_t* nrm, unsigned* bad) {
    const uint32_t row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const uint32_t lane = threadIdx.x & 31;
    if (row >= n) return;
    const float* src = x + (size_t)row * dp;
    __nv_bfloat16* dst = xb + (size_t)row * 2 * dpad;
    double s = 0.0;
    bool ok = true;
    for (uint32_t k = lane; k < dpad; k += 32) {
        float v = 0.f;
        if (k < d) {
            v = src[k];
            const float m = fabsf(v);
            if (!(m <= 0x1p50f) || (m != 0.f && m < 0x1p-60f)) ok = false;
        }
        const __nv_bfloat16 hi = __float2bfloat16_rn(v);
        dst[k] = hi;
        dst[dpad + k] = __float2bfloat16_rn(v - __bfloat162float(hi));
        s += (double)v * (double)v;
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    const bool all_ok = __all_sync(0xffffffffu, ok);
    if (lane == 0) {
        nrm[row] = __float_as_uint((float)s);
        if (!all_ok) atomicOr(bad, 1u);
    }
}

__device__ __forceinline__ float e4m3_value(__nv_fp8_storage_t q) {
    return __half2float(__half(__nv_cvt_fp8_to_halfraw(q, __NV_E4M3)));
}

// Warp per vector: the FP8 (E4M3) parts.  The row is scaled by 2^e, the
// power of two that brings its largest magnitude into (224, 448] (448 is
// E4M3's largest finite value; scaling by a power of two is exact), then
// hi = e4m3(x 2^e), mid = e4m3(x 2^e - hi), lo = e4m3(x 2^e - hi - mid),
// round to nearest even, the residuals exact in FP32.  Parts one after the
// other along K (each dpad = d rounded up to 32 bytes, zero padded); scl =
// 2^-e; squared norm as for BF16.  Flags rows with non-finite components or
// a nonzero largest magnitude outside [2^-60, 2^50].
__global__ void k_to_fp8x3(const float* x, uint32_t n, uint32_t d, uint32_t dp, uint32_t dpad, uint8_t* xq,
                           uint32_t* nrm, float* scl, unsigned* bad) {
    const uint32_t row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const uint32_t lane = threadIdx.x & 31;
    if (row >= n) return;
    const float* src = x + (size_t)row * dp;
    uint8_t* dst = xq + (size_t)row * 3 * dpad;
    float mx = 0.f;
    bool ok = true;
    double s = 0.0;
    for (uint32_t k = lane; k < d; k += 32) {
        const float v = src[k];
        if (!(fabsf(v) <= 0x1p50f)) ok = false;
        mx = fmaxf(mx, fabsf(v));
        s += (double)v * (double)v;
    }
    for (int o = 16; o > 0; o >>= 1) {
        mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        s += __shfl_xor_sync(0xffffffffu, s, o);
    }
    if (mx != 0.f && mx < 0x1p-60f) ok = false;
    // 2^e with mx 2^e in (224, 448]: e = floor(log2(448 / mx))
    int e = 0;
    if (mx > 0.f) {
        int ex;
        frexpf(mx, &ex);  // mx = f 2^ex, f in [0.5, 1)
        e = 8 - ex;       // mx 2^e in [128, 256)
        if (ldexpf(mx, e + 1) <= 448.f) e++;
    }
    for (uint32_t k = lane; k < dpad; k += 32) {
        const float v = k < d ? ldexpf(src[k], e) : 0.f;
        const __nv_fp8_storage_t h = __nv_cvt_float_to_fp8(v, __NV_SATFINITE, __NV_E4M3);
        const float r1 = v - e4m3_value(h);
        const __nv_fp8_storage_t m = __nv_cvt_float_to_fp8(r1, __NV_SATFINITE, __NV_E4M3);
        const float r2 = r1 - e4m3_value(m);
        dst[k] = h;
        dst[dpad + k] = m;
        dst[2 * dpad + k] = __nv_cvt_float_to_fp8(r2, __NV_SATFINITE, __NV_E4M3);
    }
    const bool all_ok = __all_sync(0xffffffffu, ok);
    if (lane == 0) {
        nrm[row] = __float_as_uint((float)s);
        scl[row] = ldexpf(1.f, -e);
        if (!all_ok) atomicOr(bad, 1u);
    }
}

}  // namespace

// err_c of the reduced-precision kinds: |d~ - d| <= err_c (|a|^2 + |b|^2)
// for d~ = |a|^2 + |b|^2 - 2 G~ against the reference's FP32 distance d,
// with |a||b| <= (|a|^2 + |b|^2) / 2 (so 2 |G~ - a.b| <= c (|a|^2 + |b|^2)
// when |G~ - a.b| <= c |a||b|):
//   parts      BF16 (unit roundoff u = 2^-8): a = hi + lo + e, |e| <= u^2 |a|,
//              the dropped lo.lo and e terms <= 3.1 u^2 |a_i||b_i| a component;
//              FP8 E4M3 (u = 2^-4, subnormal spacing 2^-9 after the 2^e
//              scaling): the dropped ml, lm, ll and residual terms <= 4.1 u^3
//              |a_i||b_i| + 3 2^-9 (|a_i| + |b_i|) scaled, i.e. + 6 sqrt(d)
//              2^-9 / 224 |a||b| after unscaling (the scale puts each row's
//              largest component above 224);
//   accumulate FP32 adds of all products, truncation allowed: 1.02 (P d + P)
//              2^-23 (P products per component), plus an allowance for the
//              MMA's internal grouping of 2^-16 (BF16) and 1.1 2^-13 (FP8);
//   norms      float of a double sum: 2^-24; final add and subtract: 2^-23;
//   reference  its own sequential FP32 sum: (d + 1) 2^-23 of a distance
//              <= 2 (|a|^2 + |b|^2);
// times a 1.25 safety factor.  Tests run the joins with every pair's exact
// distance checked against this bound (nnm_opts.audit).
static double err_coef(uint32_t kind, uint32_t d) {
    const double dd = (double)d, e23 = std::ldexp(1.0, -23);
    const double tail = std::ldexp(1.0, -24) + e23 + (dd + 1) * e23;
    if (kind == KIND_BF16) {
        const double u = std::ldexp(1.0, -8);
        return 1.25 * (3.1 * u * u + 1.02 * (3 * dd + 3) * e23 + std::ldexp(1.0, -16) + tail);
    }
    const double u = std::ldexp(1.0, -4);
    return 1.25 * (4.1 * u * u * u + 6.0 * std::sqrt(dd) * std::ldexp(1.0, -9) / 224.0 +
                   1.1 * std::ldexp(1.0, -13) + 1.02 * (6 * dd + 6) * e23 + tail);
}

int tc_prepare(Ctx& ctx, GraphStore& s, GraphDev& g) {
    g.xq = nullptr;
    g.nrm = nullptr;
    g.scl = nullptr;
    g.kq = 0;
    if (g.join_kernel == NNM_JOIN_FP32) return 0;
    const uint32_t kq = (g.d + 31) & ~31u;
    const char* why = nullptr;
    if (g.metric != L2) why = "the tensor-core join needs the L2 metric";
    else if (kq > TC_MAX_KQ) why = "the tensor-core join takes d <= 768";
    if (!why) {
        NNM_CUDA_TRY(s.nrm.ensure((size_t)g.n_cap * 4));
        DevBuf& m = ctx.ws.misc;
        NNM_CUDA_TRY(m.ensure(64));
        unsigned* flags = m.as<unsigned>();
        unsigned h[2] = {0, 0};
        if (g.join_kernel != NNM_JOIN_FP8) {
            NNM_CUDA_TRY(s.xq.ensure((size_t)g.n_cap * kq));
            NNM_CUDA_TRY(cudaMemsetAsync(m.p, 0, 16, ctx.stream));
            int nsm = 148;
            cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, ctx.device);
            k_quantize<<<std::min<uint32_t>((g.n_cap + 7) / 8, (uint32_t)nsm * 8), 256, 0, ctx.stream>>>(
                g.x, g.n_cap, g.d, g.dp, kq, s.xq.as<uint8_t>(),
                                                                  s.nrm.as<uint32_t>(), flags, flags + 1); count_launch();
            NNM_CUDA_TRY(cudaMemcpyAsync(h, flags, 8, cudaMemcpyDeviceToHost, ctx.stream));
            NNM_CUDA_TRY(cudaStreamSynchronize(ctx.stream));
            // every squared distance is at most |a|^2 + |b|^2 for non-negative vectors
            if (!h[0] && 2ull * h[1] < (1ull << 24)) {
                g.xq = s.xq.as<uint8_t>();
                g.nrm = s.nrm.as<uint32_t>();
                g.kq = kq;
                g.tc_kind = KIND_U8;
                return 0;
            }
        }
        // other data: BF16 (hi + lo) Gram matrices on request; FP8 (E4M3
        // hi + mid + lo, per-row power-of-two scales) on request for any data
        if (g.join_kernel == NNM_JOIN_AUTO) {
            why = "auto: FP32 join for non-integer data";
        } else if (g.join_kernel == NNM_JOIN_TENSOR) {
            const uint32_t dpad = (g.d + 15) & ~15u, kqb = 4 * dpad;
            if (kqb > TC_MAX_KQ) {
                why = "the BF16 tensor-core join takes d <= 192";
            } else {
                NNM_CUDA_TRY(s.xq.ensure((size_t)g.n_cap * kqb));
                NNM_CUDA_TRY(cudaMemsetAsync(m.p, 0, 16, ctx.stream));
                k_to_bf16x2<<<(g.n_cap + 7) / 8, 256, 0, ctx.stream>>>(g.x, g.n_cap, g.d, g.dp, dpad,
                                                                       s.xq.as<__nv_bfloat16>(),
                                                                       s.nrm.as<uint32_t>(), flags); count_launch();
                NNM_CUDA_TRY(cudaMemcpyAsync(h, flags, 4, cudaMemcpyDeviceToHost, ctx.stream));
                NNM_CUDA_TRY(cudaStreamSynchronize(ctx.stream));
                if (h[0]) {
                    why = "the BF16 tensor-core join needs finite components with magnitudes in [2^-60, 2^50]";
                } else {
                    g.xq = s.xq.as<uint8_t>();
                    g.nrm = s.nrm.as<uint32_t>();
                    g.kq = kqb;
                    g.tc_kind = KIND_BF16;
                    g.err_c = (float)err_coef(KIND_BF16, g.d);
                    return 0;
                }
            }
        } else {  // NNM_JOIN_FP8
            const uint32_t dpad = (g.d + 31) & ~31u, kq8 = 3 * dpad;
            if (kq8 > TC_MAX_KQ) {
                why = "the FP8 tensor-core join takes d <= 256";
            } else {
                NNM_CUDA_TRY(s.xq.ensure((size_t)g.n_cap * kq8));
                NNM_CUDA_TRY(s.scl.ensure((size_t)g.n_cap * 4));
                NNM_CUDA_TRY(cudaMemsetAsync(m.p, 0, 16, ctx.stream));
                k_to_fp8x3<<<(g.n_cap + 7) / 8, 256, 0, ctx.stream>>>(g.x, g.n_cap, g.d, g.dp, dpad, s.xq.as<uint8_t>(),
                                                                      s.nrm.as<uint32_t>(), s.scl.as<float>(),
                                                                      flags); count_launch();
                NNM_CUDA_TRY(cudaMemcpyAsync(h, flags, 4, cudaMemcpyDeviceToHost, ctx.stream));
                NNM_CUDA_TRY(cudaStreamSynchronize(ctx.stream));
                if (h[0]) {
                    why = "the FP8 tensor-core join needs finite components with magnitudes in [2^-60, 2^50]";
                } else {
                    g.xq = s.xq.as<uint8_t>();
                    g.nrm = s.nrm.as<uint32_t>();
                    g.scl = s.scl.as<float>();
                    g.kq = kq8;
                    g.tc_kind = KIND_FP8;
                    g.err_c = (float)err_coef(KIND_FP8, g.d);
                    return 0;
                }
            }
        }
    }
    if (why && (g.join_kernel == NNM_JOIN_TENSOR || g.join_kernel == NNM_JOIN_FP8)) {
        ctx.last_error = why;
        return 1;  // NNM_ERR_INVALID
    }
    return 0;
}

cudaError_t tc_set_attributes(uint32_t kq, uint32_t kind) {
    const int bytes = (int)std::max<size_t>(tc_smem_bytes(kq), TC_SMEM_FLOOR);
    cudaError_t e;
    const void* fns[3][4] = {{(const void*)k_join_tc<0, KIND_U8, false>, (const void*)k_join_tc<1, KIND_U8, false>,
                              (const void*)k_join_tc<1, KIND_U8, true>, (const void*)k_join_tc<0, KIND_U8, false>},
                             {(const void*)k_join_tc<0, KIND_BF16, false>, (const void*)k_join_tc<1, KIND_BF16, false>,
                              (const void*)k_join_tc<1, KIND_BF16, true>, (const void*)k_join_tc<0, KIND_BF16, false, true>},
                             {(const void*)k_join_tc<0, KIND_FP8, false>, (const void*)k_join_tc<1, KIND_FP8, false>,
                              (const void*)k_join_tc<1, KIND_FP8, true>, (const void*)k_join_tc<0, KIND_FP8, false, true>}};
    for (const void* f : fns[kind < 3 ? kind : 0])
        if ((e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes)) != cudaSuccess) return e;
    return cudaSuccess;
}

// One launch of a join variant: a persistent grid of the CTAs that are
// resident on the SMs at once, or fewer when the host knows the tile count.
// Residency is at most four CTAs per SM (TMEM: 512 columns, 128 a CTA),
// three for the u8 emit pass by registers (384 threads of 56), fewer when the
// tile buffers of wide operand rows fill the shared memory (two for BF16
// rows of d = 96).  It is counted here from the registers and shared-memory
// sizes: the occupancy query knows nothing of TMEM and reported half these
// counts, and a grid sized larger than the residency leaves a second wave of
// persistent CTAs whose tiles run last.
constexpr int TC_TMEM_CTAS = 512 / TC_COLS;
template <int PASS, int KIND, bool FAST, bool AUDIT = false>
static void launch_tc(const JoinArgs& ja, unsigned tiles, int nsm, size_t bytes, cudaStream_t st) {
    int dev = 0, smem_sm = 0, reserved = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
    cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev);
    cudaFuncAttributes fa{};
    cudaFuncGetAttributes(&fa, k_join_tc<PASS, KIND, FAST, AUDIT>);
    const int per_sm_smem = (int)((size_t)smem_sm / (bytes + fa.sharedSizeBytes + (size_t)reserved));
    int regs_sm = 65536;
    cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, dev);
    const int per_sm_regs = regs_sm / (((fa.numRegs + 7) & ~7) * tc_threads(PASS));
    const int per_sm = std::min(std::max(std::min(per_sm_smem, per_sm_regs), 1), TC_TMEM_CTAS);
    const unsigned grid = std::min<unsigned>(tiles, (unsigned)nsm * (unsigned)per_sm);
    k_join_tc<PASS, KIND, FAST, AUDIT><<<grid, tc_threads(PASS), bytes, st>>>(ja);
}

template <int KIND>
static void launch_tc_kind(int pass, const JoinArgs& ja, unsigned tiles, int nsm, size_t bytes, cudaStream_t st) {
    // the audit (reduced-precision kinds) in its own count-pass variant, so
    // that the unaudited one holds no code of it
    if (pass == 0 && KIND != KIND_U8 && ja.audit) launch_tc<0, KIND, false, KIND != KIND_U8>(ja, tiles, nsm, bytes, st);
    else if (pass == 0) launch_tc<0, KIND, false>(ja, tiles, nsm, bytes, st);
    else if (ja.fast_key) launch_tc<1, KIND, true>(ja, tiles, nsm, bytes, st);
    else launch_tc<1, KIND, false>(ja, tiles, nsm, bytes, st);
}

cudaError_t launch_join_tc(int pass, const JoinArgs& ja, const unsigned* ntier, int nsm, cudaStream_t st) {
    // ntier null: the counts are on the device only -- the full grid
    unsigned tiles = ~0u;
    if (ntier) {
        tiles = 0;
        for (int t = 0; t < 4; t++) tiles += (ntier[t] + (8u >> t) - 1) >> (3 - t);
        if (!tiles) return cudaSuccess;
    }
    const size_t bytes = std::max<size_t>(tc_smem_bytes(ja.kq), TC_SMEM_FLOOR);
    if (ja.tc_kind == KIND_U8) launch_tc_kind<KIND_U8>(pass, ja, tiles, nsm, bytes, st);
    else if (ja.tc_kind == KIND_BF16) launch_tc_kind<KIND_BF16>(pass, ja, tiles, nsm, bytes, st);
    else launch_tc_kind<KIND_FP8>(pass, ja, tiles, nsm, bytes, st);
    count_launch();
    return cudaGetLastError();
}

// k_pairs_tc: two row buffers; at least TC_SMEM_FLOOR, so that at most
// four CTAs (4 x 128 TMEM columns) share an SM.
size_t pairs_tc_smem(uint32_t R, uint32_t kq) { return std::max<size_t>(pt_smem_bytes(R, kq), TC_SMEM_FLOOR); }

cudaError_t pairs_tc_set_attributes(uint32_t R, uint32_t kq) {
    return cudaFuncSetAttribute(k_pairs_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pairs_tc_smem(R, kq));
}

// Residency counted as for the tiled join (shared memory, registers, the
// TMEM cap).
cudaError_t launch_pairs_tc(const JoinArgs& ja, uint32_t R, const unsigned* ntier, int nsm, cudaStream_t st) {
    if (ntier && !ntier[NTIER - 1]) return cudaSuccess;
    const size_t bytes = pairs_tc_smem(R, ja.kq);
    int dev = 0, smem_sm = 0, reserved = 0, regs_sm = 65536;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
    cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev);
    cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, dev);
    cudaFuncAttributes fa{};
    cudaFuncGetAttributes(&fa, k_pairs_tc);
    const int per_sm_smem = (int)((size_t)smem_sm / (bytes + fa.sharedSizeBytes + (size_t)reserved));
    const int per_sm_regs = regs_sm / (((fa.numRegs + 7) & ~7) * PT_THREADS);
    const int per_sm = std::min(std::max(std::min(per_sm_smem, per_sm_regs), 1), TC_TMEM_CTAS);
    const unsigned full = (unsigned)nsm * (unsigned)per_sm;
    const unsigned grid = ntier ? std::min<unsigned>(ntier[NTIER - 1], full) : full;
    k_pairs_tc<<<grid, PT_THREADS, bytes, st>>>(ja, R);
    count_launch();
    return cudaGetLastError();
}

}  // namespace nnm
