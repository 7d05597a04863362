// Device-wide exclusive prefix sums (u32 counts -> u64 offsets), used to lay
// out per-row and per-target segments (reverse lists, proposal buckets,
// random-draw ranges).  Three passes: per-tile totals, a scan of the tile
// totals in one block, then per-tile scans.  HBM-bound: 4 B read + 8 B
// written per element.
#include <cstdint>
#include <cuda_runtime.h>

#include "nnm_scan.h"
#include "nnm_launch.h"

namespace nnm {
namespace {
constexpr int SCAN_THREADS = 512;
constexpr int SCAN_ITEMS = 8;
constexpr int TILE = SCAN_THREADS * SCAN_ITEMS;

__device__ __forceinline__ uint64_t block_exclusive_scan(uint64_t v, uint64_t* sh, uint64_t* total) {
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    uint64_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint64_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) sh[wid] = x;
    __syncthreads();
    if (wid == 0) {
        uint64_t s = lane < (int)(blockDim.x >> 5) ? sh[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint64_t y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        sh[lane] = s;
    }
    __syncthreads();
    uint64_t before = wid ? sh[wid - 1] : 0;
    if (total) *total = sh[(blockDim.x >> 5) - 1];
    __syncthreads();
    return before + x - v;
}

__global__ void k_tile_sums(const uint32_t* __restrict__ in, size_t n, uint64_t* __restrict__ sums) {
    __shared__ uint64_t sh[32];
    size_t base = (size_t)blockIdx.x * TILE + (size_t)threadIdx.x * SCAN_ITEMS;
    uint64_t s = 0;
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; i++)
        if (base + i < n) s += in[base + i];
    uint64_t tot;
    block_exclusive_scan(s, sh, &tot);
    if (threadIdx.x == 0) sums[blockIdx.x] = tot;
}

__global__ void k_scan_sums(uint64_t* __restrict__ sums, size_t m, uint64_t* __restrict__ grand) {
    __shared__ uint64_t sh[32];
    uint64_t carry = 0;
    for (size_t b = 0; b < m; b += SCAN_THREADS) {
        size_t i = b + threadIdx.x;
        uint64_t v = i < m ? sums[i] : 0;
        uint64_t tot;
        uint64_t ex = block_exclusive_scan(v, sh, &tot);
        if (i < m) sums[i] = carry + ex;
        carry += tot;
    }
    if (threadIdx.x == 0 && grand) *grand = carry;
}

__global__ void k_tile_scan(const uint32_t* __restrict__ in, size_t n, const uint64_t* __restrict__ sums,
                            uint64_t* __restrict__ out) {
    __shared__ uint64_t sh[32];
    size_t base = (size_t)blockIdx.x * TILE + (size_t)threadIdx.x * SCAN_ITEMS;
    uint32_t v[SCAN_ITEMS];
    uint64_t s = 0;
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; i++) {
        v[i] = base + i < n ? in[base + i] : 0;
        s += v[i];
    }
    uint64_t ex = block_exclusive_scan(s, sh, nullptr) + sums[blockIdx.x];
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; i++) {
        if (base + i < n) out[base + i] = ex;
        ex += v[i];
    }
    if (base < n && base + SCAN_ITEMS >= n) out[n] = ex;  // thread owning the last element
}
}  // namespace

size_t scan_temp_elems(size_t n) { return (n + TILE - 1) / TILE + 1; }

cudaError_t exclusive_scan(const uint32_t* in, uint64_t* out, size_t n, uint64_t* temp, uint64_t* d_total,
                           cudaStream_t st) {
    if (n == 0) {
        cudaError_t e = cudaMemsetAsync(out, 0, sizeof(uint64_t), st);
        if (e == cudaSuccess && d_total) e = cudaMemsetAsync(d_total, 0, sizeof(uint64_t), st);
        return e;
    }
    size_t tiles = (n + TILE - 1) / TILE;
    k_tile_sums<<<(unsigned)tiles, SCAN_THREADS, 0, st>>>(in, n, temp); count_launch();
    k_scan_sums<<<1, SCAN_THREADS, 0, st>>>(temp, tiles, d_total); count_launch();
    k_tile_scan<<<(unsigned)tiles, SCAN_THREADS, 0, st>>>(in, n, temp, out); count_launch();
    return cudaGetLastError();
}

}  // namespace nnm
