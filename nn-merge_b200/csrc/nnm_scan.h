#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace nnm {
// Scratch size (in u64 elements) that exclusive_scan needs for n inputs.
size_t scan_temp_elems(size_t n);
// out[i] = in[0] + ... + in[i-1] for i in [0, n]; out has n+1 entries and
// out[n] is the total, also written to *d_total when non-null.
cudaError_t exclusive_scan(const uint32_t* in, uint64_t* out, size_t n, uint64_t* temp, uint64_t* d_total,
                           cudaStream_t st);
}  // namespace nnm
