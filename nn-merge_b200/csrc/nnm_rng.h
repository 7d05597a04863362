// Reference-exact random streams (see rng.cu).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace nnm {
// s[0..61] of the glibc rand() sequence after srand(seed) (see rng.cu).
struct GlibcBase {
    uint32_t s[62];
};
GlibcBase glibc_base(uint32_t seed);
// Loads the seed-independent jump table x^(2^b) mod P into constant memory
// of the current device.  Must run once per device before generating.
cudaError_t glibc_tables_init();
// Writes rand() outputs #first_output .. #first_output+count-1 (counted from
// srand) to out[0..count).  count is read on the device from *d_count when
// d_count is non-null (capped at count_cap), else count = count_cap.
cudaError_t glibc_stream_generate(int32_t* out, const GlibcBase& base, uint64_t first_output,
                                  const uint64_t* d_count, uint64_t count_cap, cudaStream_t st);
// std::mt19937(seed) outputs, in order, on the host.
void gen_mt19937(uint32_t seed, uint64_t count, uint32_t* out);
}  // namespace nnm
