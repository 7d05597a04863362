// Process-wide count of kernel launches made by this library (reported to
// callers through nnm_profile_get).
#pragma once
#include <atomic>
#include <cstdint>

namespace nnm {
inline std::atomic<uint64_t>& launch_counter() {
    static std::atomic<uint64_t> c{0};
    return c;
}
inline void count_launch(uint64_t k = 1) { launch_counter().fetch_add(k, std::memory_order_relaxed); }
}  // namespace nnm
