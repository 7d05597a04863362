/* Stand-in for boost::timer::cpu_timer as the reference uses it
 * (kgraph.cpp:219-225, smerge.cpp:75-82, jmerge.cpp:63-71,
 * lynndescent.cpp:753-814): construct, then elapsed().wall in ns. */
#ifndef NNM_REFSHIM_TIMER_HPP
#define NNM_REFSHIM_TIMER_HPP
#include <chrono>
#include <cstdint>
namespace boost { namespace timer {
struct cpu_times { std::int64_t wall, user, system; };
class cpu_timer {
    std::chrono::steady_clock::time_point t0_ = std::chrono::steady_clock::now();
public:
    cpu_times elapsed() const {
        auto ns = std::chrono::duration_cast<std::chrono::nanoseconds>(
                      std::chrono::steady_clock::now() - t0_).count();
        return cpu_times{ns, ns, 0};
    }
};
}}
#endif
