/* Stand-in for boost::accumulators as the reference uses it: one
 * accumulator_set<float, stats<tag::mean>> per NN-Descent iteration
 * (kgraph.cpp:324-331, abstractmerge.cpp:215-224, lynndescent.cpp:288-296).
 *
 * Boost's sum feature keeps a running sum of the sample type (float here),
 * adds each sample in call order, and mean() divides that float sum by the
 * std::size_t count (an ordinary float / size_t division, so the count is
 * converted to float).  The convergence test "mean < 0.002" is decided on
 * that exact float value, so this stand-in reproduces it operation for
 * operation.
 *
 * For parity checks every mean() result is also appended to a process-wide
 * trace (nnm_refshim_mean_trace), which tells the driver how many
 * iterations each NN-Descent loop ran and what its delta was. */
#ifndef NNM_REFSHIM_ACCUMULATORS_HPP
#define NNM_REFSHIM_ACCUMULATORS_HPP
#include <cstddef>
#include <vector>

std::vector<float> &nnm_refshim_mean_trace();

namespace boost { namespace accumulators {
namespace tag { struct mean {}; struct moment {}; }
template <typename... Features> struct stats {};
template <typename Sample, typename Features>
struct accumulator_set {
    Sample sum_ = Sample(0);
    std::size_t count_ = 0;
    void operator()(Sample x) { sum_ += x; ++count_; }
};
template <typename Sample, typename Features>
Sample mean(const accumulator_set<Sample, Features> &acc) {
    Sample m = acc.sum_ / acc.count_;
    nnm_refshim_mean_trace().push_back(m);
    return m;
}
}}
#endif
