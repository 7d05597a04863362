/* Force-included into every reference translation unit by oracle/Makefile.
 *
 * The reference seeds each phase's generator with std::mt19937 rng(time(NULL))
 * (kgraph.cpp:65, smerge.cpp:97, jmerge.cpp:86, lynndescent.cpp:156 and :357,
 * lysearch.cpp:456).  Within one wall-clock second every phase gets the same
 * seed.  Routing time() to nnm_refshim_time() freezes that clock at a value
 * the driver chooses, which makes a reference run reproducible without
 * editing its sources.  <ctime> is included first so that its declarations
 * are seen before the macro exists. */
#ifndef NNM_REFSEED_H
#define NNM_REFSEED_H
#include <ctime>
#include <cstddef>
#include <algorithm>
extern "C" time_t nnm_refshim_time(time_t *t);
#define time(t) nnm_refshim_time(t)
#endif
