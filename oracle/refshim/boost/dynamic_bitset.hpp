/* The reference includes this header (kgraph.h:5, lynndescent.h:8,
 * lysearch.h:7) but uses nothing from it. */
#ifndef NNM_REFSHIM_DYNAMIC_BITSET_HPP
#define NNM_REFSHIM_DYNAMIC_BITSET_HPP
#endif
