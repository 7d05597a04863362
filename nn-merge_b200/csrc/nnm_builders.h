// Device graph builders (builders.cu).
#pragma once
#include <functional>
#include <vector>

#include "nnm_engine.h"

namespace nnm {

// Called after each H-Merge level that the reference turns into a DPG
// layer (lynndescent.cpp:767, :780-785, :797-799).
using LayerHook = std::function<int(Ctx&, GraphDev&)>;

// Copies n_cap x d vectors (host or device) into zero-padded rows of dp
// floats owned by `store`; sets g.dp and g.x.
int upload_vectors(Ctx& ctx, GraphStore& store, GraphDev& g, const float* x, bool x_on_device);
// Writes ids / distances / flags of rows [0, g.n); host or device outputs.
int export_graph(Ctx& ctx, const GraphDev& g, uint32_t* ids, float* dists, uint8_t* flags, bool host_out);

unsigned blocks_for(size_t n, unsigned per);
// Reads the device counters; a set error flag becomes status 6 with a message.
int check_counters(Ctx& ctx);

int kgraph_build(Ctx& ctx, GraphDev& g);
// Builds one graph per leaf [leaf_off[l], leaf_off[l+1]) and merges them;
// with two leaves split at n*5/10 this is Smerge::buildKGraph.
int merge_leaves(Ctx& ctx, GraphDev& g, const std::vector<uint32_t>& leaf_off, uint64_t* sub_ncmps);
int jmerge_build(Ctx& ctx, GraphDev& g, uint64_t* sub_ncmps);
// Fast tier, the two halves of merge_leaves: the leaf builds alone (leaf0:
// the index of the first leaf among all leaves of the build; pools end with
// ids of g's rows), and the merge of leaves whose graphs are in g's pools.
int build_leaves(Ctx& ctx, GraphDev& g, const std::vector<uint32_t>& leaf_off, uint32_t leaf0, uint64_t* ncmps);
int merge_prebuilt(Ctx& ctx, GraphDev& g, const std::vector<uint32_t>& leaf_off);
// Copies a caller's n x K device pools (ids of g's rows, distances) into g.
int load_pools(Ctx& ctx, GraphDev& g, const uint32_t* ids_dev, const float* dists_dev);
int hmerge_build(Ctx& ctx, GraphDev& g, const LayerHook& on_layer);

// Staged merge (reference streams): the steps of Smerge::buildKGraph
// (smerge.cpp:46-91) and Jmerge::buildKGraph (jmerge.cpp:43-80) as separate
// calls on one graph, its std::rand() stream continuing across them.
//   stage_subgraph      KGraph::buildKGraph on rows [b, e), in place (local ids)
//   stage_init_sgraph   AbstractMerge::InitSGraph from a device graph of local ids
//   stage_initial_graph Smerge::InitialGraph (MODE_SMERGE, halves split at pre)
//                       or Jmerge::InitialGraph (MODE_JMERGE, built rows [0, pre))
//   stage_nndescent     AbstractMerge::nnDescent with that class's localJoin filter
//   stage_merge2one     AbstractMerge::merge2one(sz)
// d_leaf_off: {0, pre, n} on the device (MODE_SMERGE).
int stage_subgraph(Ctx& ctx, GraphDev& g, uint32_t b, uint32_t e, uint64_t* ncmps);
int stage_init_sgraph(Ctx& ctx, GraphDev& g, uint32_t b, const uint32_t* d_graph, uint32_t gid, uint32_t rows);
int stage_initial_graph(Ctx& ctx, GraphDev& g, JoinMode mode, uint32_t pre, const uint32_t* d_leaf_off);
int stage_nndescent(Ctx& ctx, GraphDev& g, JoinMode mode, uint32_t pre, const uint32_t* d_leaf_off);
int stage_merge2one(Ctx& ctx, GraphDev& g, uint32_t sz);

}  // namespace nnm
