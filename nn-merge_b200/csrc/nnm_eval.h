// Recall of a k-NN graph against exact brute force on the device (eval.cu).
#pragma once
#include <cstdint>

#include "nnm_engine.h"

namespace nnm {

constexpr int EVAL_MAX_ATOP = 16;

// Recall@atop of rows[0, nrows) of the graph ids (n x k, device) over the
// vectors x (n x dp, device); rows is a device array.
int graph_recall_dev(Ctx& ctx, const float* x, uint32_t n, uint32_t dp, int metric, const uint32_t* ids, uint32_t k,
                     const uint32_t* rows, uint32_t nrows, uint32_t atop, double* recall);

}  // namespace nnm
