// Learned initialisation: the code MLP (learned.cu) and the code-ordered
// candidate graphs built from it (learned_init.cu).
#pragma once
#include <cstdint>
#include <vector>

#include <cuda_bf16.h>

#include "../../include/nnm.h"
#include "nnm_engine.h"

namespace nnm {

constexpr uint32_t MLP_H = NNM_MLP_HIDDEN;  // 256
constexpr uint32_t MLP_O = NNM_MLP_OUT;     // 32: one code bit per lane
constexpr uint32_t MLP_MAX_D = 256;

// Device copy of a model: BF16 weights, transposed for coalesced reads
// (w1t: d x 256, w2t: 256 x 32), FP32 biases.
struct DevMlp {
    uint32_t d = 0;
    float scale = 1.f, shift = 0.f;
    DevBuf w1t, b1, w2t, b2;
    void release() {
        w1t.release();
        b1.release();
        w2t.release();
        b2.release();
    }
};

// Read-only view the kernels take.
struct MlpView {
    const __nv_bfloat16* w1t;
    const float* b1;
    const __nv_bfloat16* w2t;
    const float* b2;
    uint32_t d;
    float scale, shift;
};

int mlp_upload(Ctx& ctx, DevMlp& m, const nnm_mlp& h);
// codes (n) and optionally z (n x 32) of rows [0, n) of x (stride dp).
int mlp_codes_dev(Ctx& ctx, const DevMlp& m, const float* x, uint32_t n, uint32_t dp, uint32_t* codes, float* z);
int mlp_train(Ctx& ctx, const float* x_dev, uint32_t n, uint32_t dp, const uint32_t* graph_dev, uint32_t K,
              const nnm_train_opts& o, nnm_mlp& model, float* loss_trace);
int mlp_grad(Ctx& ctx, const nnm_mlp& model, const float* x_dev, uint32_t n, uint32_t dp, const uint32_t* trip_host,
             uint32_t ntrip, float margin, float* loss, nnm_mlp& grad);

// Kernels shared with the entry network (entry.cu); neither counts its launch.
// dW1 (256 x d) and db1 of dL/dh over rows idx[0..R) of x.
void launch_grad_w1(const float* dh, const float* x, uint32_t dp, const uint32_t* idx, uint32_t R, uint32_t d,
                    float scale, float shift, float* gw1, float* gb1, cudaStream_t st);
// One Adam step over cnt parameters; the step number is read from *step.
void launch_adam(float* p, float* mo, float* ve, const float* g, uint32_t cnt, float lr, const uint32_t* step,
                 cudaStream_t st);

// Code orderings of a graph's rows, per leaf: V views (the code rotated by
// 8v bits), each leaf's rows sorted by (view key, row) into a segment of P
// slots (padded with all-ones keys).
struct CodeViews {
    uint32_t V = 0, nleaf = 0, P = 0, n = 0;
    std::vector<uint32_t> leaf_off;
    const unsigned long long* keys = nullptr;  // V*nleaf*P sorted (key << 32 | row)
    const uint32_t* pos = nullptr;             // V x n: position of each row in its leaf's segment
    const unsigned long long* fence = nullptr; // V*nleaf*(P / VFENCE): key VFENCE*i of each segment
};
constexpr uint32_t VFENCE = 256;
int views_build(Ctx& ctx, const GraphDev& g, const std::vector<uint32_t>& leaf_off, CodeViews& out);
// Initial pools of rows [0, s.n) of the leaf sub-graph s (leaf `leaf` of vw).
int learned_rows(Ctx& ctx, GraphDev& s, const CodeViews& vw, uint32_t leaf);
// Merge cross samples: every row keeps its best K - g.cut entries and takes
// g.cut rows of other leaves, the nearest among its code neighbours there.
int learned_cross(Ctx& ctx, GraphDev& g, const CodeViews& vw, const uint32_t* d_leaf_off);

}  // namespace nnm
