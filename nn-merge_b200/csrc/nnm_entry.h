// Entry-point network of the serving path (entry.cu).
#pragma once
#include <cstdint>

#include <cuda_bf16.h>

#include "../../include/nnm.h"
#include "nnm_hier.h"

namespace nnm {

constexpr uint32_t ENTRY_H = NNM_MLP_HIDDEN;            // 256 hidden units
constexpr uint32_t ENTRY_MAX_C = NNM_ENTRY_MAX_CLASSES;  // 4096
constexpr uint32_t ENTRY_MAX_D = 256;
constexpr int ENTRY_MAX_PROBES = 8;
constexpr uint32_t ENTRY_POOL = 262144;                 // training rows sampled from the index

// Device copy of a model: BF16 weights (w1t: d x 256; w2t: 256 x C and w2r:
// C x 256, the layouts the forward and backward kernels read coalesced),
// FP32 biases.
struct DevEntry {
    uint32_t d = 0, C = 0;
    float scale = 1.f, shift = 0.f;
    DevBuf w1t, b1, w2t, w2r, b2;
    void release();
};

int entry_upload(Ctx& ctx, DevEntry& m, const nnm_entry_mlp& h);
// Inference of rows [0, n) of x (stride dp): BF16 hidden rows into hbuf
// (n x 256 x 2 bytes), then either the scores (n x C, when scores is
// non-null) or the P probes of every row (n x P) from the tensor-core
// kernel.  A wait of that kernel that runs out sets 64 in *err.
int entry_infer(Ctx& ctx, const DevEntry& m, const float* x, uint32_t n, uint32_t dp, void* hbuf, float* scores,
                uint32_t P, uint32_t* probes, unsigned* err);
// Probes (nq x ix.nprobe rows) of queries q (stride ix.dp), with ix.net.
int entry_predict(Ctx& ctx, IndexDev& ix, const float* q, uint32_t nq, uint32_t* probes, unsigned* err);
int entry_grad(Ctx& ctx, const nnm_entry_mlp& model, const float* x_dev, uint32_t n, uint32_t dp,
               const uint32_t* lab_host, float* loss, nnm_entry_mlp& grad);
int entry_train(Ctx& ctx, IndexDev& ix, uint32_t layer, const nnm_train_opts& o, nnm_entry_mlp& model,
                float* loss_trace);

}  // namespace nnm
