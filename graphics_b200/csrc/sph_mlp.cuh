// sph_mlp.cuh -- the warm-start network: 16 -> 64 -> 64 -> 1, GELU, BF16
// weights and activations in the tensor-core GEMMs, FP32 accumulation,
// FP32 master weights and biases.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#define MLP_IN 16
#define MLP_H 64
// FP32 parameter vector: W1[16][64] b1[64] W2[64][64] b2[64] W3[64] b3[1] (+3 pad)
#define MLP_OFF_W1 0
#define MLP_OFF_B1 (MLP_OFF_W1 + MLP_IN * MLP_H)
#define MLP_OFF_W2 (MLP_OFF_B1 + MLP_H)
#define MLP_OFF_B2 (MLP_OFF_W2 + MLP_H * MLP_H)
#define MLP_OFF_W3 (MLP_OFF_B2 + MLP_H)
#define MLP_OFF_B3 (MLP_OFF_W3 + MLP_H)
#define MLP_NPARAM (MLP_OFF_B3 + 1)
#define MLP_NPARAM_PAD 5316

struct MlpDev {
    float* master;          // FP32 parameters (Adam updates these)
    float* grad;            // FP32 gradient of the last mini-batch
    float* gpart;           // [blocks][MLP_NPARAM_PAD] per-block gradients and
                            // [blocks] squared errors (after them): summed in a
                            // fixed order, so training is run-to-run deterministic
    float* adam_m;
    float* adam_v;
    __nv_bfloat16* w_bf16;  // BF16 copies of W1, W2, W3 used by the GEMMs
    float* loss;            // summed squared error of the last batch
    // feature normalisation (per input: x' = (x - mean) * inv_std) and
    // label scale (y = y' * y_std + y_mean)
    float* norm;            // 2*16 + 2
};

// per-particle feature / label buffers for dataset recording
struct WsRecord {
    float* X;       // [n][16] features of the current step
    float* y;       // [n] labels of the current step
    float* dsX;     // dataset features [cap][16]
    float* dsy;     // dataset labels [cap]
    int* ds_count;  // samples in the dataset
    int ds_cap;
};

void launch_mlp_train_batch(const MlpDev& m, const float* X, const float* y, int n, int b0, int bsz, float inv_total,
                            cudaStream_t st);
void launch_mlp_adam(const MlpDev& m, float lr, int t, cudaStream_t st);
void launch_mlp_predict(const MlpDev& m, const float* X, float* y, int n, cudaStream_t st);
void launch_mlp_sync_bf16(const MlpDev& m, cudaStream_t st);
