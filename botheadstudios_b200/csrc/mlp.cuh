// Learned smoothing-length MLP (8 → 64 → 64 → 1, GELU; BF16 tensor-core operands, FP32 accumulation):
// parameter layout, packed device weights and the launchers shared by the solver and the trainer.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "sph_kernels.cuh"

namespace sphb {

constexpr int MLP_IN = 8, MLP_H = 64;
// Parameter block (floats): W1[8][64] b1[64] W2[64][64] b2[64] W3[64] b3 | x_mean[8] x_scale[8] y_mean y_scale
constexpr int MLP_W1 = 0, MLP_B1 = MLP_W1 + MLP_IN * MLP_H, MLP_W2 = MLP_B1 + MLP_H, MLP_B2 = MLP_W2 + MLP_H * MLP_H,
              MLP_W3 = MLP_B2 + MLP_H, MLP_B3 = MLP_W3 + MLP_H, MLP_TRAIN = MLP_B3 + 1, MLP_XM = MLP_TRAIN,
              MLP_XS = MLP_XM + MLP_IN, MLP_YM = MLP_XS + MLP_IN, MLP_YS = MLP_YM + 1, MLP_TOTAL = MLP_YS + 1;
static_assert(MLP_TRAIN == 4801 && MLP_TOTAL == 4819, "parameter block");

// Weights as the kernels read them: BF16 matrices row by row (the kernels copy them into the tcgen05 operand layout; K padded to
// 16 for the first layer), FP32 biases and normalisation, W3 rounded to BF16 and held as FP32.
struct MlpPacked {
  __nv_bfloat16 w1t[MLP_H * 16];     // [out][in], in 8..15 zero
  __nv_bfloat16 w2t[MLP_H * MLP_H];  // [out][in]
  __nv_bfloat16 w2[MLP_H * MLP_H];   // [in][out]
  float w3[MLP_H];
  float b1[MLP_H], b2[MLP_H];
  float b3;
  float xm[MLP_IN], xs[MLP_IN];
  float ym, ys;
};

// FP32 parameter block → packed weights (one block of 256 threads).
int launch_mlp_pack(const float* params, MlpPacked* out, cudaStream_t s);

// Inputs of the proposal, per particle, from the state of the step that is being taken (before the drift's
// new positions are sorted): the solver's feature definition, shared by the in-step proposal and the
// recorded training features.
struct MlpFeatureArgs {
  float eta;         // h = eta (m/rho)^(1/3) at the target neighbour count
  float n_target;    // target neighbour count
};

// In-step proposal: features → MLP y = log(h_next/h(ρ)) → Δlog h = y − log(h/h(ρ)) → h ← h·exp(clamp(Δ, ±0.03))
// in pos_h.w (sorted order). With `rec` non-null, also writes each particle's 8 features to rec[id]
// (original order) and its Δlog h to dh[id].
int launch_mlp_propose(const Dev& d, const MlpPacked* w, const MlpFeatureArgs& fa, const float* divv,
                       float* rec, float* dh, bool apply, cudaStream_t s);

// Standalone forward over feature rows x[n][8] → de-normalised outputs; *err |= 1 if a tensor-core barrier
// wait gave up (the outputs are then NaN).
int launch_mlp_forward(const MlpPacked* w, const float* x, int n, float* out, unsigned* err, cudaStream_t s);

// One training minibatch on tcgen05: forward + backward over rows idx[0..m) of (x, t), gradients of the mean
// squared error on the normalised target (divided by `denom`) accumulated into grad[4801], the summed squared
// error into *loss; *err |= 1 if a tensor-core barrier wait gave up (the tile's gradients are then incomplete).
int launch_mlp_train_batch(const MlpPacked* w, const float* x, const float* t, const unsigned* idx, int m,
                           float denom, float* grad, float* loss, unsigned* err, cudaStream_t s);

// Adam on the trainable parameters (FP32 master copy), step count `step` (1-based).
int launch_mlp_adam(float* params, const float* grad, float* m, float* v, int step, float lr, float b1, float b2,
                    float eps, float wd, cudaStream_t s);

}  // namespace sphb
