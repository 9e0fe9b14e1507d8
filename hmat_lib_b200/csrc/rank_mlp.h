// Learned rank predictor: a small MLP (8 -> 64 -> 64 -> 1, ReLU, FP32) that
// maps a block's features to log2(rank + 1) at the requested tolerance, so
// the randomized range finder can size its sketch in one shot.  Training and
// inference run on the GPU with the kernels of rank_mlp.cu.
//
// Features of an off-diagonal block (all FP32):
//   0  log2(min(m, n))                block size
//   1  depth of the block's node      level
//   2  ln(l)                          kernel length (option "kernel_length"; 0 if unknown)
//   3..7  log10(s_i / s_1), i = 2, 4, 8, 12, 16, of the 16 singular values of
//         a Gaussian sketch A_b Omega (Omega n x 16), floored at -20
//
// Parameter vector layout (kRankParams floats): feature mean[8], feature
// scale[8] (inputs are (f - mean) / scale), W1[8][64], b1[64], W2[64][64],
// b2[64], W3[64], b3.
#pragma once

#include <vector>

#include "common.h"

namespace hb {

constexpr int kRankIn = 8, kRankH = 64;
constexpr int kRankNorm = 2 * kRankIn;
constexpr int kRankW1 = kRankNorm, kRankB1 = kRankW1 + kRankIn * kRankH;
constexpr int kRankW2 = kRankB1 + kRankH, kRankB2 = kRankW2 + kRankH * kRankH;
constexpr int kRankW3 = kRankB2 + kRankH, kRankB3 = kRankW3 + kRankH;
constexpr int kRankParams = kRankB3 + 1;   // 4817
constexpr int kRankTrain = kRankParams - kRankNorm;   // trainable (all but the normalisation)

// out[i] = network(params, x[i]) for n samples (x: n x 8 row-major), device pointers.
void rank_mlp_predict(const float *d_params, const float *d_x, int n, float *d_out,
                      cudaStream_t stream);

// Mean squared error over n samples and its gradient with respect to the
// trainable parameters (d_grad: kRankParams floats, the normalisation part
// left zero); deterministic.  d_loss: one float.
void rank_mlp_gradient(const float *d_params, const float *d_x, const float *d_t, int n,
                       float *d_grad, float *d_loss, cudaStream_t stream);

struct RankTrainConfig {
  int steps = 3000;
  int batch = 8192;
  float lr = 3e-3f;
  float beta1 = 0.9f, beta2 = 0.999f, eps = 1e-8f;
  unsigned long long seed = 1;
};

// Trains from scratch on n samples (host arrays; targets log2(rank + 1)):
// normalisation from the data, He-initialised weights, Adam on mini-batches
// drawn without replacement each epoch.  Returns the parameters; `loss_log`
// receives the full-data loss every 100 steps.
std::vector<float> rank_mlp_train(const std::vector<float> &x, const std::vector<float> &t,
                                  const RankTrainConfig &cfg, std::vector<float> *loss_log,
                                  cudaStream_t stream);

// One Adam update of the trainable parameters (exposed for the parity test).
void rank_mlp_adam(float *d_params, const float *d_grad, float *d_m, float *d_v, int step,
                   const RankTrainConfig &cfg, cudaStream_t stream);

// The model used by builds (set through the C API; empty: none).
void set_rank_model(const std::vector<float> &params);
bool rank_model(std::vector<float> &out);

}  // namespace hb
