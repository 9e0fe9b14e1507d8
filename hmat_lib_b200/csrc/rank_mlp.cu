// Training and inference kernels of the rank predictor (rank_mlp.h).
//
// One thread evaluates one sample with the parameters staged in shared
// memory.  The gradient kernel runs the forward and backward pass per lane,
// stages the activations and errors of a warp's 32 samples in shared memory
// and lets each lane sum the gradient terms of its own slice of the
// parameters over those samples; each warp accumulates into its own
// shared-memory copy, the warps of a block are summed in a fixed order, and
// the blocks' partial sums are added by a second kernel in a fixed order, so
// a gradient is reproducible bit for bit.
#include <algorithm>
#include <cmath>
#include <mutex>
#include <numeric>
#include <random>

#include "rank_mlp.h"

namespace hb {

namespace {

constexpr int kPredThreads = 64;
constexpr int kGradWarps = 2;
constexpr int kGradThreads = 32 * kGradWarps;
constexpr int kSamplesPerBlock = 256;

// Normalised input and first hidden layer (after ReLU) of one sample.
__device__ __forceinline__ void mlp_layer1(const float *__restrict__ P, const float *x,
                                           float (&xn)[kRankIn], float (&h1)[kRankH]) {
#pragma unroll
  for (int k = 0; k < kRankIn; ++k) xn[k] = (x[k] - P[k]) / P[kRankIn + k];
#pragma unroll
  for (int j = 0; j < kRankH; ++j) {
    float s = P[kRankB1 + j];
#pragma unroll
    for (int k = 0; k < kRankIn; ++k) s = fmaf(xn[k], P[kRankW1 + k * kRankH + j], s);
    h1[j] = fmaxf(s, 0.f);
  }
}

// Second hidden unit j (after ReLU) from the first layer.
__device__ __forceinline__ float mlp_unit2(const float *__restrict__ P, const float (&h1)[kRankH],
                                           int j) {
  float s = P[kRankB2 + j];
#pragma unroll
  for (int k = 0; k < kRankH; ++k) s = fmaf(h1[k], P[kRankW2 + k * kRankH + j], s);
  return fmaxf(s, 0.f);
}

// The first hidden layer of each thread's sample goes through shared memory,
// so layer 2 holds one accumulator at a time.
__global__ void __launch_bounds__(kPredThreads)
predict_kernel(const float *__restrict__ params, const float *__restrict__ x, int n, float *out) {
  __shared__ float P[kRankParams];
  __shared__ float H[kPredThreads][kRankH + 1];
  for (int i = threadIdx.x; i < kRankParams; i += blockDim.x) P[i] = params[i];
  __syncthreads();
  float *h = H[threadIdx.x];
#pragma unroll 1
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
    float xn[kRankIn];
#pragma unroll
    for (int k = 0; k < kRankIn; ++k)
      xn[k] = (x[(long long)s * kRankIn + k] - P[k]) / P[kRankIn + k];
#pragma unroll 4
    for (int j = 0; j < kRankH; ++j) {
      float a = P[kRankB1 + j];
#pragma unroll
      for (int k = 0; k < kRankIn; ++k) a = fmaf(xn[k], P[kRankW1 + k * kRankH + j], a);
      h[j] = fmaxf(a, 0.f);
    }
    float y = P[kRankB3];
#pragma unroll 1
    for (int j = 0; j < kRankH; ++j) {
      float a = P[kRankB2 + j];
#pragma unroll 8
      for (int k = 0; k < kRankH; ++k) a = fmaf(h[k], P[kRankW2 + k * kRankH + j], a);
      y = fmaf(fmaxf(a, 0.f), P[kRankW3 + j], y);
    }
    out[s] = y;
  }
}

// Block b: samples [b kSamplesPerBlock, (b + 1) kSamplesPerBlock); writes
// its partial gradient (kRankParams floats, then the partial loss) to
// partial[b].  Per group of 32 samples a warp stages the normalised inputs,
// activations and back-propagated errors of its lanes in shared memory; each
// lane then owns a fixed slice of the parameters and sums their gradient
// terms over the 32 samples.
__global__ void __launch_bounds__(kGradThreads)
gradient_kernel(const float *__restrict__ params, const float *__restrict__ x,
                const float *__restrict__ t, int n, float *__restrict__ partial) {
  extern __shared__ float sm[];
  constexpr int stride = kRankParams + 1;
  constexpr int kStage = 32 * (kRankIn + 4 * kRankH + 2);
  float *P = sm;                                             // kRankParams
  float *acc = P + kRankParams;                              // [kGradWarps][stride]
  float *stage = acc + kGradWarps * stride;                  // [kGradWarps][kStage]
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int i = threadIdx.x; i < kRankParams; i += blockDim.x) P[i] = params[i];
  for (int i = threadIdx.x; i < kGradWarps * stride; i += blockDim.x) acc[i] = 0.f;
  __syncthreads();
  float *A = acc + warp * stride;
  float *Sx = stage + warp * kStage;           // [32][8]   normalised inputs
  float *Sh1 = Sx + 32 * kRankIn;              // [32][64]  first hidden layer
  float *Sh2 = Sh1 + 32 * kRankH;              // [32][64]  second hidden layer
  float *Sd2 = Sh2 + 32 * kRankH;              // [32][64]  dL / d(pre-activation 2)
  float *Sd1 = Sd2 + 32 * kRankH;              // [32][64]  dL / d(pre-activation 1)
  float *Sdy = Sd1 + 32 * kRankH;              // [32]
  float *Se2 = Sdy + 32;                       // [32]
  const float inv_n = 1.f / (float)n;
  const int s0 = blockIdx.x * kSamplesPerBlock;
  for (int g = warp * 32; g < kSamplesPerBlock; g += kGradWarps * 32) {
    const int s = s0 + g + lane;
    const bool live = s < n;
    float xin[kRankIn], xn[kRankIn], h1[kRankH];
#pragma unroll
    for (int k = 0; k < kRankIn; ++k) xin[k] = live ? x[(long long)s * kRankIn + k] : P[k];
    mlp_layer1(P, xin, xn, h1);
    __syncwarp();
    unsigned long long mask2 = 0ULL;
    float y = P[kRankB3];
    for (int j = 0; j < kRankH; ++j) {
      const float h = mlp_unit2(P, h1, j);
      Sh2[lane * kRankH + j] = h;
      y = fmaf(h, P[kRankW3 + j], y);
      mask2 |= (unsigned long long)(h > 0.f) << j;
    }
    const float e = live ? y - t[s] : 0.f;
    const float dy = 2.f * e * inv_n;
#pragma unroll
    for (int k = 0; k < kRankIn; ++k) Sx[lane * kRankIn + k] = xn[k];
    for (int j = 0; j < kRankH; ++j)
      Sd2[lane * kRankH + j] = ((mask2 >> j) & 1ULL) ? dy * P[kRankW3 + j] : 0.f;
#pragma unroll
    for (int k = 0; k < kRankH; ++k) {
      Sh1[lane * kRankH + k] = h1[k];
      float s2 = 0.f;
      for (int j = 0; j < kRankH; ++j)
        s2 = fmaf(P[kRankW2 + k * kRankH + j], Sd2[lane * kRankH + j], s2);
      Sd1[lane * kRankH + k] = h1[k] > 0.f ? s2 : 0.f;
    }
    Sdy[lane] = dy;
    Se2[lane] = e * e * inv_n;
    __syncwarp();
    // W2: 4096 entries, 128 per lane; entry (k, j) = sum_l h1[l][k] dh2[l][j]
    for (int idx = lane; idx < kRankH * kRankH; idx += 32) {
      const int k = idx / kRankH, j = idx % kRankH;
      float v = 0.f;
#pragma unroll 8
      for (int l = 0; l < 32; ++l) v = fmaf(Sh1[l * kRankH + k], Sd2[l * kRankH + j], v);
      A[kRankW2 + idx] += v;
    }
    // W1: 512 entries; entry (i, k) = sum_l xn[l][i] dh1[l][k]
    for (int idx = lane; idx < kRankIn * kRankH; idx += 32) {
      const int i = idx / kRankH, k = idx % kRankH;
      float v = 0.f;
#pragma unroll 8
      for (int l = 0; l < 32; ++l) v = fmaf(Sx[l * kRankIn + i], Sd1[l * kRankH + k], v);
      A[kRankW1 + idx] += v;
    }
    // biases and W3 (entry j = sum_l dy_l h2[l][j])
    for (int j = lane; j < kRankH; j += 32) {
      float b1 = 0.f, b2 = 0.f, w3 = 0.f;
#pragma unroll 8
      for (int l = 0; l < 32; ++l) {
        b1 += Sd1[l * kRankH + j];
        b2 += Sd2[l * kRankH + j];
        w3 = fmaf(Sdy[l], Sh2[l * kRankH + j], w3);
      }
      A[kRankB1 + j] += b1;
      A[kRankB2 + j] += b2;
      A[kRankW3 + j] += w3;
    }
    if (lane == 0) {
      float b3 = 0.f, l2 = 0.f;
      for (int l = 0; l < 32; ++l) {
        b3 += Sdy[l];
        l2 += Se2[l];
      }
      A[kRankB3] += b3;
      A[kRankParams] += l2;
    }
    __syncwarp();
  }
  __syncthreads();
  float *out = partial + (long long)blockIdx.x * stride;
  for (int i = threadIdx.x; i < stride; i += blockDim.x) {
    float v = 0.f;
    for (int w = 0; w < kGradWarps; ++w) v += acc[w * stride + i];
    out[i] = i < kRankNorm ? 0.f : v;
  }
}

__global__ void reduce_partials_kernel(const float *__restrict__ partial, int nblocks,
                                       float *grad, float *loss) {
  constexpr int stride = kRankParams + 1;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < stride; i += gridDim.x * blockDim.x) {
    float s = 0.f;
    for (int b = 0; b < nblocks; ++b) s += partial[(long long)b * stride + i];
    if (i < kRankParams)
      grad[i] = s;
    else if (loss)
      *loss = s;
  }
}

__global__ void adam_kernel(float *params, const float *grad, float *m, float *v, float lr,
                            float b1, float b2, float eps, float c1, float c2) {
  const int i = kRankNorm + blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= kRankParams) return;
  const float g = grad[i];
  const float mi = b1 * m[i] + (1.f - b1) * g;
  const float vi = b2 * v[i] + (1.f - b2) * g * g;
  m[i] = mi;
  v[i] = vi;
  params[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

struct DevF {
  float *p = nullptr;
  explicit DevF(size_t n) { HB_CUDA(cudaMalloc((void **)&p, sizeof(float) * std::max<size_t>(n, 1))); }
  ~DevF() {
    if (p) cudaFree(p);
  }
};

std::mutex g_model_mutex;
std::vector<float> g_model;

}  // namespace

void rank_mlp_predict(const float *d_params, const float *d_x, int n, float *d_out,
                      cudaStream_t stream) {
  if (n <= 0) return;
  const int grid = std::min((n + kPredThreads - 1) / kPredThreads, 4 * num_sms());
  predict_kernel<<<grid, kPredThreads, 0, stream>>>(d_params, d_x, n, d_out);
  HB_LAUNCHED();
}

void rank_mlp_gradient(const float *d_params, const float *d_x, const float *d_t, int n,
                       float *d_grad, float *d_loss, cudaStream_t stream) {
  HB_REQUIRE(n > 0, INPUT_ERROR, "rank model gradient: no samples");
  const int nblocks = (n + kSamplesPerBlock - 1) / kSamplesPerBlock;
  const size_t smem = sizeof(float) * (kRankParams + kGradWarps * (kRankParams + 1) +
                                      kGradWarps * 32 * (kRankIn + 4 * kRankH + 2));
  static bool configured = false;
  if (!configured) {
    HB_CUDA(cudaFuncSetAttribute(gradient_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem));
    configured = true;
  }
  float *partial = nullptr;
  HB_CUDA(cudaMallocAsync((void **)&partial, sizeof(float) * nblocks * (kRankParams + 1), stream));
  gradient_kernel<<<nblocks, kGradThreads, smem, stream>>>(d_params, d_x, d_t, n, partial);
  HB_LAUNCHED();
  reduce_partials_kernel<<<(kRankParams + 256) / 256, 256, 0, stream>>>(partial, nblocks, d_grad,
                                                                      d_loss);
  HB_LAUNCHED();
  cudaFreeAsync(partial, stream);
}

void rank_mlp_adam(float *d_params, const float *d_grad, float *d_m, float *d_v, int step,
                   const RankTrainConfig &cfg, cudaStream_t stream) {
  const float c1 = 1.f - std::pow(cfg.beta1, (float)step);
  const float c2 = 1.f - std::pow(cfg.beta2, (float)step);
  adam_kernel<<<(kRankTrain + 255) / 256, 256, 0, stream>>>(d_params, d_grad, d_m, d_v, cfg.lr,
                                                           cfg.beta1, cfg.beta2, cfg.eps, c1, c2);
  HB_LAUNCHED();
}

std::vector<float> rank_mlp_train(const std::vector<float> &x, const std::vector<float> &t,
                                  const RankTrainConfig &cfg, std::vector<float> *loss_log,
                                  cudaStream_t stream) {
  const int n = (int)t.size();
  HB_REQUIRE(n > 0 && x.size() == (size_t)n * kRankIn, INPUT_ERROR,
             "rank model training: features must be n x 8");
  std::vector<float> P(kRankParams, 0.f);
  // normalisation from the data
  for (int k = 0; k < kRankIn; ++k) {
    double mu = 0.0, var = 0.0;
    for (int s = 0; s < n; ++s) mu += x[(size_t)s * kRankIn + k];
    mu /= n;
    for (int s = 0; s < n; ++s) {
      const double d = x[(size_t)s * kRankIn + k] - mu;
      var += d * d;
    }
    P[k] = (float)mu;
    P[kRankIn + k] = (float)std::max(std::sqrt(var / n), 1e-3);
  }
  std::mt19937_64 rng(cfg.seed);
  std::normal_distribution<float> nd(0.f, 1.f);
  for (int i = 0; i < kRankIn * kRankH; ++i) P[kRankW1 + i] = nd(rng) * std::sqrt(2.f / kRankIn);
  for (int i = 0; i < kRankH * kRankH; ++i) P[kRankW2 + i] = nd(rng) * std::sqrt(2.f / kRankH);
  for (int i = 0; i < kRankH; ++i) P[kRankW3 + i] = nd(rng) * std::sqrt(1.f / kRankH);
  P[kRankB3] = (float)(std::accumulate(t.begin(), t.end(), 0.0) / n);

  DevF dp(kRankParams), dg(kRankParams), dm(kRankParams), dv(kRankParams), dl(1);
  DevF dxa((size_t)n * kRankIn), dta(n);
  const int bs = std::min(cfg.batch, n);
  DevF dxb((size_t)bs * kRankIn), dtb(bs);
  HB_CUDA(cudaMemcpyAsync(dp.p, P.data(), sizeof(float) * kRankParams, cudaMemcpyHostToDevice,
                          stream));
  HB_CUDA(cudaMemsetAsync(dm.p, 0, sizeof(float) * kRankParams, stream));
  HB_CUDA(cudaMemsetAsync(dv.p, 0, sizeof(float) * kRankParams, stream));
  HB_CUDA(cudaMemcpyAsync(dxa.p, x.data(), sizeof(float) * x.size(), cudaMemcpyHostToDevice,
                          stream));
  HB_CUDA(cudaMemcpyAsync(dta.p, t.data(), sizeof(float) * t.size(), cudaMemcpyHostToDevice,
                          stream));
  std::vector<int> perm(n);
  std::iota(perm.begin(), perm.end(), 0);
  std::vector<float> bx((size_t)bs * kRankIn), bt(bs);
  int pos = n;   // forces a shuffle on the first step
  for (int step = 1; step <= cfg.steps; ++step) {
    if (pos + bs > n) {
      std::shuffle(perm.begin(), perm.end(), rng);
      pos = 0;
    }
    for (int i = 0; i < bs; ++i) {
      const int s = perm[pos + i];
      std::copy(&x[(size_t)s * kRankIn], &x[(size_t)s * kRankIn] + kRankIn, &bx[(size_t)i * kRankIn]);
      bt[i] = t[s];
    }
    pos += bs;
    HB_CUDA(cudaMemcpyAsync(dxb.p, bx.data(), sizeof(float) * bx.size(), cudaMemcpyHostToDevice,
                            stream));
    HB_CUDA(cudaMemcpyAsync(dtb.p, bt.data(), sizeof(float) * bt.size(), cudaMemcpyHostToDevice,
                            stream));
    rank_mlp_gradient(dp.p, dxb.p, dtb.p, bs, dg.p, nullptr, stream);
    rank_mlp_adam(dp.p, dg.p, dm.p, dv.p, step, cfg, stream);
    // the host staging buffers are reused next step
    HB_CUDA(cudaStreamSynchronize(stream));
    if (loss_log && (step % 100 == 0 || step == cfg.steps)) {
      rank_mlp_gradient(dp.p, dxa.p, dta.p, n, dg.p, dl.p, stream);
      float l = 0.f;
      HB_CUDA(cudaMemcpyAsync(&l, dl.p, sizeof(float), cudaMemcpyDeviceToHost, stream));
      HB_CUDA(cudaStreamSynchronize(stream));
      loss_log->push_back(l);
    }
  }
  HB_CUDA(cudaMemcpyAsync(P.data(), dp.p, sizeof(float) * kRankParams, cudaMemcpyDeviceToHost,
                          stream));
  HB_CUDA(cudaStreamSynchronize(stream));
  return P;
}

void set_rank_model(const std::vector<float> &params) {
  std::lock_guard<std::mutex> lk(g_model_mutex);
  g_model = params;
}

bool rank_model(std::vector<float> &out) {
  std::lock_guard<std::mutex> lk(g_model_mutex);
  if (g_model.size() != (size_t)kRankParams) return false;
  out = g_model;
  return true;
}

}  // namespace hb
