// Batched TSQR (Householder QR of 256-row chunks in shared memory, reduced
// up a tree of stacked R factors, explicit Q rebuilt top-down) plus the
// small utility kernels of the randomized compression: Gaussian test
// matrices, column norms.
//
// Replaces the dgeqrt factorisations of hmat_lib (src/hodlr_algebra.c:120,
// 126) and provides the orthonormal bases of the randomized range finder
// that stands in for dgesdd on large blocks (src/constructors.c:323).
#include <algorithm>
#include <chrono>

#include "gemm_f64.h"
#include "tsqr.h"

namespace hb {

namespace {

constexpr int kQT = 256;   // threads per CTA (one row of a chunk each)

struct QrChunk {
  double *A;
  long long lda;
  int rows, w;
  double *R;
  long long ldr;
};

struct MulChunk {
  double *Q;
  long long ldq;
  int rows, w;
  const double *M;
  long long ldm;
};

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ double block_sum(double v, double *red) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  v = warp_sum(v);
  if (lane == 0) red[warp] = v;
  __syncthreads();
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < kQT / 32; ++k) s += red[k];
  __syncthreads();
  return s;
}

constexpr size_t kQrSmem = sizeof(double) * (2 * kChunk * kPanel + 2 * kPanel + kQT / 32);
static_assert(kChunk == kQT, "one thread per row of a chunk");

// Householder QR of one chunk (rows <= 256, w <= 32), LAPACK dlarfg
// convention: H_j = I - tau_j v_j v_j^T, v_j(j) = 1, beta_j = -sign(x0)||x||.
__global__ void __launch_bounds__(kQT) qr_chunk_kernel(const QrChunk *__restrict__ descs) {
  const QrChunk D = descs[blockIdx.x];
  extern __shared__ double sm[];
  double *S = sm;                          // chunk, column-major, ld kChunk
  double *E = S + kChunk * kPanel;         // explicit Q under construction
  double *tau = E + kChunk * kPanel;
  double *wv = tau + kPanel;
  double *red = wv + kPanel;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int r = D.rows, w = D.w, k = min(r, w);

  for (int e = tid; e < kChunk * kPanel; e += kQT) {
    const int i = e % kChunk, j = e / kChunk;
    S[e] = (i < r && j < w) ? D.A[i + (long long)j * D.lda] : 0.0;
  }
  __syncthreads();

  for (int j = 0; j < k; ++j) {
    double part = 0.0;
    for (int i = j + 1 + tid; i < r; i += kQT) part = fma(S[i + j * kChunk], S[i + j * kChunk], part);
    const double sigma2 = block_sum(part, red);
    const double x0 = S[j + j * kChunk];
    double beta = x0, t = 0.0, scale = 0.0;
    if (sigma2 > 0.0) {
      const double nrm = sqrt(fma(x0, x0, sigma2));
      beta = x0 >= 0.0 ? -nrm : nrm;
      t = (beta - x0) / beta;
      scale = 1.0 / (x0 - beta);
    }
    __syncthreads();
    for (int i = j + 1 + tid; i < r; i += kQT) S[i + j * kChunk] *= scale;
    if (tid == 0) {
      S[j + j * kChunk] = beta;
      tau[j] = t;
    }
    __syncthreads();
    for (int c = j + 1 + warp; c < w; c += kQT / 32) {
      double dot = lane == 0 ? S[j + c * kChunk] : 0.0;
      for (int i = j + 1 + lane; i < r; i += 32) dot = fma(S[i + j * kChunk], S[i + c * kChunk], dot);
      dot = warp_sum(dot);
      if (lane == 0) wv[c] = dot * t;
    }
    __syncthreads();
    // trailing update, one thread per row (no index division)
    if (tid >= j && tid < r) {
      const double vi = (tid == j) ? 1.0 : S[tid + j * kChunk];
      for (int c = j + 1; c < w; ++c) S[tid + c * kChunk] -= vi * wv[c];
    }
    __syncthreads();
  }

  // R (w x w): upper triangle of the first k rows
  for (int e = tid; e < w * w; e += kQT) {
    const int i = e % w, c = e / w;
    D.R[i + (long long)c * D.ldr] = (i <= c && i < k) ? S[i + c * kChunk] : 0.0;
  }
  // explicit Q = H_0 ... H_{k-1} [I; 0]
  for (int e = tid; e < kChunk * kPanel; e += kQT) {
    const int i = e % kChunk, c = e / kChunk;
    E[e] = (i == c && i < r && c < w) ? 1.0 : 0.0;
  }
  __syncthreads();
  for (int j = k - 1; j >= 0; --j) {
    const double t = tau[j];
    for (int c = j + warp; c < w; c += kQT / 32) {
      double dot = lane == 0 ? E[j + c * kChunk] : 0.0;
      for (int i = j + 1 + lane; i < r; i += 32) dot = fma(S[i + j * kChunk], E[i + c * kChunk], dot);
      dot = warp_sum(dot);
      if (lane == 0) wv[c] = dot * t;
    }
    __syncthreads();
    if (tid >= j && tid < r) {
      const double vi = (tid == j) ? 1.0 : S[tid + j * kChunk];
      for (int c = j; c < w; ++c) E[tid + c * kChunk] -= vi * wv[c];
    }
    __syncthreads();
  }
  for (int e = tid; e < r * w; e += kQT) {
    const int i = e % r, c = e / r;
    D.A[i + (long long)c * D.lda] = E[i + c * kChunk];
  }
}

// Q (rows x w) <- Q M (M: w x w)
__global__ void __launch_bounds__(kQT) mul_chunk_kernel(const MulChunk *__restrict__ descs) {
  const MulChunk D = descs[blockIdx.x];
  __shared__ double M[kPanel * kPanel];
  const int tid = threadIdx.x, w = D.w;
  for (int e = tid; e < w * w; e += kQT) M[e] = D.M[(e % w) + (long long)(e / w) * D.ldm];
  __syncthreads();
  for (int i = tid; i < D.rows; i += kQT) {
    double q[kPanel];
#pragma unroll
    for (int l = 0; l < kPanel; ++l) q[l] = l < w ? D.Q[i + (long long)l * D.ldq] : 0.0;
    for (int c = 0; c < w; ++c) {
      double acc = 0.0;
#pragma unroll
      for (int l = 0; l < kPanel; ++l) acc = fma(q[l], l < w ? M[l + c * w] : 0.0, acc);
      D.Q[i + (long long)c * D.ldq] = acc;
    }
  }
}

__device__ __forceinline__ unsigned long long splitmix64(unsigned long long x) {
  x += 0x9E3779B97F4A7C15ULL;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
  return x ^ (x >> 31);
}

__global__ void gaussian_kernel(const RandDesc *__restrict__ descs, unsigned long long seed) {
  const RandDesc D = descs[blockIdx.y];
  const unsigned long long base = splitmix64(seed ^ splitmix64(D.id + 0x632BE59BD9B4E019ULL));
  const long long total = (long long)D.rows * D.cols;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const unsigned long long h1 = splitmix64(base + (unsigned long long)e);
    const unsigned long long h2 = splitmix64(h1);
    const double u1 = ((double)(h1 >> 11) + 1.0) * 0x1.0p-53;   // (0, 1]
    const double u2 = (double)(h2 >> 11) * 0x1.0p-53;           // [0, 1)
    const double z = sqrt(-2.0 * log(u1)) * cospi(2.0 * u2);
    const long long i = e % D.rows, j = e / D.rows;
    D.X[i + j * D.ld] = z;
  }
}

__global__ void colnorm_kernel(const NormDesc *__restrict__ descs) {
  const NormDesc D = descs[blockIdx.y];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int c = blockIdx.x * nw + warp; c < D.cols; c += gridDim.x * nw) {
    const double *x = D.X + (long long)c * D.ld;
    double s = 0.0;
    for (int i = lane; i < D.rows; i += 32) s = fma(x[i], x[i], s);
    s = warp_sum(s);
    if (lane == 0) D.out[c] = s;
  }
}

template <class T>
T *upload(const std::vector<T> &v, cudaStream_t s) {
  T *d = nullptr;
  HB_CUDA(cudaMallocAsync((void **)&d, sizeof(T) * std::max<size_t>(v.size(), 1), s));
  h2d_async(d, v.data(), sizeof(T) * v.size(), s);
  return d;
}

__global__ void panel_clean_kernel(const CleanDesc *__restrict__ descs, double rel) {
  const CleanDesc D = descs[blockIdx.y];
  double scale2 = 0.0;
  for (int c = 0; c < D.w; ++c) scale2 = fmax(scale2, D.prenorm2[c]);
  const double thr = rel * sqrt(scale2);
  for (int c = 0; c < D.w; ++c) {
    if (fabs(D.R[c + (long long)c * D.ldr]) > thr) continue;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < D.rows; i += gridDim.x * blockDim.x)
      D.Q[i + (long long)c * D.ldq] = 0.0;
  }
}

}  // namespace

void panel_clean(const std::vector<CleanDesc> &descs, double rel, cudaStream_t s) {
  if (descs.empty()) return;
  CleanDesc *d = upload(descs, s);
  for (size_t off = 0; off < descs.size(); off += 65535) {
    dim3 grid(8, (unsigned)std::min<size_t>(65535, descs.size() - off));
    panel_clean_kernel<<<grid, 256, 0, s>>>(d + off, rel);
    HB_LAUNCHED();
  }
  cudaFreeAsync(d, s);
}

// The chunk lists of every level of a batch of TSQR problems, uploaded, with
// the scratch of the stacked R factors: made once, run any number of times
// (the panels' contents may change between runs, not their addresses).
struct TsqrPlan {
  std::vector<QrChunk *> up;        // per level: QR of the chunks
  std::vector<int> up_n;
  std::vector<MulChunk *> down;     // per level (top first): Q times the parent's Q
  std::vector<int> down_n;
  double *buf = nullptr;
  cudaStream_t stream = nullptr;
  ~TsqrPlan() {
    for (auto *p : up) cudaFreeAsync(p, stream);
    for (auto *p : down) cudaFreeAsync(p, stream);
    if (buf) cudaFreeAsync(buf, stream);
  }
};

void TsqrPlanDeleter::operator()(TsqrPlan *p) const { delete p; }

std::unique_ptr<TsqrPlan, TsqrPlanDeleter> tsqr_plan(const std::vector<TsqrProb> &probs,
                                                     cudaStream_t s) {
  struct Clock {
    std::chrono::steady_clock::time_point t = std::chrono::steady_clock::now();
    ~Clock() {
      plan_host_ms() +=
          std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t).count();
    }
  } clock;
  std::unique_ptr<TsqrPlan, TsqrPlanDeleter> plan(new TsqrPlan);
  plan->stream = s;
  if (probs.empty()) return plan;
  // level structure of every problem: level 0 is the panel itself, level
  // l + 1 stacks the w x w R factors of level l's chunks
  struct Level {
    double *A;
    long long lda;
    int rows;
    int nchunks;
  };
  // levels of problem p: lev[lo[p] .. lo[p + 1]) (flat, no per-problem
  // allocations: a round of the build makes plans for thousands of panels)
  constexpr int kMaxLevels = 16;
  std::vector<Level> lev;
  std::vector<int> lo(probs.size() + 1, 0);
  lev.reserve(probs.size() * 3);
  long long scratch = 0;
  std::vector<long long> stack_off;   // per level >= 1, same indexing as lev
  stack_off.reserve(probs.size() * 3);
  for (size_t p = 0; p < probs.size(); ++p) {
    const TsqrProb &P = probs[p];
    HB_REQUIRE(P.w >= 1 && P.w <= kPanel, INPUT_ERROR, "TSQR panel wider than 32 columns");
    lo[p] = (int)lev.size();
    int rows = P.m;
    long long off = -1;   // stacked-R scratch of this level (-1: the panel itself)
    for (int l = 0; l < kMaxLevels; ++l) {
      const int nch = std::max(1, (rows + kChunk - 1) / kChunk);
      lev.push_back(Level{nullptr, 0, rows, nch});
      stack_off.push_back(off);
      if (nch == 1) break;
      rows = nch * P.w;
      off = scratch;
      scratch += align_up((long long)rows * P.w);
    }
  }
  lo[probs.size()] = (int)lev.size();
  if (scratch) HB_CUDA(cudaMallocAsync((void **)&plan->buf, scratch * sizeof(double), s));
  int max_levels = 0;
  for (size_t p = 0; p < probs.size(); ++p) {
    Level *L = lev.data() + lo[p];
    const int nl = lo[p + 1] - lo[p];
    L[0].A = probs[p].Y;
    L[0].lda = probs[p].ldy;
    for (int l = 1; l < nl; ++l) {
      L[l].A = plan->buf + stack_off[lo[p] + l];
      L[l].lda = L[l].rows;
    }
    max_levels = std::max(max_levels, nl);
  }
  // up-sweep
  for (int l = 0; l < max_levels; ++l) {
    std::vector<QrChunk> chunks;
    for (size_t p = 0; p < probs.size(); ++p) {
      const Level *L = lev.data() + lo[p];
      const int nl = lo[p + 1] - lo[p];
      if (l >= nl) continue;
      const int w = probs[p].w;
      for (int c = 0; c < L[l].nchunks; ++c) {
        QrChunk q;
        q.A = L[l].A + (long long)c * kChunk;
        q.lda = L[l].lda;
        q.rows = std::min(kChunk, L[l].rows - c * kChunk);
        q.w = w;
        if (l + 1 < nl) {
          q.R = L[l + 1].A + (long long)c * w;
          q.ldr = L[l + 1].lda;
        } else {
          q.R = probs[p].R;
          q.ldr = probs[p].ldr;
        }
        if (q.rows > 0) chunks.push_back(q);
      }
    }
    plan->up.push_back(chunks.empty() ? nullptr : upload(chunks, s));
    plan->up_n.push_back((int)chunks.size());
  }
  // down-sweep: every chunk's Q times its block of the parent's Q
  for (int l = max_levels - 2; l >= 0; --l) {
    std::vector<MulChunk> chunks;
    for (size_t p = 0; p < probs.size(); ++p) {
      const Level *L = lev.data() + lo[p];
      const int nl = lo[p + 1] - lo[p];
      if (l + 1 >= nl) continue;
      const int w = probs[p].w;
      for (int c = 0; c < L[l].nchunks; ++c) {
        MulChunk mc;
        mc.Q = L[l].A + (long long)c * kChunk;
        mc.ldq = L[l].lda;
        mc.rows = std::min(kChunk, L[l].rows - c * kChunk);
        mc.w = w;
        mc.M = L[l + 1].A + (long long)c * w;
        mc.ldm = L[l + 1].lda;
        if (mc.rows > 0) chunks.push_back(mc);
      }
    }
    plan->down.push_back(chunks.empty() ? nullptr : upload(chunks, s));
    plan->down_n.push_back((int)chunks.size());
  }
  return plan;
}

void tsqr_run(const TsqrPlan &plan, cudaStream_t s) {
  static bool configured = false;
  if (!configured) {
    HB_CUDA(cudaFuncSetAttribute(qr_chunk_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)kQrSmem));
    configured = true;
  }
  for (size_t l = 0; l < plan.up.size(); ++l)
    for (int off = 0; off < plan.up_n[l]; off += 65535) {
      const int cnt = std::min(65535, plan.up_n[l] - off);
      qr_chunk_kernel<<<cnt, kQT, kQrSmem, s>>>(plan.up[l] + off);
      HB_LAUNCHED();
    }
  for (size_t l = 0; l < plan.down.size(); ++l)
    for (int off = 0; off < plan.down_n[l]; off += 65535) {
      const int cnt = std::min(65535, plan.down_n[l] - off);
      mul_chunk_kernel<<<cnt, kQT, 0, s>>>(plan.down[l] + off);
      HB_LAUNCHED();
    }
}

void tsqr_batched(const std::vector<TsqrProb> &probs, cudaStream_t s) {
  if (probs.empty()) return;
  auto plan = tsqr_plan(probs, s);
  tsqr_run(*plan, s);
}

void gaussian_fill(const std::vector<RandDesc> &descs, unsigned long long seed, cudaStream_t s) {
  if (descs.empty()) return;
  RandDesc *d = upload(descs, s);
  for (size_t off = 0; off < descs.size(); off += 65535) {
    dim3 grid(64, (unsigned)std::min<size_t>(65535, descs.size() - off));
    gaussian_kernel<<<grid, 256, 0, s>>>(d + off, seed);
    HB_LAUNCHED();
  }
  cudaFreeAsync(d, s);
}

void column_norms2(const std::vector<NormDesc> &descs, cudaStream_t s) {
  if (descs.empty()) return;
  NormDesc *d = upload(descs, s);
  for (size_t off = 0; off < descs.size(); off += 65535) {
    dim3 grid(8, (unsigned)std::min<size_t>(65535, descs.size() - off));
    colnorm_kernel<<<grid, 256, 0, s>>>(d + off);
    HB_LAUNCHED();
  }
  cudaFreeAsync(d, s);
}

}  // namespace hb
