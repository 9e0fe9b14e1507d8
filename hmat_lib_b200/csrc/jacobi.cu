// Batched one-sided (Hestenes) Jacobi SVD in FP64, one CTA per problem.
//
// Replaces the LAPACK dgesdd calls of hmat_lib (src/lapack_wrapper.c:8-59
// via src/constructors.c:323 for compression; src/hodlr_algebra.c:153 and
// :301 for recompression) on blocks small enough for one CTA.  Columns of the
// tall orientation are orthogonalised pairwise in round-robin order: each
// round pairs every column with one other (C/2 disjoint pairs, one warp per
// pair), so a sweep is C-1 rounds separated by __syncthreads.  The singular
// values come out with high relative accuracy, so the relative truncation
// rule picks the same rank as the reference's dgesdd on its test matrices.
// Every loop is bounded: a problem that has not converged after max_sweeps
// sweeps still writes its outputs and raises SVD_FAILURE in the status word.
#include <algorithm>

#include "jacobi.h"

namespace hb {

namespace {

constexpr int kJThreads = 256;

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__global__ void __launch_bounds__(kJThreads)
jacobi_svd_kernel(const JacobiProb *__restrict__ probs, JacobiParams prm, int *status) {
  const JacobiProb P = probs[blockIdx.x];
  const int m = P.m, n = P.n;
  const bool tall = m >= n;
  const int R = tall ? m : n, C = tall ? n : m;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5;
  extern __shared__ double sh[];
  double *s_sig = sh;                              // C
  int *s_perm = reinterpret_cast<int *>(sh + C);   // C
  __shared__ double s_off[32];

  if (C == 0) {
    if (tid == 0 && P.rank) *P.rank = 0;
    return;
  }
  double *G = P.G, *W = P.W;
  for (long long e = tid; e < (long long)R * C; e += blockDim.x) {
    const int r = (int)(e % R), c = (int)(e / R);
    // logical element (i, j) of the m x n input
    const int i = tall ? r : c, j = tall ? c : r;
    G[e] = P.transA ? P.A[j + (long long)i * P.lda] : P.A[i + (long long)j * P.lda];
  }
  for (long long e = tid; e < (long long)C * C; e += blockDim.x)
    W[e] = ((e % C) == (e / C)) ? 1.0 : 0.0;
  __syncthreads();

  // a computed dot product of length R carries ~sqrt(R) eps relative noise:
  // below that no rotation can make progress
  const double conv = fmax(prm.conv_tol, 4.0 * sqrt((double)R) * 2.220446049250313e-16);
  const int players = C + (C & 1);
  int sweep = 0;
  bool converged = (C == 1);
  for (; sweep < prm.max_sweeps && !converged; ++sweep) {
    double off = 0.0;
    for (int r = 0; r < players - 1; ++r) {
      for (int k = warp; k < players / 2; k += nwarps) {
        int a, b;
        if (k == 0) {
          a = r;
          b = players - 1;
        } else {
          a = (r + k) % (players - 1);
          b = (r - k + (players - 1)) % (players - 1);
        }
        if (a >= C || b >= C) continue;
        const int p = min(a, b), q = max(a, b);
        double *gp = G + (long long)p * R, *gq = G + (long long)q * R;
        double al = 0.0, be = 0.0, ga = 0.0;
        for (int i = lane; i < R; i += 32) {
          const double x = gp[i], y = gq[i];
          al = fma(x, x, al);
          be = fma(y, y, be);
          ga = fma(x, y, ga);
        }
        al = warp_sum(al);
        be = warp_sum(be);
        ga = warp_sum(ga);
        if (ga == 0.0 || al <= 0.0 || be <= 0.0) continue;
        const double rel = fabs(ga) / (sqrt(al) * sqrt(be));
        off = fmax(off, rel);
        if (rel <= conv) continue;
        const double zeta = (be - al) / (2.0 * ga);
        // tan of the rotation angle; for |zeta| beyond 1e100 zeta^2 would
        // overflow and the exact value is 1 / (2 zeta) to double precision
        const double t = fabs(zeta) > 1e100
                             ? 0.5 / zeta
                             : (zeta >= 0.0 ? 1.0 : -1.0) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
        const double cs = 1.0 / sqrt(1.0 + t * t), sn = cs * t;
        for (int i = lane; i < R; i += 32) {
          const double x = gp[i], y = gq[i];
          gp[i] = cs * x - sn * y;
          gq[i] = sn * x + cs * y;
        }
        double *wp = W + (long long)p * C, *wq = W + (long long)q * C;
        for (int i = lane; i < C; i += 32) {
          const double x = wp[i], y = wq[i];
          wp[i] = cs * x - sn * y;
          wq[i] = sn * x + cs * y;
        }
      }
      __syncthreads();
    }
    // block-wide max of `off`
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) off = fmax(off, __shfl_xor_sync(0xffffffffu, off, o));
    if (lane == 0) s_off[warp] = off;
    __syncthreads();
    double mx = 0.0;
    for (int w = 0; w < nwarps; ++w) mx = fmax(mx, s_off[w]);
    converged = mx <= conv;
    __syncthreads();
  }
  if (!converged && tid == 0) atomicExch(status, (int)SVD_FAILURE);
  if (tid == 0 && P.sweeps) *P.sweeps = converged ? sweep : prm.max_sweeps + 1;

  // singular values = column norms of G
  for (int j = warp; j < C; j += nwarps) {
    const double *gj = G + (long long)j * R;
    double s = 0.0;
    for (int i = lane; i < R; i += 32) s = fma(gj[i], gj[i], s);
    s = warp_sum(s);
    if (lane == 0) s_sig[j] = sqrt(s);
  }
  __syncthreads();
  // descending order, ties by index (stable)
  for (int j = tid; j < C; j += blockDim.x) {
    const double sj = s_sig[j];
    int pos = 0;
    for (int i = 0; i < C; ++i) {
      const double si = s_sig[i];
      pos += (si > sj) || (si == sj && i < j);
    }
    s_perm[pos] = j;
  }
  __syncthreads();
  if (tid == 0) {
    const double s0 = s_sig[s_perm[0]];
    int k = 1;
    if (prm.trunc == Truncation::Relative) {
      if (s0 > prm.tol)
        while (k < C && s_sig[s_perm[k]] >= prm.tol * s0) ++k;
    } else if (prm.trunc == Truncation::Absolute) {
      while (k < C && s_sig[s_perm[k]] > prm.tol) ++k;
    } else {
      k = C;
    }
    if (P.rank) *P.rank = k;
  }
  for (int k = tid; k < C; k += blockDim.x)
    if (P.sigma) P.sigma[k] = s_sig[s_perm[k]];
  // outputs, one warp per column
  for (int k = warp; k < C; k += nwarps) {
    const int j = s_perm[k];
    const double sg = s_sig[j];
    const double *gj = G + (long long)j * R;
    const double *wj = W + (long long)j * C;
    double *u = P.U + (long long)k * P.ldu;
    double *v = P.V + (long long)k * P.ldv;
    if (tall) {  // A = (G / sigma) Sigma W^T
      for (int i = lane; i < m; i += 32) {
        double x = gj[i];
        if (!prm.scale_u) x = sg > 0.0 ? x / sg : (i == k % m ? 1.0 : 0.0);
        u[i] = x;
      }
      for (int i = lane; i < n; i += 32) v[i] = wj[i];
    } else {     // A^T = (G / sigma) Sigma W^T  =>  A = W Sigma (G / sigma)^T
      for (int i = lane; i < m; i += 32) u[i] = prm.scale_u ? wj[i] * sg : wj[i];
      for (int i = lane; i < n; i += 32) v[i] = sg > 0.0 ? gj[i] / sg : (i == k % n ? 1.0 : 0.0);
    }
  }
}

__global__ void copy2d_kernel(const CopyDesc *__restrict__ descs) {
  const CopyDesc D = descs[blockIdx.y];
  const long long total = (long long)D.rows * D.cols;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const long long r = e % D.rows, c = e / D.rows;
    D.dst[r + c * D.ldd] = D.src[r + c * D.lds];
  }
}

__global__ void add2d_kernel(const CopyDesc *__restrict__ descs, double alpha) {
  const CopyDesc D = descs[blockIdx.y];
  const long long total = (long long)D.rows * D.cols;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const long long r = e % D.rows, c = e / D.rows;
    D.dst[r + c * D.ldd] += alpha * D.src[r + c * D.lds];
  }
}

}  // namespace

void jacobi_svd_batched(const JacobiProb *d_probs, int nprobs, const JacobiParams &prm,
                        int *d_status, int max_c, cudaStream_t stream) {
  if (nprobs <= 0) return;
  const size_t smem = (size_t)std::max(max_c, 1) * (sizeof(double) + sizeof(int));
  HB_REQUIRE(smem <= 200 * 1024, INPUT_ERROR, "Jacobi SVD problem too wide for one CTA");
  if (smem > 48 * 1024)
    HB_CUDA(cudaFuncSetAttribute(jacobi_svd_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem));
  jacobi_svd_kernel<<<nprobs, kJThreads, smem, stream>>>(d_probs, prm, d_status);
  HB_LAUNCHED();
}

void copy2d_batched(const CopyDesc *d_descs, int n, cudaStream_t stream) {
  if (n <= 0) return;
  for (int off = 0; off < n; off += 65535) {
    dim3 grid(32, std::min(65535, n - off));
    copy2d_kernel<<<grid, 256, 0, stream>>>(d_descs + off);
    HB_LAUNCHED();
  }
}

}  // namespace hb

namespace hb {
void add2d_batched(const CopyDesc *d_descs, int n, double alpha, cudaStream_t stream) {
  if (n <= 0) return;
  for (int off = 0; off < n; off += 65535) {
    dim3 grid(32, std::min(65535, n - off));
    add2d_kernel<<<grid, 256, 0, stream>>>(d_descs + off, alpha);
    HB_LAUNCHED();
  }
}
}  // namespace hb
