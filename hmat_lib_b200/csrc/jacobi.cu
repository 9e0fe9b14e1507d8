// Batched one-sided (Hestenes) Jacobi SVD in FP64, one CTA per problem, or a
// cluster of CTAs per wide problem.
//
// Replaces the LAPACK dgesdd calls of hmat_lib (src/lapack_wrapper.c:8-59
// via src/constructors.c:323 for compression; src/hodlr_algebra.c:153 and
// :301 for recompression) on blocks small enough for one CTA.  Columns of the
// tall orientation are orthogonalised pairwise in round-robin order: each
// round pairs every column with one other (C/2 disjoint pairs, one warp per
// pair), so a sweep is C-1 rounds separated by barriers.  The singular
// values come out with high relative accuracy, so the relative truncation
// rule picks the same rank as the reference's dgesdd on its test matrices.
// Every loop is bounded: a problem that has not converged after max_sweeps
// sweeps still writes its outputs and raises SVD_FAILURE in the status word.
#include <algorithm>

#include <cooperative_groups.h>

#include "jacobi.h"

namespace cg = cooperative_groups;

namespace hb {

namespace {

constexpr int kJThreads = 256;
constexpr int kJCluster = 8;        // CTAs per problem cluster
constexpr int kJUnroll = 8;         // column elements per lane in flight in the pair loops

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Global loads and stores of G and W.  A problem solved by a cluster of CTAs
// reads columns that other CTAs of the cluster rotated in the previous round,
// so it bypasses L1 (cache-global) and relies on the cluster barrier's
// release / acquire ordering at L2.
template <bool kTeam>
__device__ __forceinline__ double gld(const double *p) {
  if constexpr (kTeam) return __ldcg(p);
  return *p;
}
template <bool kTeam>
__device__ __forceinline__ void gst(double *p, double v) {
  if constexpr (kTeam)
    __stcg(p, v);
  else
    *p = v;
}

template <bool kTeam>
__device__ __forceinline__ void team_sync() {
  if constexpr (kTeam)
    cg::this_cluster().sync();
  else
    __syncthreads();
}

// (x, y) <- (c x - s y, s x + c y) over `len` elements, the warp's lanes
// striding by 32, eight elements per lane in flight.
template <bool kTeam>
__device__ __forceinline__ void rotate_pair(double *xp, double *yp, int len, int lane, double cs,
                                            double sn) {
  for (int i0 = lane; i0 < len; i0 += 32 * kJUnroll) {
    double x[kJUnroll], y[kJUnroll];
#pragma unroll
    for (int u = 0; u < kJUnroll; ++u) {
      const int i = i0 + 32 * u;
      x[u] = i < len ? gld<kTeam>(xp + i) : 0.0;
      y[u] = i < len ? gld<kTeam>(yp + i) : 0.0;
    }
#pragma unroll
    for (int u = 0; u < kJUnroll; ++u) {
      const int i = i0 + 32 * u;
      if (i < len) {
        gst<kTeam>(xp + i, cs * x[u] - sn * y[u]);
        gst<kTeam>(yp + i, sn * x[u] + cs * y[u]);
      }
    }
  }
}

// One problem, by one CTA (kTeam false) or by the kJCluster CTAs of a
// cluster (kTeam true, `crank` = this CTA's rank in it): the disjoint pairs
// of a round are spread over every warp of the team, rounds are separated by
// a barrier of the team, and the team agrees on convergence through the
// CTAs' shared memory.  Every pair's arithmetic is the same in both modes.
template <bool kTeam>
__device__ void jacobi_solve(const JacobiProb &P, const JacobiParams &prm, int *status,
                             int crank, int team, const KernelSpec &gen) {
  const int m = P.m, n = P.n;
  const bool tall = m >= n;
  const int R = tall ? m : n, C = tall ? n : m;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5;
  extern __shared__ double sh[];
  double *s_sig = sh;                              // C
  int *s_perm = reinterpret_cast<int *>(sh + C);   // C
  __shared__ double s_off[32];
  __shared__ double s_team_off;

  double *G = P.G, *W = P.W;
  const int gtid = crank * blockDim.x + tid, gthreads = team * blockDim.x;
  double fro2 = 0.0;   // this thread's share of ||A||_F^2
  for (long long e = gtid; e < (long long)R * C; e += gthreads) {
    const int r = (int)(e % R), c = (int)(e / R);
    // logical element (i, j) of the m x n input
    const int i = tall ? r : c, j = tall ? c : r;
    double a;
    if (P.gen_r0 >= 0)
      a = P.transA ? kernel_entry(gen, P.gen_r0 + j, P.gen_c0 + i)
                   : kernel_entry(gen, P.gen_r0 + i, P.gen_c0 + j);
    else
      a = P.transA ? P.A[j + (long long)i * P.lda] : P.A[i + (long long)j * P.lda];
    fro2 = fma(a, a, fro2);
    gst<kTeam>(G + e, a);
  }
  for (long long e = gtid; e < (long long)C * C; e += gthreads)
    gst<kTeam>(W + e, ((e % C) == (e / C)) ? 1.0 : 0.0);
  team_sync<kTeam>();

  // ||A||_F over the team
  fro2 = warp_sum(fro2);
  if (lane == 0) s_off[warp] = fro2;
  __syncthreads();
  double f2 = 0.0;
  for (int w = 0; w < nwarps; ++w) f2 += s_off[w];
  if constexpr (kTeam) {
    cg::cluster_group cl = cg::this_cluster();
    if (tid == 0) s_team_off = f2;
    cl.sync();
    f2 = 0.0;
    for (int rk = 0; rk < team; ++rk) f2 += *cl.map_shared_rank(&s_team_off, rk);
    cl.sync();
  }
  __syncthreads();
  // Pairs with a column of norm below theta are neither rotated nor tested:
  // all such columns together hold at most sqrt(C) theta = 1e-3 tol s_0 of the
  // matrix (||A||_F / C <= s_0 / sqrt(C) for the relative rule), so no
  // singular value moves by more than 0.1% of the truncation threshold
  // (Weyl) and none of theirs reaches it.  Columns at rounding level otherwise
  // keep the sweeps going: their computed cosines with any column are
  // rounding noise.  No skipping when every singular value is kept.
  double theta = 0.0;
  if (prm.trunc == Truncation::Relative)
    theta = 1e-3 * prm.tol * sqrt(f2) / C;
  else if (prm.trunc == Truncation::Absolute)
    theta = 1e-3 * prm.tol / sqrt((double)C);
  theta = fmax(theta, P.skip_abs);
  const double skip2 = theta * theta;
  const double cscale = P.conv_scale > 0.0 ? P.conv_scale : (prm.norm_stop ? sqrt(f2) : 0.0);

  // a computed dot product of length R carries ~sqrt(R) eps relative noise:
  // below that no rotation can make progress
  const double conv = fmax(prm.conv_tol, 4.0 * sqrt((double)R) * 2.220446049250313e-16);
  const int players = C + (C & 1);
  const int gwarp = crank * nwarps + warp, gwarps = team * nwarps;
  int sweep = 0;
  bool converged = (C == 1);
  for (; sweep < prm.max_sweeps && !converged; ++sweep) {
    double off = 0.0;
    for (int r = 0; r < players - 1; ++r) {
      for (int k = gwarp; k < players / 2; k += gwarps) {
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
        // eight elements per lane in flight, the last chunk predicated (each
        // sum keeps the element order of a plain loop: arithmetic unchanged)
        double al = 0.0, be = 0.0, ga = 0.0;
        for (int i0 = lane; i0 < R; i0 += 32 * kJUnroll) {
          double x[kJUnroll], y[kJUnroll];
#pragma unroll
          for (int u = 0; u < kJUnroll; ++u) {
            const int i = i0 + 32 * u;
            x[u] = i < R ? gld<kTeam>(gp + i) : 0.0;
            y[u] = i < R ? gld<kTeam>(gq + i) : 0.0;
          }
#pragma unroll
          for (int u = 0; u < kJUnroll; ++u)
            if (i0 + 32 * u < R) {
              al = fma(x[u], x[u], al);
              be = fma(y[u], y[u], be);
              ga = fma(x[u], y[u], ga);
            }
        }
        al = warp_sum(al);
        be = warp_sum(be);
        ga = warp_sum(ga);
        if (ga == 0.0 || al <= 0.0 || be <= 0.0) continue;
        if (al <= skip2 || be <= skip2) continue;
        double rel = fabs(ga) / (sqrt(al) * sqrt(be));
        // coupling at rounding level of the problem's own scale (a block of a
        // larger matrix, whose columns were recomputed by a GEMM) counts as
        // converged: it moves no singular value by more than that level
        if (cscale > 0.0) rel = fmin(rel, fabs(ga) / (cscale * fmax(sqrt(al), sqrt(be))));
        off = fmax(off, rel);
        if (rel <= conv) continue;
        const double zeta = (be - al) / (2.0 * ga);
        // tan of the rotation angle; for |zeta| beyond 1e100 zeta^2 would
        // overflow and the exact value is 1 / (2 zeta) to double precision
        const double t = fabs(zeta) > 1e100
                             ? 0.5 / zeta
                             : (zeta >= 0.0 ? 1.0 : -1.0) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
        const double cs = 1.0 / sqrt(1.0 + t * t), sn = cs * t;
        rotate_pair<kTeam>(gp, gq, R, lane, cs, sn);
        rotate_pair<kTeam>(W + (long long)p * C, W + (long long)q * C, C, lane, cs, sn);
      }
      team_sync<kTeam>();
    }
    // team-wide max of `off`
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) off = fmax(off, __shfl_xor_sync(0xffffffffu, off, o));
    if (lane == 0) s_off[warp] = off;
    __syncthreads();
    double mx = 0.0;
    for (int w = 0; w < nwarps; ++w) mx = fmax(mx, s_off[w]);
    if constexpr (kTeam) {
      // every CTA reads every CTA's maximum, so all take the same decision;
      // the second barrier keeps every CTA (and its shared memory) alive and
      // unchanged until all reads are done
      cg::cluster_group cl = cg::this_cluster();
      if (tid == 0) s_team_off = mx;
      cl.sync();
      mx = 0.0;
      for (int rk = 0; rk < team; ++rk) mx = fmax(mx, *cl.map_shared_rank(&s_team_off, rk));
      cl.sync();
    }
    converged = mx <= conv;
    __syncthreads();
  }
  if (crank != 0) return;
  if (!converged && tid == 0) atomicExch(status, (int)SVD_FAILURE);
  if (tid == 0 && P.sweeps) *P.sweeps = converged ? sweep : prm.max_sweeps + 1;

  // singular values = column norms of G
  for (int j = warp; j < C; j += nwarps) {
    const double *gj = G + (long long)j * R;
    double s = 0.0;
    for (int i = lane; i < R; i += 32) {
      const double x = gld<kTeam>(gj + i);
      s = fma(x, x, s);
    }
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
        double x = gld<kTeam>(gj + i);
        if (!prm.scale_u) x = sg > 0.0 ? x / sg : (i == k % m ? 1.0 : 0.0);
        u[i] = x;
      }
      for (int i = lane; i < n; i += 32) v[i] = gld<kTeam>(wj + i);
    } else {     // A^T = (G / sigma) Sigma W^T  =>  A = W Sigma (G / sigma)^T
      for (int i = lane; i < m; i += 32) {
        const double x = gld<kTeam>(wj + i);
        u[i] = prm.scale_u ? x * sg : x;
      }
      for (int i = lane; i < n; i += 32) {
        const double x = gld<kTeam>(gj + i);
        v[i] = sg > 0.0 ? x / sg : (i == k % n ? 1.0 : 0.0);
      }
    }
  }
}

// One CTA per problem.
__global__ void __launch_bounds__(kJThreads)
jacobi_svd_kernel(const JacobiProb *__restrict__ probs, JacobiParams prm, int *status,
                  KernelSpec gen) {
  const JacobiProb P = probs[blockIdx.x];
  const int C = P.m < P.n ? P.m : P.n;
  if (C == 0) {
    if (threadIdx.x == 0 && P.rank) *P.rank = 0;
    return;
  }
  jacobi_solve<false>(P, prm, status, 0, 1, gen);
}

// A cluster of kJCluster CTAs per problem; problems with at least
// `team_min_c` columns are solved by the whole cluster, the others by its
// first CTA alone (the rest return at once, before any cluster barrier).
__global__ void __cluster_dims__(kJCluster, 1, 1) __launch_bounds__(kJThreads)
jacobi_svd_cluster_kernel(const JacobiProb *__restrict__ probs, JacobiParams prm, int *status,
                          int team_min_c, KernelSpec gen) {
  const int crank = (int)cg::this_cluster().block_rank();
  const JacobiProb P = probs[blockIdx.x / kJCluster];
  const int C = P.m < P.n ? P.m : P.n;
  if (C == 0) {
    if (crank == 0 && threadIdx.x == 0 && P.rank) *P.rank = 0;
    return;
  }
  if (C >= team_min_c) {
    jacobi_solve<true>(P, prm, status, crank, kJCluster, gen);
  } else {
    if (crank != 0) return;
    jacobi_solve<false>(P, prm, status, 0, 1, gen);
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
                        int *d_status, int max_c, cudaStream_t stream, const KernelSpec &gen) {
  if (nprobs <= 0) return;
  const size_t smem = (size_t)std::max(max_c, 1) * (sizeof(double) + sizeof(int));
  HB_REQUIRE(smem <= 200 * 1024, INPUT_ERROR, "Jacobi SVD problem too wide for one CTA");
  // launches whose widest problem reaches team_min_c columns give every
  // problem a cluster of CTAs; the others one CTA
  const int team_min_c = (int)std::min(option("jacobi_cluster_min_c", 192.0), 1e9);
  if (max_c >= team_min_c) {
    if (smem > 48 * 1024)
      HB_CUDA(cudaFuncSetAttribute(jacobi_svd_cluster_kernel,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    jacobi_svd_cluster_kernel<<<nprobs * kJCluster, kJThreads, smem, stream>>>(
        d_probs, prm, d_status, team_min_c, gen);
  } else {
    if (smem > 48 * 1024)
      HB_CUDA(cudaFuncSetAttribute(jacobi_svd_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)smem));
    jacobi_svd_kernel<<<nprobs, kJThreads, smem, stream>>>(d_probs, prm, d_status, gen);
  }
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
