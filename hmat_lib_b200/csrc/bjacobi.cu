// Block one-sided Jacobi SVD (see bjacobi.h).
//
// Per problem, one workspace holds X (the columns being orthogonalised,
// L x Lp, Lp = L rounded up to whole 32-column blocks, padding columns zero)
// and V (the accumulated right rotations, Lp x Lp).  A round is ONE launch of
// bj_pair_kernel for every pair of every active problem: a cluster of CTAs
// per pair of blocks (64 columns), each CTA owning a slice of the rows.
//   1. Gram matrix of the pair, G = X_pair^T X_pair (64 x 64), on the FP64
//      tensor cores (mma m8n8k4), each CTA over its rows, then summed over the
//      cluster through distributed shared memory in rank order, so every CTA
//      of the cluster holds the same G bit for bit;
//   2. if some column pair of G is coupled above the convergence test, every
//      CTA solves G = W diag W^T by cyclic two-sided Jacobi in shared memory
//      (the same arithmetic in every CTA, so the same W) and sorts the
//      eigenvalues in descending order;
//   3. X[:, pair] = X[:, pair] W and V[:, pair] = V[:, pair] W over its rows
//      (mma m8n8k4 again), in place: a warp loads a whole 8-row strip before
//      it writes it, and strips of different warps and CTAs are disjoint.
// Rotations act on the columns themselves (no re-factorisation of a pair), so
// small columns keep their relative accuracy; the rotation is applied only
// when the pair needs it, so the late sweeps are mostly Gram passes.
// Round r of a sweep pairs blocks as the round-robin tournament does (block
// players - 1 fixed, the others rotating), so a sweep of players - 1 rounds
// pairs every block with every other once.  All active problems advance one
// round per launch: problem p is in round g mod (players_p - 1) of global
// round g.
#include <cooperative_groups.h>

#include <algorithm>
#include <cmath>
#include <numeric>

#include "bjacobi.h"
#include "dtree.h"
#include "jacobi.h"
#include "tsqr.h"

namespace cg = cooperative_groups;

namespace hb {

namespace {

constexpr int kBj = 32;          // columns per block
constexpr int kPair = 2 * kBj;   // columns per pair
constexpr int kLd = 68;          // leading dimension of the 64 x 64 tiles in shared memory
constexpr int kPT = 256;         // threads of the pair kernel (8 warps)
constexpr int kInner = 30;       // sweeps of a pair's eigensolver at most (option bj_inner_sweeps)
constexpr int kT = 32;           // transpose tile
constexpr int kMaxCluster = 8;

template <class T>
T *upload_vec(const std::vector<T> &v, cudaStream_t s) {
  T *d = nullptr;
  HB_CUDA(cudaMallocAsync((void **)&d, sizeof(T) * std::max<size_t>(v.size(), 1), s));
  if (!v.empty())
    h2d_async(d, v.data(), sizeof(T) * v.size(), s);
  return d;
}

// dst[i + j ldd] = src[j + i lds] for i, j < n (32 x 32 tiles through shared
// memory, one padding column against bank conflicts)
__global__ void bj_transpose_kernel(const double *__restrict__ src, long long lds, int n,
                                    double *__restrict__ dst, long long ldd) {
  __shared__ double tile[kT][kT + 1];
  const int i0 = blockIdx.x * kT, j0 = blockIdx.y * kT;
  const int tx = threadIdx.x, ty = threadIdx.y;   // 32 x 8 threads
  // tile[jj][ii] = src[(j0 + ii) + (i0 + jj) lds]: coalesced along ii
  for (int jj = ty; jj < kT; jj += 8)
    if (i0 + jj < n && j0 + tx < n) tile[jj][tx] = src[(j0 + tx) + (long long)(i0 + jj) * lds];
  __syncthreads();
  // dst[(i0 + ii) + (j0 + jj) ldd] = src[(j0 + jj) + (i0 + ii) lds] = tile[ii][jj]
  for (int jj = ty; jj < kT; jj += 8)
    if (i0 + tx < n && j0 + jj < n) dst[(i0 + tx) + (long long)(j0 + jj) * ldd] = tile[tx][jj];
}

__global__ void bj_identity_kernel(double *__restrict__ v, long long ld, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    v[i + (long long)i * ld] = 1.0;
}

// Blocks (a, b), a < b, of pair k in round r of a round-robin over `players` (even).
__host__ __device__ inline void round_pair(int k, int r, int players, int &a, int &b) {
  if (k == 0) {
    a = r;
    b = players - 1;
  } else {
    a = (r + k) % (players - 1);
    b = (r - k + (players - 1)) % (players - 1);
  }
  if (a > b) {
    const int t = a;
    a = b;
    b = t;
  }
}

struct BjDev {
  double *X, *V;   // L x Lp (ld L), Lp x Lp (ld Lp)
  int L, Lp, nblk, players;
  double theta2;   // columns of squared norm at or below this are not rotated
  double fro;      // ||A||_F, the scale of the norm-relative convergence test
  double conv;     // convergence threshold of a column pair
  int *rot;        // set when a pair of the problem rotated in the current sweep
};

// Shared memory of the pair kernel; element (i, j) of a 64 x 64 tile at i + j kLd.
struct PairSmem {
  double gp[kPair * kLd];   // this CTA's partial Gram (tiles I <= J), later W with sorted columns
  double g[kPair * kLd];    // the pair's Gram, rotated in place by the eigensolver
  double w[kPair * kLd];    // accumulated rotations
  double cs[kPair / 2], sn[kPair / 2], tn[kPair / 2];
  int pp[kPair / 2], qq[kPair / 2];
  int perm[kPair];
  int flag[2];   // a rotation in the inner sweep of that parity
  int work;      // the pair failed the convergence test
};

__device__ __forceinline__ void dmma(double (&c)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(c[0]), "+d"(c[1])
               : "d"(a), "d"(b));
}

// The test of a column pair with squared norms al, be and product ga: true
// when it must be rotated.  Columns at or below theta are neither rotated nor
// tested (all of them together hold at most sqrt(L) theta = 1e-3 tol ||A||_F
// / sqrt(L) of the matrix: no kept singular value moves by more than 0.1% of
// the truncation threshold).  A coupling at rounding level of the problem's
// own scale counts as converged: a column recomputed from others carries an
// error of about eps ||A|| times its weight, which no rotation removes.
__device__ __forceinline__ bool needs_rotation(double al, double be, double ga, double theta2,
                                               double fro, double conv) {
  if (ga == 0.0 || al <= theta2 || be <= theta2) return false;
  const double sa = sqrt(al), sb = sqrt(be);
  const double rel = fmin(fabs(ga) / (sa * sb), fabs(ga) / (fro * fmax(sa, sb)));
  return rel > conv;
}

// X[rs:re, pair] = X[rs:re, pair] Wp (ld = rows of X, pair columns at xa, xb)
// by warps over 8-row strips; Wp in shared memory.
__device__ __forceinline__ void rotate_rows(double *xa, double *xb, long long ld, int rs, int re,
                                            const double *wp, int warp, int gq, int tq) {
  for (int r0 = rs + 8 * warp; r0 < re; r0 += 8 * (kPT / 32)) {
    const int row = r0 + gq;
    const bool in = row < re;
    double a[kPair / 4];
#pragma unroll
    for (int kk = 0; kk < kPair / 4; ++kk) {
      const int k = 4 * kk + tq;
      const double *src = (k < kBj ? xa + (long long)k * ld : xb + (long long)(k - kBj) * ld);
      a[kk] = in ? src[row] : 0.0;
    }
#pragma unroll
    for (int nt = 0; nt < kPair / 8; ++nt) {
      double c[2] = {0.0, 0.0};
#pragma unroll
      for (int kk = 0; kk < kPair / 4; ++kk) dmma(c, a[kk], wp[(4 * kk + tq) + (8 * nt + gq) * kLd]);
      if (in) {
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int j = 8 * nt + 2 * tq + h;
          double *dst = (j < kBj ? xa + (long long)j * ld : xb + (long long)(j - kBj) * ld);
          dst[row] = c[h];
        }
      }
    }
  }
}

// One round for every pair slot: blockIdx.x / cluster size = slot.
__global__ void __launch_bounds__(kPT, 1)
bj_pair_kernel(const BjDev *__restrict__ probs, const int2 *__restrict__ slots, long long g_round,
               int inner_max) {
  extern __shared__ __align__(16) unsigned char bj_smem_raw[];
  PairSmem &S = *reinterpret_cast<PairSmem *>(bj_smem_raw);
  cg::cluster_group cl = cg::this_cluster();
  const int ncl = (int)cl.num_blocks();
  const int crank = (int)cl.block_rank();
  const int2 sl = slots[blockIdx.x / ncl];
  const BjDev P = probs[sl.x];
  int a, b;
  round_pair(sl.y, (int)(g_round % (P.players - 1)), P.players, a, b);
  if (b >= P.nblk) return;   // the bye of an odd block count (the whole cluster)

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int gq = lane >> 2, tq = lane & 3;
  const long long L = P.L, Lp = P.Lp;
  double *xa = P.X + (long long)a * kBj * L, *xb = P.X + (long long)b * kBj * L;
  double *va = P.V + (long long)a * kBj * Lp, *vb = P.V + (long long)b * kBj * Lp;
  const int xchunk = ((P.L + ncl - 1) / ncl + 7) / 8 * 8;
  const int xr0 = min(P.L, crank * xchunk), xr1 = min(P.L, xr0 + xchunk);
  const int vchunk = ((P.Lp + ncl - 1) / ncl + 7) / 8 * 8;
  const int vr0 = min(P.Lp, crank * vchunk), vr1 = min(P.Lp, vr0 + vchunk);

  // ---- 1. Gram of this CTA's rows: warps take 4-row steps in turn, each
  // holding the 36 tiles I <= J of the 8 x 8 tiling (column j of the pair is
  // fragment j / 8, lane row j % 8)
  {
    const double *col[8];
#pragma unroll
    for (int I = 0; I < 8; ++I)
      col[I] = (I < 4 ? xa + (long long)(8 * I + gq) * L : xb + (long long)(8 * (I - 4) + gq) * L);
    double acc[36][2];
#pragma unroll
    for (int t = 0; t < 36; ++t) acc[t][0] = acc[t][1] = 0.0;
    double f[8], nf[8];
    int r = xr0 + 4 * warp;
#pragma unroll
    for (int I = 0; I < 8; ++I) f[I] = (r + tq < xr1) ? col[I][r + tq] : 0.0;
    for (; r < xr1; r += 4 * (kPT / 32)) {
      const int rn = r + 4 * (kPT / 32) + tq;
#pragma unroll
      for (int I = 0; I < 8; ++I) nf[I] = (rn < xr1) ? col[I][rn] : 0.0;
      int t = 0;
#pragma unroll
      for (int I = 0; I < 8; ++I)
#pragma unroll
        for (int J = I; J < 8; ++J) dmma(acc[t++], f[I], f[J]);
#pragma unroll
      for (int I = 0; I < 8; ++I) f[I] = nf[I];
    }
    // warps add their sums into gp in warp order (deterministic)
    for (int w = 0; w < kPT / 32; ++w) {
      if (warp == w) {
        int t = 0;
#pragma unroll
        for (int I = 0; I < 8; ++I)
#pragma unroll
          for (int J = I; J < 8; ++J) {
#pragma unroll
            for (int h = 0; h < 2; ++h) {
              double &e = S.gp[(8 * I + gq) + (8 * J + 2 * tq + h) * kLd];
              e = (w == 0 ? 0.0 : e) + acc[t][h];
            }
            ++t;
          }
      }
      __syncthreads();
    }
  }
  // ---- the cluster's sum, in rank order, into every CTA's g (symmetric:
  // element (i, j) from the stored (min, max))
  if (ncl > 1) cl.sync();
  for (int e = tid; e < kPair * kPair; e += kPT) {
    const int i = e % kPair, j = e / kPair;
    const int off = min(i, j) + max(i, j) * kLd;
    double s = 0.0;
    if (ncl == 1) {
      s = S.gp[off];
    } else {
      for (int rk = 0; rk < ncl; ++rk) s += *cl.map_shared_rank(S.gp + off, rk);
    }
    S.g[i + j * kLd] = s;
  }
  if (tid == 0) {
    S.work = 0;
    S.flag[0] = S.flag[1] = 0;
  }
  // after this barrier no CTA reads another's gp any more
  if (ncl > 1) cl.sync();
  __syncthreads();

  // ---- 2. convergence test of the pair, then the eigensolver
  for (int e = tid; e < kPair * kPair; e += kPT) {
    const int i = e % kPair, j = e / kPair;
    if (i < j && needs_rotation(S.g[i + i * kLd], S.g[j + j * kLd], S.g[i + j * kLd], P.theta2,
                                P.fro, P.conv))
      S.work = 1;
  }
  for (int e = tid; e < kPair * kPair; e += kPT) {
    const int i = e % kPair, j = e / kPair;
    S.w[i + j * kLd] = (i == j) ? 1.0 : 0.0;
  }
  __syncthreads();
  if (!S.work) return;   // the same decision in every CTA of the cluster

  for (int sweep = 0; sweep < inner_max; ++sweep) {
    for (int step = 0; step < kPair - 1; ++step) {
      if (tid < kPair / 2) {
        int p, q;
        round_pair(tid, step, kPair, p, q);
        const double app = S.g[p + p * kLd], aqq = S.g[q + q * kLd], apq = S.g[p + q * kLd];
        double c = 1.0, s = 0.0, t = 0.0;
        if (needs_rotation(app, aqq, apq, P.theta2, P.fro, P.conv)) {
          // x_p' = c x_p - s x_q, x_q' = s x_p + c x_q zeroes the pair's
          // product; t = tan of the smaller angle (1 / (2 zeta) beyond 1e100,
          // where zeta^2 would overflow)
          const double zeta = (aqq - app) / (2.0 * apq);
          t = fabs(zeta) > 1e100 ? 0.5 / zeta
                                 : (zeta >= 0.0 ? 1.0 : -1.0) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
          c = 1.0 / sqrt(1.0 + t * t);
          s = c * t;
          S.flag[sweep & 1] = 1;
        }
        S.pp[tid] = p;
        S.qq[tid] = q;
        S.cs[tid] = c;
        S.sn[tid] = s;
        S.tn[tid] = t;
      }
      __syncthreads();
      // the previous sweep's flag was read before this step's barrier
      if (step == 0 && tid == 0) S.flag[(sweep + 1) & 1] = 0;
      // G = J^T G J over the 2 x 2 blocks of pairs (K, M), K <= M, both halves
      for (int e = tid; e < (kPair / 2) * (kPair / 2); e += kPT) {
        const int K = e % (kPair / 2), M = e / (kPair / 2);
        if (K > M) continue;
        const double sK = S.sn[K], sM = S.sn[M];
        if (sK == 0.0 && sM == 0.0) continue;
        const int pK = S.pp[K], qK = S.qq[K];
        if (K == M) {
          const double tK = S.tn[K], apq = S.g[pK + qK * kLd];
          S.g[pK + pK * kLd] -= tK * apq;
          S.g[qK + qK * kLd] += tK * apq;
          S.g[pK + qK * kLd] = 0.0;
          S.g[qK + pK * kLd] = 0.0;
          continue;
        }
        const double cK = S.cs[K], cM = S.cs[M];
        const int pM = S.pp[M], qM = S.qq[M];
        const double b00 = S.g[pK + pM * kLd], b01 = S.g[pK + qM * kLd];
        const double b10 = S.g[qK + pM * kLd], b11 = S.g[qK + qM * kLd];
        // rows: J_K^T B
        const double r00 = cK * b00 - sK * b10, r01 = cK * b01 - sK * b11;
        const double r10 = sK * b00 + cK * b10, r11 = sK * b01 + cK * b11;
        // columns: (J_K^T B) J_M
        const double n00 = cM * r00 - sM * r01, n01 = sM * r00 + cM * r01;
        const double n10 = cM * r10 - sM * r11, n11 = sM * r10 + cM * r11;
        S.g[pK + pM * kLd] = n00;
        S.g[pK + qM * kLd] = n01;
        S.g[qK + pM * kLd] = n10;
        S.g[qK + qM * kLd] = n11;
        S.g[pM + pK * kLd] = n00;
        S.g[qM + pK * kLd] = n01;
        S.g[pM + qK * kLd] = n10;
        S.g[qM + qK * kLd] = n11;
      }
      // W = W J
      for (int e = tid; e < kPair * (kPair / 2); e += kPT) {
        const int i = e % kPair, K = e / kPair;
        const double sK = S.sn[K];
        if (sK == 0.0) continue;
        const double cK = S.cs[K];
        double &wp = S.w[i + S.pp[K] * kLd];
        double &wq = S.w[i + S.qq[K] * kLd];
        const double x = wp, y = wq;
        wp = cK * x - sK * y;
        wq = sK * x + cK * y;
      }
      __syncthreads();
    }
    if (!S.flag[sweep & 1]) break;
  }

  // ---- sort the eigenvalues in descending order (ties by index); the
  // sorted W into gp
  if (tid < kPair) {
    const double d = S.g[tid + tid * kLd];
    int pos = 0;
    for (int j = 0; j < kPair; ++j) {
      const double dj = S.g[j + j * kLd];
      pos += (dj > d || (dj == d && j < tid)) ? 1 : 0;
    }
    S.perm[pos] = tid;
  }
  __syncthreads();
  for (int e = tid; e < kPair * kPair; e += kPT) {
    const int i = e % kPair, j = e / kPair;
    S.gp[i + j * kLd] = S.w[i + S.perm[j] * kLd];
  }
  if (crank == 0 && tid == 0) *P.rot = 1;
  __syncthreads();

  // ---- 3. the rotation of this CTA's rows of X and V
  rotate_rows(xa, xb, L, xr0, xr1, S.gp, warp, gq, tq);
  rotate_rows(va, vb, Lp, vr0, vr1, S.gp, warp, gq, tq);
}

// The integer outputs of one problem.
struct BjIntOut {
  int *rank, *sweeps;
  int r, sw;
};

__global__ void bj_int_out_kernel(const BjIntOut *__restrict__ o, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    *o[i].rank = o[i].r;
    if (o[i].sweeps) *o[i].sweeps = o[i].sw;
  }
}

struct Work {
  int L = 0, Lp = 0, nblk = 0, players = 0, npairs = 0;
  long long x = 0, v = 0;
  int sweep = 0;
  bool active = true, converged = false;
};

}  // namespace

void block_jacobi_svd(const std::vector<BjProb> &probs, double tol, int max_sweeps,
                      int *d_status, cudaStream_t s) {
  const int np = (int)probs.size();
  if (np == 0) return;
  // ---- layout ------------------------------------------------------------------------
  std::vector<Work> wk(np);
  long long total = 0;
  auto take = [&](long long e) {
    const long long o = total;
    total += align_up(std::max<long long>(e, 1));
    return o;
  };
  int lmax = 0;
  for (int p = 0; p < np; ++p) {
    Work &W = wk[p];
    W.L = probs[p].L;
    HB_REQUIRE(W.L >= kPair, INPUT_ERROR, "block Jacobi SVD: problem narrower than 64 columns");
    W.Lp = (W.L + kBj - 1) / kBj * kBj;
    W.nblk = W.Lp / kBj;
    W.players = W.nblk + (W.nblk & 1);
    W.npairs = W.players / 2;
    W.x = take((long long)W.L * W.Lp);
    W.v = take((long long)W.Lp * W.Lp);
    lmax = std::max(lmax, W.L);
  }
  std::vector<long long> noff(np);   // squared column norms of X
  for (int p = 0; p < np; ++p) noff[p] = take(wk[p].Lp);
  double *w = dev_alloc(total, s);
  HB_CUDA(cudaMemsetAsync(w, 0, sizeof(double) * total, s));
  int *d_rot = nullptr;   // per problem: a pair rotated in this sweep
  HB_CUDA(cudaMallocAsync((void **)&d_rot, sizeof(int) * np, s));
  HB_CUDA(cudaMemsetAsync(d_rot, 0, sizeof(int) * np, s));
  // ---- X = A^T, V = I, thresholds -------------------------------------------------------
  std::vector<NormDesc> nd;
  for (int p = 0; p < np; ++p) {
    const Work &W = wk[p];
    dim3 grid((W.L + kT - 1) / kT, (W.L + kT - 1) / kT);
    bj_transpose_kernel<<<grid, dim3(kT, 8), 0, s>>>(probs[p].A, probs[p].lda, W.L, w + W.x, W.L);
    HB_LAUNCHED();
    bj_identity_kernel<<<(W.Lp + 255) / 256, 256, 0, s>>>(w + W.v, W.Lp, W.Lp);
    HB_LAUNCHED();
    nd.push_back(NormDesc{w + W.x, W.L, W.L, W.Lp, w + noff[p]});
  }
  column_norms2(nd, s);
  // a column pair of length L recomputed by a 64-term sum is orthogonal to
  // about sqrt(L) eps
  const double conv = 8.0 * std::sqrt((double)lmax) * 2.220446049250313e-16;
  // the column norms of every problem lie in one range of the workspace:
  // read them in one copy
  const long long n_lo = noff[0], n_hi = noff[np - 1] + wk[np - 1].Lp;
  std::vector<double> hn((size_t)(n_hi - n_lo));
  auto read_norms = [&]() {
    HB_CUDA(cudaMemcpyAsync(hn.data(), w + n_lo, sizeof(double) * (n_hi - n_lo),
                            cudaMemcpyDeviceToHost, s));
    HB_CUDA(cudaStreamSynchronize(s));
  };
  std::vector<BjDev> hd(np);
  {
    read_norms();
    for (int p = 0; p < np; ++p) {
      double f2 = 0.0;
      for (int c = 0; c < wk[p].Lp; ++c) f2 += hn[noff[p] - n_lo + c];
      const Work &W = wk[p];
      // the scalar solver's skip rule for the relative truncation
      const double theta = 1e-3 * tol * std::sqrt(f2) / W.L;
      hd[p] = BjDev{w + W.x, w + W.v, W.L, W.Lp, W.nblk, W.players, theta * theta,
                    std::sqrt(f2), conv, d_rot + p};
    }
  }
  BjDev *d_probs = upload_vec(hd, s);
  std::vector<int> rot(np, 0);

  // A pair's eigensolver may stop before it converges: its rotation is still
  // orthogonal, and the outer sweeps finish the job.
  const int inner_max = std::max(1, std::min(kInner, (int)option("bj_inner_sweeps", kInner)));
  int dev = 0, nsm = 148;
  HB_CUDA(cudaGetDevice(&dev));
  HB_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  const size_t smem = sizeof(PairSmem);
  HB_CUDA(cudaFuncSetAttribute(bj_pair_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)smem));

  // The pair slots of the active problems and the cluster size (CTAs per
  // pair: as many as keep one wave of CTAs on the SMs, at most 8, and at
  // least 64 rows per CTA); made again when a problem leaves.
  int2 *d_slots = nullptr;
  int nslots = 0, ncl = 1;
  auto make_slots = [&]() {
    std::vector<int2> sl;
    int lmin = 1 << 30;
    for (int p = 0; p < np; ++p) {
      if (!wk[p].active) continue;
      for (int k = 0; k < wk[p].npairs; ++k) sl.push_back(make_int2(p, k));
      lmin = std::min(lmin, wk[p].L);
    }
    nslots = (int)sl.size();
    ncl = std::max(1, std::min({kMaxCluster, nsm / std::max(nslots, 1), lmin / 64}));
    if (d_slots) cudaFreeAsync(d_slots, s);
    d_slots = upload_vec(sl, s);
  };
  make_slots();

  // ---- rounds ------------------------------------------------------------------------------
  for (long long g = 0;; ++g) {
    bool any = false;
    for (const Work &W : wk) any = any || W.active;
    if (!any) break;
    {
      cudaLaunchConfig_t cfg = {};
      cfg.gridDim = dim3((unsigned)(nslots * ncl));
      cfg.blockDim = dim3(kPT);
      cfg.dynamicSmemBytes = smem;
      cfg.stream = s;
      cudaLaunchAttribute attr[1];
      attr[0].id = cudaLaunchAttributeClusterDimension;
      attr[0].val.clusterDim.x = (unsigned)ncl;
      attr[0].val.clusterDim.y = 1;
      attr[0].val.clusterDim.z = 1;
      cfg.attrs = attr;
      cfg.numAttrs = 1;
      HB_CUDA(cudaLaunchKernelEx(&cfg, bj_pair_kernel, (const BjDev *)d_probs,
                                 (const int2 *)d_slots, g, inner_max));
      HB_LAUNCHED();
    }
    // end of a sweep of some problem: a problem whose sweep rotated nothing
    // has converged
    bool check = false;
    for (const Work &W : wk)
      if (W.active && (g + 1) % (W.players - 1) == 0) check = true;
    if (!check) continue;
    HB_CUDA(cudaMemcpyAsync(rot.data(), d_rot, sizeof(int) * np, cudaMemcpyDeviceToHost, s));
    HB_CUDA(cudaStreamSynchronize(s));
    bool changed = false;
    for (int p = 0; p < np; ++p) {
      Work &W = wk[p];
      if (!W.active || (g + 1) % (W.players - 1) != 0) continue;
      ++W.sweep;
      if (!rot[p]) {
        W.active = false;
        W.converged = true;
        changed = true;
      } else if (W.sweep >= max_sweeps) {
        W.active = false;
        changed = true;
      } else {
        HB_CUDA(cudaMemsetAsync(d_rot + p, 0, sizeof(int), s));
      }
    }
    if (changed) make_slots();
  }
  if (d_slots) cudaFreeAsync(d_slots, s);
  cudaFreeAsync(d_probs, s);

  // ---- singular values, order, rank, outputs -------------------------------------------
  nd.clear();
  for (int p = 0; p < np; ++p) nd.push_back(NormDesc{w + wk[p].x, wk[p].L, wk[p].L, wk[p].Lp,
                                                     w + noff[p]});
  column_norms2(nd, s);
  std::vector<CopyDesc> gather;
  std::vector<std::vector<double>> sig(np);
  std::vector<int> ranks(np), sweeps(np);
  read_norms();
  for (int p = 0; p < np; ++p) {
    const Work &W = wk[p];
    const std::vector<double> n2(hn.begin() + (noff[p] - n_lo),
                                 hn.begin() + (noff[p] - n_lo) + W.Lp);
    std::vector<int> perm(W.Lp);
    std::iota(perm.begin(), perm.end(), 0);
    std::stable_sort(perm.begin(), perm.end(), [&](int a, int b) { return n2[a] > n2[b]; });
    sig[p].resize(W.L);
    for (int c = 0; c < W.L; ++c) sig[p][c] = std::sqrt(std::max(n2[perm[c]], 0.0));
    const double s0 = sig[p][0];
    int r = 1;
    if (s0 > tol)
      while (r < W.L && sig[p][r] >= tol * s0) ++r;
    ranks[p] = r;
    sweeps[p] = W.converged ? W.sweep : max_sweeps + 1;
    for (int c = 0; c < W.L; ++c) {
      gather.push_back(CopyDesc{w + W.x + (long long)perm[c] * W.L, W.L,
                                probs[p].U + (long long)c * W.L, W.L, W.L, 1});
      gather.push_back(CopyDesc{w + W.v + (long long)perm[c] * W.Lp, W.Lp,
                                probs[p].V + (long long)c * W.L, W.L, W.L, 1});
    }
  }
  CopyDesc *dg = upload_vec(gather, s);
  copy2d_batched(dg, (int)gather.size(), s);
  cudaFreeAsync(dg, s);
  // singular values (one upload, scattered by one copy launch), ranks and
  // sweeps (one launch)
  bool failed = false;
  {
    std::vector<double> hs;
    std::vector<long long> so(np);
    for (int p = 0; p < np; ++p) {
      so[p] = (long long)hs.size();
      hs.insert(hs.end(), sig[p].begin(), sig[p].end());
    }
    double *ds = upload_vec(hs, s);
    std::vector<CopyDesc> sc;
    std::vector<BjIntOut> io;
    for (int p = 0; p < np; ++p) {
      sc.push_back(CopyDesc{ds + so[p], wk[p].L, probs[p].sigma, wk[p].L, wk[p].L, 1});
      io.push_back(BjIntOut{probs[p].rank, probs[p].sweeps, ranks[p], sweeps[p]});
      failed = failed || !wk[p].converged;
    }
    CopyDesc *dsc = upload_vec(sc, s);
    copy2d_batched(dsc, (int)sc.size(), s);
    BjIntOut *dio = upload_vec(io, s);
    bj_int_out_kernel<<<(np + 127) / 128, 128, 0, s>>>(dio, np);
    HB_LAUNCHED();
    cudaFreeAsync(dsc, s);
    cudaFreeAsync(dio, s);
    cudaFreeAsync(ds, s);
  }
  if (failed) {
    const int st = SVD_FAILURE;
    HB_CUDA(cudaMemcpyAsync(d_status, &st, sizeof(int), cudaMemcpyHostToDevice, s));
    set_last_error("block Jacobi SVD of a sketch core did not converge within "
                   "jacobi_max_sweeps sweeps");
  }
  HB_CUDA(cudaStreamSynchronize(s));
  cudaFreeAsync(d_rot, s);
  dev_free(w, s);
}

}  // namespace hb
