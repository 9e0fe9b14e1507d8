// Block one-sided Jacobi SVD (see bjacobi.h).
//
// Per problem, one workspace holds X (the columns being orthogonalised,
// L x Lp, Lp = L rounded up to whole 16-column blocks, padding columns zero),
// V (the accumulated right rotations, Lp x Lp), and per pair of blocks a
// 32-column panel, a copy of the pair's V columns, R, the Jacobi workspace
// and its outputs.  A round, for every problem at once:
//   1. copy the pair's X columns into its panel and its V columns aside;
//   2. TSQR of every panel: panel = Q R (Q written over the panel);
//   3. one-sided Jacobi SVD of every R: R = (U_R Sigma) W^T, sorted;
//   4. X[:, pair] = Q (U_R Sigma), V[:, pair] = V_old[:, pair] W, and a pair
//      whose Jacobi rotated anything marks its problem (one update launch).
// The TSQR plan and the Jacobi problems of the pair slots are made once per
// set of active problems; a round only uploads its copy and update
// descriptors.
// Round r of a sweep pairs blocks as the round-robin tournament does (block
// players - 1 fixed, the others rotating), so a sweep of players - 1 rounds
// pairs every block with every other once.
#include <algorithm>
#include <cmath>
#include <numeric>

#include "bjacobi.h"
#include "dtree.h"
#include "jacobi.h"
#include "tsqr.h"

namespace hb {

namespace {

constexpr int kBj = 16;          // columns per block
constexpr int kPair = 2 * kBj;   // columns per pair: one TSQR panel
constexpr int kT = 32;           // transpose tile

template <class T>
T *upload_vec(const std::vector<T> &v, cudaStream_t s) {
  T *d = nullptr;
  HB_CUDA(cudaMallocAsync((void **)&d, sizeof(T) * std::max<size_t>(v.size(), 1), s));
  if (!v.empty())
    HB_CUDA(cudaMemcpyAsync(d, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice, s));
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

// One pair's update: X[:, a | b] = P (U_R Sigma) with P the pair's Q (L x 32),
// V[:, a | b] = T W with T the pair's old V columns (Lp x 32); 64 rows and 32
// columns per CTA (a thread: one row, eight columns), the two 32 x 32 factors
// in shared memory.  The first CTA of a pair also marks the problem when the
// pair's Jacobi SVD rotated anything (more than its first, checking sweep).
struct BjUpdate {
  const double *P, *T, *JU, *JV;
  double *xa, *xb, *va, *vb;
  int L, Lp;
  const int *sweeps;
  int *rotated;
};

__global__ void __launch_bounds__(256) bj_update_kernel(const BjUpdate *__restrict__ ups) {
  const BjUpdate U = ups[blockIdx.y];
  __shared__ double ju[kPair * kPair], jv[kPair * kPair];
  for (int e = threadIdx.x; e < kPair * kPair; e += blockDim.x) {
    ju[e] = U.JU[e];
    jv[e] = U.JV[e];
  }
  __syncthreads();
  if (blockIdx.x == 0 && threadIdx.x == 0 && *U.sweeps > 1) *U.rotated = 1;
  const int row = blockIdx.x * 64 + (threadIdx.x & 63), g = threadIdx.x >> 6;   // columns 8g..8g+7
  if (row < U.L) {
    double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int k = 0; k < kPair; ++k) {
      const double pk = U.P[row + (long long)k * U.L];
#pragma unroll
      for (int c = 0; c < 8; ++c) acc[c] = fma(pk, ju[k + (8 * g + c) * kPair], acc[c]);
    }
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      const int col = 8 * g + c;
      double *dst = col < kBj ? U.xa + (long long)col * U.L : U.xb + (long long)(col - kBj) * U.L;
      dst[row] = acc[c];
    }
  }
  if (row < U.Lp) {
    double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int k = 0; k < kPair; ++k) {
      const double tk = U.T[row + (long long)k * U.Lp];
#pragma unroll
      for (int c = 0; c < 8; ++c) acc[c] = fma(tk, jv[k + (8 * g + c) * kPair], acc[c]);
    }
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      const int col = 8 * g + c;
      double *dst = col < kBj ? U.va + (long long)col * U.Lp : U.vb + (long long)(col - kBj) * U.Lp;
      dst[row] = acc[c];
    }
  }
}

// Blocks (a, b) of pair k in round r of a round-robin over `players` (even).
void round_pair(int k, int r, int players, int &a, int &b) {
  if (k == 0) {
    a = r;
    b = players - 1;
  } else {
    a = (r + k) % (players - 1);
    b = (r - k + (players - 1)) % (players - 1);
  }
  if (a > b) std::swap(a, b);
}

struct Work {
  int L = 0, Lp = 0, nblk = 0, players = 0, npairs = 0;
  long long x = 0, v = 0, pnl = 0, tmp = 0, r = 0, jw = 0, ju = 0, jv = 0, js = 0;
  int slot0 = 0;          // first pair slot of this problem
  int round = 0, sweep = 0;
  bool active = true, converged = false;
  double theta = 0.0;     // column norms at or below this are not rotated
  double fro = 0.0;       // ||A||_F
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
  const long long jws = jacobi_workspace(kPair, kPair);
  int nslots = 0, lmax = 0;
  for (int p = 0; p < np; ++p) {
    Work &W = wk[p];
    W.L = probs[p].L;
    HB_REQUIRE(W.L >= kPair, INPUT_ERROR, "block Jacobi SVD: problem narrower than 32 columns");
    W.Lp = (W.L + kBj - 1) / kBj * kBj;
    W.nblk = W.Lp / kBj;
    W.players = W.nblk + (W.nblk & 1);
    W.npairs = W.players / 2;
    W.x = take((long long)W.L * W.Lp);
    W.v = take((long long)W.Lp * W.Lp);
    W.pnl = take((long long)W.npairs * W.L * kPair);
    W.tmp = take((long long)W.npairs * W.Lp * kPair);
    W.r = take((long long)W.npairs * kPair * kPair);
    W.jw = take((long long)W.npairs * jws);
    W.ju = take((long long)W.npairs * kPair * kPair);
    W.jv = take((long long)W.npairs * kPair * kPair);
    W.js = take((long long)W.npairs * kPair);
    W.slot0 = nslots;
    nslots += W.npairs;
    lmax = std::max(lmax, W.L);
  }
  std::vector<long long> noff(np);   // squared column norms of X
  for (int p = 0; p < np; ++p) noff[p] = take(wk[p].Lp);
  double *w = dev_alloc(total, s);
  HB_CUDA(cudaMemsetAsync(w, 0, sizeof(double) * total, s));
  int *d_ints = nullptr;   // per slot: rank, sweeps; per problem: rotated flag
  HB_CUDA(cudaMallocAsync((void **)&d_ints, sizeof(int) * (2 * nslots + np), s));
  HB_CUDA(cudaMemsetAsync(d_ints, 0, sizeof(int) * (2 * nslots + np), s));
  int *d_rank = d_ints, *d_sw = d_ints + nslots;
  int *d_rot = d_ints + 2 * nslots;
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
  {
    std::vector<double> h;
    for (int p = 0; p < np; ++p) {
      h.resize(wk[p].Lp);
      HB_CUDA(cudaMemcpyAsync(h.data(), w + noff[p], sizeof(double) * wk[p].Lp,
                              cudaMemcpyDeviceToHost, s));
      HB_CUDA(cudaStreamSynchronize(s));
      double f2 = 0.0;
      for (double v : h) f2 += v;
      // the scalar solver's skip rule for the relative truncation
      wk[p].theta = 1e-3 * tol * std::sqrt(f2) / wk[p].L;
      wk[p].fro = std::sqrt(f2);
    }
  }
  JacobiParams prm;
  prm.trunc = Truncation::None;
  prm.scale_u = 1;
  prm.max_sweeps = 60;
  // a recomputed column pair of length L is orthogonal to about sqrt(L) eps
  prm.conv_tol = 8.0 * std::sqrt((double)lmax) * 2.220446049250313e-16;
  std::vector<int> rot(np, 0);

  // The TSQR plan and the Jacobi problems cover every pair slot of every
  // active problem; they depend only on the slots' addresses, so they are
  // made once per set of active problems.  A slot whose pair is a bye this
  // round computes on stale values that nothing reads.
  std::unique_ptr<TsqrPlan, TsqrPlanDeleter> tplan;
  JacobiProb *d_jp = nullptr;
  int njp = 0;
  auto make_plans = [&]() {
    std::vector<TsqrProb> tq;
    std::vector<JacobiProb> jp;
    for (int p = 0; p < np; ++p) {
      const Work &W = wk[p];
      if (!W.active) continue;
      for (int k = 0; k < W.npairs; ++k) {
        const long long pk = W.pnl + (long long)k * W.L * kPair;
        const long long rk = W.r + (long long)k * kPair * kPair;
        tq.push_back(TsqrProb{w + pk, W.L, W.L, kPair, w + rk, kPair});
        JacobiProb j{};
        j.A = w + rk;
        j.lda = kPair;
        j.transA = 0;
        j.m = kPair;
        j.n = kPair;
        j.G = w + W.jw + (long long)k * jws;
        j.W = j.G + align_up((long long)kPair * kPair);
        j.U = w + W.ju + (long long)k * kPair * kPair;
        j.ldu = kPair;
        j.V = w + W.jv + (long long)k * kPair * kPair;
        j.ldv = kPair;
        j.sigma = w + W.js + (long long)k * kPair;
        j.rank = d_rank + W.slot0 + k;
        j.sweeps = d_sw + W.slot0 + k;
        j.skip_abs = W.theta;
        // A pair's columns are recomputed every round, so a large and a small
        // column keep a coupling of about eps ||A|| ||large||; such pairs
        // count as orthogonal (singular values then carry an absolute error
        // of that order, far below the truncation threshold tol ||A||),
        // otherwise sweeps would never end.
        j.conv_scale = W.fro;
        jp.push_back(j);
      }
    }
    tplan = tsqr_plan(tq, s);
    if (d_jp) cudaFreeAsync(d_jp, s);
    d_jp = upload_vec(jp, s);
    njp = (int)jp.size();
  };
  make_plans();
  int lpmax = 0;
  for (const Work &W : wk) lpmax = std::max(lpmax, W.Lp);

  // ---- rounds ------------------------------------------------------------------------------
  for (long long guard = 0; guard < 1000000; ++guard) {
    bool any = false;
    for (const Work &W : wk) any = any || W.active;
    if (!any) break;
    std::vector<CopyDesc> cp;
    std::vector<BjUpdate> up;
    for (int p = 0; p < np; ++p) {
      const Work &W = wk[p];
      if (!W.active) continue;
      const long long L = W.L, Lp = W.Lp;
      for (int k = 0; k < W.npairs; ++k) {
        int a, b;
        round_pair(k, W.round, W.players, a, b);
        if (b >= W.nblk) continue;   // the bye of an odd block count
        const long long pk = W.pnl + (long long)k * L * kPair;
        const long long tk = W.tmp + (long long)k * Lp * kPair;
        double *xa = w + W.x + (long long)a * kBj * L, *xb = w + W.x + (long long)b * kBj * L;
        double *va = w + W.v + (long long)a * kBj * Lp, *vb = w + W.v + (long long)b * kBj * Lp;
        cp.push_back(CopyDesc{xa, L, w + pk, L, (int)L, kBj});
        cp.push_back(CopyDesc{xb, L, w + pk + kBj * L, L, (int)L, kBj});
        cp.push_back(CopyDesc{va, Lp, w + tk, Lp, (int)Lp, kBj});
        cp.push_back(CopyDesc{vb, Lp, w + tk + kBj * Lp, Lp, (int)Lp, kBj});
        up.push_back(BjUpdate{w + pk, w + tk, w + W.ju + (long long)k * kPair * kPair,
                              w + W.jv + (long long)k * kPair * kPair, xa, xb, va, vb, (int)L,
                              (int)Lp, d_sw + W.slot0 + k, d_rot + p});
      }
    }
    if (!cp.empty()) {
      CopyDesc *d = upload_vec(cp, s);
      copy2d_batched(d, (int)cp.size(), s);
      cudaFreeAsync(d, s);
      tsqr_run(*tplan, s);
      jacobi_svd_batched(d_jp, njp, prm, d_status, kPair, s);
      BjUpdate *du = upload_vec(up, s);
      for (size_t o = 0; o < up.size(); o += 65535) {
        dim3 grid((lpmax + 63) / 64, (unsigned)std::min<size_t>(65535, up.size() - o));
        bj_update_kernel<<<grid, 256, 0, s>>>(du + o);
        HB_LAUNCHED();
      }
      cudaFreeAsync(du, s);
    }
    // end of a sweep: a problem whose sweep rotated nothing has converged
    bool check = false;
    for (Work &W : wk) {
      if (!W.active) continue;
      if (++W.round == W.players - 1) check = true;
    }
    if (!check) continue;
    HB_CUDA(cudaMemcpyAsync(rot.data(), d_rot, sizeof(int) * np, cudaMemcpyDeviceToHost, s));
    HB_CUDA(cudaStreamSynchronize(s));
    bool changed = false;
    for (int p = 0; p < np; ++p) {
      Work &W = wk[p];
      if (!W.active || W.round != W.players - 1) continue;
      W.round = 0;
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
    if (changed) {
      bool more = false;
      for (const Work &W : wk) more = more || W.active;
      if (more) make_plans();
    }
  }
  if (d_jp) cudaFreeAsync(d_jp, s);
  tplan.reset();

  // ---- singular values, order, rank, outputs -------------------------------------------
  nd.clear();
  for (int p = 0; p < np; ++p) nd.push_back(NormDesc{w + wk[p].x, wk[p].L, wk[p].L, wk[p].Lp,
                                                     w + noff[p]});
  column_norms2(nd, s);
  std::vector<CopyDesc> gather;
  std::vector<std::vector<double>> sig(np);
  std::vector<int> ranks(np), sweeps(np);
  for (int p = 0; p < np; ++p) {
    const Work &W = wk[p];
    std::vector<double> n2(W.Lp);
    HB_CUDA(cudaMemcpyAsync(n2.data(), w + noff[p], sizeof(double) * W.Lp,
                            cudaMemcpyDeviceToHost, s));
    HB_CUDA(cudaStreamSynchronize(s));
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
  bool failed = false;
  for (int p = 0; p < np; ++p) {
    HB_CUDA(cudaMemcpyAsync(probs[p].sigma, sig[p].data(), sizeof(double) * wk[p].L,
                            cudaMemcpyHostToDevice, s));
    HB_CUDA(cudaMemcpyAsync(probs[p].rank, &ranks[p], sizeof(int), cudaMemcpyHostToDevice, s));
    if (probs[p].sweeps)
      HB_CUDA(cudaMemcpyAsync(probs[p].sweeps, &sweeps[p], sizeof(int), cudaMemcpyHostToDevice,
                              s));
    failed = failed || !wk[p].converged;
  }
  if (failed) {
    const int st = SVD_FAILURE;
    HB_CUDA(cudaMemcpyAsync(d_status, &st, sizeof(int), cudaMemcpyHostToDevice, s));
    set_last_error("block Jacobi SVD of a sketch core did not converge within "
                   "jacobi_max_sweeps sweeps");
  }
  HB_CUDA(cudaStreamSynchronize(s));
  cudaFreeAsync(d_ints, s);
  dev_free(w, s);
}

}  // namespace hb
