// HODLR factorisation and solve (see solve.h for the algebra).
//
// The capacitance matrix of a node, C = [I, P; Q, I] with P = V_tr^T W2 and
// Q = V_bl^T W1, has identity diagonal blocks, so only its Schur complement
// S = I - Q P (order s_bl) is inverted; C^-1 is then assembled from P, Q and
// S^-1 by two small GEMM launches and kept, so that a solve applies it as one
// GEMM per level instead of three dependent ones.
#include <algorithm>
#include <cmath>

#include "gemm_f64.h"
#include "jacobi.h"
#include "solve.h"

namespace hb {

namespace {

constexpr int kGjThreads = 256;

struct GjProb {
  const double *A;   // n x n input (ld lda)
  long long lda;
  int n;
  double *work;      // n x 2n scratch, ld n
  double *inv;       // n x n output (ld ldi)
  long long ldi;
};

// Gauss-Jordan inversion with partial pivoting, one CTA per matrix, on the
// augmented [A | I] in global memory.  A pivot at rounding level relative to
// the matrix's largest entry sets *status (the output is then not used).
__global__ void __launch_bounds__(kGjThreads)
gj_inverse_kernel(const GjProb *__restrict__ probs, int *status) {
  const GjProb P = probs[blockIdx.x];
  const int n = P.n, tid = threadIdx.x;
  extern __shared__ double f[];              // n: the pivot column before elimination
  __shared__ double s_val[kGjThreads];
  __shared__ int s_idx[kGjThreads];
  __shared__ int s_stop;
  double *W = P.work;
  double amax = 0.0;
  for (long long e = tid; e < (long long)n * n; e += blockDim.x) {
    const int r = (int)(e % n), c = (int)(e / n);
    const double a = P.A[r + (long long)c * P.lda];
    W[e] = a;
    W[(long long)n * n + e] = (r == c) ? 1.0 : 0.0;
    amax = fmax(amax, fabs(a));
  }
  s_val[tid] = amax;
  if (tid == 0) s_stop = 0;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (tid < o) s_val[tid] = fmax(s_val[tid], s_val[tid + o]);
    __syncthreads();
  }
  const double tiny = fmax(64.0 * 2.220446049250313e-16 * s_val[0], 1e-300);
  __syncthreads();
  for (int k = 0; k < n; ++k) {
    // pivot: largest |W[r, k]|, r >= k
    double best = -1.0;
    int bi = k;
    for (int r = k + tid; r < n; r += blockDim.x) {
      const double v = fabs(W[r + (long long)k * n]);
      if (v > best) {
        best = v;
        bi = r;
      }
    }
    s_val[tid] = best;
    s_idx[tid] = bi;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
      if (tid < o && (s_val[tid + o] > s_val[tid] ||
                      (s_val[tid + o] == s_val[tid] && s_idx[tid + o] < s_idx[tid]))) {
        s_val[tid] = s_val[tid + o];
        s_idx[tid] = s_idx[tid + o];
      }
      __syncthreads();
    }
    const int p = s_idx[0];
    if (s_val[0] <= tiny) {
      if (tid == 0) {
        s_stop = 1;
        atomicExch(status, 1);
      }
    }
    __syncthreads();
    if (s_stop) break;
    // swap rows k and p, scale row k
    const double inv = 1.0 / W[p + (long long)k * n];
    for (int c = tid; c < 2 * n; c += blockDim.x) {
      const double a = W[k + (long long)c * n], b = W[p + (long long)c * n];
      W[p + (long long)c * n] = a;
      W[k + (long long)c * n] = b * inv;
    }
    __syncthreads();
    for (int r = tid; r < n; r += blockDim.x) f[r] = W[r + (long long)k * n];
    __syncthreads();
    // eliminate column k from every other row (columns < k of row k are 0)
    const long long cols = 2LL * n - k;
    for (long long e = tid; e < (long long)n * cols; e += blockDim.x) {
      const int r = (int)(e % n);
      const long long c = k + e / n;
      if (r != k) W[r + c * n] -= f[r] * W[k + c * n];
    }
    __syncthreads();
  }
  for (long long e = tid; e < (long long)n * n; e += blockDim.x) {
    const int r = (int)(e % n), c = (int)(e / n);
    P.inv[r + (long long)c * P.ldi] = W[(long long)n * n + e];
  }
}

struct EyeDesc {
  double *X;
  long long ld;
  int n;
};

__global__ void eye_kernel(const EyeDesc *__restrict__ d) {
  const EyeDesc E = d[blockIdx.y];
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < (long long)E.n * E.n;
       e += (long long)gridDim.x * blockDim.x) {
    const int r = (int)(e % E.n), c = (int)(e / E.n);
    E.X[r + (long long)c * E.ld] = (r == c) ? 1.0 : 0.0;
  }
}

template <class T>
T *upload_tmp(const std::vector<T> &v, cudaStream_t s) {
  T *d = nullptr;
  HB_CUDA(cudaMallocAsync((void **)&d, sizeof(T) * std::max<size_t>(v.size(), 1), s));
  if (!v.empty())
    HB_CUDA(cudaMemcpyAsync(d, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice, s));
  return d;
}

void gj_inverse(std::vector<GjProb> probs, int *d_status, cudaStream_t s) {
  if (probs.empty()) return;
  int nmax = 0;
  long long work = 0;
  for (auto &p : probs) {
    nmax = std::max(nmax, p.n);
    work += align_up(2LL * p.n * p.n);
  }
  double *w = dev_alloc(work, s);
  long long o = 0;
  for (auto &p : probs) {
    p.work = w + o;
    o += align_up(2LL * p.n * p.n);
  }
  GjProb *d = upload_tmp(probs, s);
  const size_t smem = sizeof(double) * std::max(nmax, 1);
  HB_REQUIRE(smem <= 200 * 1024, INPUT_ERROR, "solve: capacitance matrix too large");
  if (smem > 48 * 1024)
    HB_CUDA(cudaFuncSetAttribute(gj_inverse_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem));
  gj_inverse_kernel<<<(int)probs.size(), kGjThreads, smem, s>>>(d, d_status);
  HB_LAUNCHED();
  cudaFreeAsync(d, s);
  dev_free(w, s);
}

void eye(const std::vector<EyeDesc> &v, cudaStream_t s) {
  if (v.empty()) return;
  EyeDesc *d = upload_tmp(v, s);
  for (size_t off = 0; off < v.size(); off += 65535) {
    eye_kernel<<<dim3(8, (unsigned)std::min<size_t>(65535, v.size() - off)), 256, 0, s>>>(d + off);
    HB_LAUNCHED();
  }
  cudaFreeAsync(d, s);
}

int node_index(int d, int j) { return (1 << d) - 1 + j; }

// Base slots of the solver's GEMM launches.
enum Slot { kS_Arena = 0, kS_Buf = 1, kS_X = 2, kS_B = 3, kS_T = 4, kS_Z = 5 };

GemmBases solver_bases(const HodlrFactor &f, double *X, const double *B, double *T, double *Z) {
  GemmBases b{};
  b.p[kS_Arena] = f.tree->arena;
  b.p[kS_Buf] = f.buf;
  b.p[kS_X] = X;
  b.p[kS_B] = const_cast<double *>(B);
  b.p[kS_T] = T;
  b.p[kS_Z] = Z;
  return b;
}

// Scratch of one level: t and z of node j at off[j] (q_j x k, ld q_j).
long long level_scratch(const HodlrFactor &f, int l, int k, std::vector<long long> *off) {
  long long tot = 0;
  if (off) off->assign(1 << l, 0);
  for (int j = 0; j < (1 << l); ++j) {
    if (off) (*off)[j] = tot;
    tot += align_up((long long)f.q[node_index(l, j)] * k);
  }
  return tot;
}

// The three launches of x <- (I + W_l V_l^T)^-1 x, x in slot kS_X (ld ldx, k
// columns), t in kS_T, z in kS_Z.
struct LevelBatches {
  GemmBatch vt, cz, wx;
};

LevelBatches level_batches(const HodlrFactor &f, int l, int k, long long ldx) {
  const Geometry &g = f.tree->g;
  std::vector<long long> off;
  level_scratch(f, l, k, &off);
  LevelBatches L;
  const long long wl = f.w_off[l];
  for (int j = 0; j < (1 << l); ++j) {
    const BlockDesc &tr = g.blocks[block_index(l, j, 1)], &bl = g.blocks[block_index(l, j, 2)];
    const int q = tr.s + bl.s;
    if (q == 0) continue;
    // t = [V_tr^T x[child 2]; V_bl^T x[child 1]]
    if (tr.s) {
      const int p = L.vt.add(kS_T, off[j], q, tr.s, k);
      L.vt.seg(p, kS_Arena, tr.v_off, tr.n, 1, kS_X, tr.c0, ldx, 0, tr.n);
    }
    if (bl.s) {
      const int p = L.vt.add(kS_T, off[j] + tr.s, q, bl.s, k);
      L.vt.seg(p, kS_Arena, bl.v_off, bl.n, 1, kS_X, bl.c0, ldx, 0, bl.n);
    }
    // z = C^-1 t
    const int p = L.cz.add(kS_Z, off[j], q, q, k);
    L.cz.seg(p, kS_Buf, f.cinv_off[node_index(l, j)], q, 0, kS_T, off[j], q, 0, q);
    // x[child 1] -= W1 z1, x[child 2] -= W2 z2
    if (tr.s) {
      const int p1 = L.wx.add(kS_X, tr.r0, ldx, tr.m, k, -1.0, 1.0);
      L.wx.seg(p1, kS_Buf, wl + tr.r0, g.n, 0, kS_Z, off[j], q, 0, tr.s);
    }
    if (bl.s) {
      const int p2 = L.wx.add(kS_X, bl.r0, ldx, bl.m, k, -1.0, 1.0);
      L.wx.seg(p2, kS_Buf, wl + bl.r0, g.n, 0, kS_Z, off[j] + tr.s, q, 0, bl.s);
    }
  }
  return L;
}

// X = D^-1 B: X in slot kS_X, B in kS_B (distinct).
GemmBatch leaf_batch(const HodlrFactor &f, int k, long long ldb, long long ldx) {
  const DeviceTree &t = *f.tree;
  GemmBatch gb;
  for (int i = 0; i < t.g.nleaf(); ++i) {
    const LeafDesc &L = t.leaves[i];
    if (L.m == 0) continue;
    const int p = gb.add(kS_X, L.r0, ldx, L.m, k);
    gb.seg(p, kS_Buf, f.leaf_inv_off[i], L.m, 0, kS_B, L.r0, ldb, 0, L.m);
  }
  return gb;
}

constexpr TileShape kShapeLeaves = TileShape::M128N64;
constexpr TileShape kShapeVt = TileShape::M64N128;
constexpr TileShape kShapeCz = TileShape::M64N128;
constexpr TileShape kShapeWx = TileShape::M128N64;

// One-shot application (factorisation, where k is a level's rank).
void apply_leaves_once(const HodlrFactor &f, const double *B, long long ldb, double *X,
                       long long ldx, int k, cudaStream_t s) {
  GemmBatch gb = leaf_batch(f, k, ldb, ldx);
  gemm_f64_run(gb, solver_bases(f, X, B, nullptr, nullptr), kShapeLeaves, s);
}

void apply_level_once(const HodlrFactor &f, int l, double *X, int k, long long ldx,
                      cudaStream_t s) {
  const long long tot = level_scratch(f, l, k, nullptr);
  if (tot == 0) return;
  double *T = dev_alloc(tot, s), *Z = dev_alloc(tot, s);
  const GemmBases b = solver_bases(f, X, nullptr, T, Z);
  LevelBatches L = level_batches(f, l, k, ldx);
  gemm_f64_run(L.vt, b, kShapeVt, s);
  gemm_f64_run(L.cz, b, kShapeCz, s);
  gemm_f64_run(L.wx, b, kShapeWx, s, false);
  dev_free(T, s);
  dev_free(Z, s);
}

}  // namespace

struct SolvePlan {
  GemmPlan leaves;
  std::vector<std::unique_ptr<GemmPlan>> vt, cz, wx;   // per depth
  double *T = nullptr, *Z = nullptr;                  // scratch of the largest level
  ~SolvePlan() {
    if (T) cudaFree(T);
    if (Z) cudaFree(Z);
  }
};

HodlrFactor::HodlrFactor() = default;

HodlrFactor::~HodlrFactor() {
  plans.clear();
  if (buf) cudaFree(buf);
}

namespace {

void build_plan(GemmPlan &plan, GemmBatch &batch, TileShape shape, bool split, cudaStream_t s) {
  if (!batch.empty()) gemm_plan_build(plan, batch, shape, split, s);
}

SolvePlan &solve_plan(HodlrFactor &f, int k, long long ldb, long long ldx, cudaStream_t s) {
  std::lock_guard<std::mutex> lk(f.plan_mutex);
  const auto key = std::make_tuple(k, ldb, ldx, s);
  auto it = f.plans.find(key);
  if (it != f.plans.end()) return *it->second;
  auto P = std::make_unique<SolvePlan>();
  const int h = f.tree->g.h;
  GemmBatch lb = leaf_batch(f, k, ldb, ldx);
  build_plan(P->leaves, lb, kShapeLeaves, true, s);
  long long scratch = 0;
  for (int l = 0; l < h; ++l) {
    scratch = std::max(scratch, level_scratch(f, l, k, nullptr));
    LevelBatches L = level_batches(f, l, k, ldx);
    P->vt.push_back(std::make_unique<GemmPlan>());
    P->cz.push_back(std::make_unique<GemmPlan>());
    P->wx.push_back(std::make_unique<GemmPlan>());
    build_plan(*P->vt.back(), L.vt, kShapeVt, true, s);
    build_plan(*P->cz.back(), L.cz, kShapeCz, true, s);     // K = q: split near the root
    build_plan(*P->wx.back(), L.wx, kShapeWx, false, s);
  }
  HB_CUDA(cudaMalloc(&P->T, sizeof(double) * std::max<long long>(scratch, 1)));
  HB_CUDA(cudaMalloc(&P->Z, sizeof(double) * std::max<long long>(scratch, 1)));
  auto &ref = *P;
  f.plans[key] = std::move(P);
  return ref;
}

}  // namespace

std::unique_ptr<HodlrFactor> hodlr_factorize(std::shared_ptr<DeviceTree> tp, cudaStream_t s,
                                             int *status) {
  auto f = std::make_unique<HodlrFactor>();
  f->tree = tp;
  const DeviceTree &t = *tp;
  const Geometry &g = t.g;
  const int h = g.h, n = g.n;
  *status = SUCCESS;
  // ---- layout of the factor buffer ------------------------------------------------
  long long total = 0;
  f->leaf_inv_off.resize(g.nleaf());
  for (int i = 0; i < g.nleaf(); ++i) {
    f->leaf_inv_off[i] = total;
    total += align_up((long long)g.leaf_m[i] * g.leaf_m[i]);
  }
  f->w_off.assign(h, 0);
  f->w_cols.assign(h, 0);
  for (int l = 0; l < h; ++l) {
    int w = 0;
    for (int j = 0; j < (1 << l); ++j)
      w = std::max({w, g.blocks[block_index(l, j, 1)].s, g.blocks[block_index(l, j, 2)].s});
    f->w_cols[l] = w;
    f->w_off[l] = total;
    total += align_up((long long)n * w);
  }
  const int nnodes = (1 << h) - 1;
  f->cinv_off.assign(nnodes, 0);
  f->q.assign(nnodes, 0);
  for (int d = 0; d < h; ++d)
    for (int j = 0; j < (1 << d); ++j) {
      const int q = g.blocks[block_index(d, j, 1)].s + g.blocks[block_index(d, j, 2)].s;
      f->cinv_off[node_index(d, j)] = total;
      f->q[node_index(d, j)] = q;
      total += align_up((long long)q * q);
    }
  HB_CUDA(cudaMalloc(&f->buf, sizeof(double) * std::max<long long>(total, 1)));
  HB_CUDA(cudaMemsetAsync(f->buf, 0, sizeof(double) * std::max<long long>(total, 1), s));
  int *d_status = nullptr;
  HB_CUDA(cudaMallocAsync((void **)&d_status, sizeof(int), s));
  HB_CUDA(cudaMemsetAsync(d_status, 0, sizeof(int), s));

  // ---- leaf inverses -----------------------------------------------------------------
  {
    std::vector<GjProb> probs;
    for (int i = 0; i < g.nleaf(); ++i) {
      const LeafDesc &lf = t.leaves[i];
      if (lf.m == 0) continue;
      probs.push_back(GjProb{t.arena + lf.off, lf.m, lf.m, nullptr,
                             f->buf + f->leaf_inv_off[i], lf.m});
    }
    gj_inverse(probs, d_status, s);
  }

  // ---- levels, deepest first -----------------------------------------------------------
  const int wmax = *std::max_element(f->w_cols.begin(), f->w_cols.end());
  double *tmp = dev_alloc((long long)n * std::max(wmax, 1), s);
  for (int l = h - 1; l >= 0; --l) {
    const int w = f->w_cols[l];
    if (w == 0) continue;
    double *Wl = f->buf + f->w_off[l];
    // stack the level's U blocks, band by band, then W_l = D^-1 U
    HB_CUDA(cudaMemsetAsync(tmp, 0, sizeof(double) * (long long)n * w, s));
    std::vector<CopyDesc> cp;
    for (int j = 0; j < (1 << l); ++j)
      for (int c = 1; c <= 2; ++c) {
        const BlockDesc &B = g.blocks[block_index(l, j, c)];
        if (B.s) cp.push_back(CopyDesc{t.arena + B.u_off, B.m, tmp + B.r0, n, B.m, B.s});
      }
    CopyDesc *dcp = upload_tmp(cp, s);
    copy2d_batched(dcp, (int)cp.size(), s);
    cudaFreeAsync(dcp, s);
    apply_leaves_once(*f, tmp, n, Wl, n, w, s);
    for (int lev = h - 1; lev > l; --lev) apply_level_once(*f, lev, Wl, w, n, s);

    // C^-1 of every node of the level.  Scratch per node with both ranks
    // nonzero: P (s_tr x s_bl), Q (s_bl x s_tr), S (s_bl x s_bl).
    std::vector<long long> p_off(1 << l, 0), q_off(1 << l, 0), s_off(1 << l, 0);
    long long scratch = 0;
    for (int j = 0; j < (1 << l); ++j) {
      const int s1 = g.blocks[block_index(l, j, 1)].s, s2 = g.blocks[block_index(l, j, 2)].s;
      if (!s1 || !s2) continue;
      p_off[j] = scratch;
      scratch += align_up((long long)s1 * s2);
      q_off[j] = scratch;
      scratch += align_up((long long)s2 * s1);
      s_off[j] = scratch;
      scratch += align_up((long long)s2 * s2);
    }
    std::vector<EyeDesc> eyes;
    for (int j = 0; j < (1 << l); ++j) {
      const int q = f->q[node_index(l, j)];
      if (q) eyes.push_back(EyeDesc{f->buf + f->cinv_off[node_index(l, j)], q, q});
    }
    eye(eyes, s);                              // C^-1 = I where a rank is zero
    if (scratch == 0) continue;
    double *Ps = dev_alloc(scratch, s);
    const GemmBases b = solver_bases(*f, nullptr, nullptr, Ps, nullptr);
    GemmBatch gpq, gs, c1, c2;
    std::vector<EyeDesc> s_eye;
    std::vector<GjProb> inv;
    for (int j = 0; j < (1 << l); ++j) {
      const BlockDesc &tr = g.blocks[block_index(l, j, 1)], &bl = g.blocks[block_index(l, j, 2)];
      const int s1 = tr.s, s2 = bl.s, q = s1 + s2;
      if (!s1 || !s2) continue;
      const long long ci = f->cinv_off[node_index(l, j)];
      const long long br = ci + s1 + (long long)s1 * q, bl_off = ci + s1, tr_off = ci + (long long)s1 * q;
      int p = gpq.add(kS_T, p_off[j], s1, s1, s2);                 // P = V_tr^T W2
      gpq.seg(p, kS_Arena, tr.v_off, tr.n, 1, kS_Buf, f->w_off[l] + bl.r0, n, 0, tr.n);
      p = gpq.add(kS_T, q_off[j], s2, s2, s1);                     // Q = V_bl^T W1
      gpq.seg(p, kS_Arena, bl.v_off, bl.n, 1, kS_Buf, f->w_off[l] + tr.r0, n, 0, bl.n);
      p = gs.add(kS_T, s_off[j], s2, s2, s2, -1.0, 1.0);           // S = I - Q P
      gs.seg(p, kS_T, q_off[j], s2, 0, kS_T, p_off[j], s1, 0, s1);
      s_eye.push_back(EyeDesc{Ps + s_off[j], s2, s2});
      inv.push_back(GjProb{Ps + s_off[j], s2, s2, nullptr, f->buf + br, q});   // S^-1 -> C^-1[bl, bl]
      p = c1.add(kS_Buf, tr_off, q, s1, s2, -1.0);                 // C^-1[tr, bl] = -P S^-1
      c1.seg(p, kS_T, p_off[j], s1, 0, kS_Buf, br, q, 0, s2);
      p = c1.add(kS_Buf, bl_off, q, s2, s1, -1.0);                 // C^-1[bl, tr] = -S^-1 Q
      c1.seg(p, kS_Buf, br, q, 0, kS_T, q_off[j], s2, 0, s2);
      p = c2.add(kS_Buf, ci, q, s1, s1, -1.0, 1.0);                // C^-1[tr, tr] = I - P C^-1[bl, tr]
      c2.seg(p, kS_T, p_off[j], s1, 0, kS_Buf, bl_off, q, 0, s2);
    }
    gemm_f64_run(gpq, b, TileShape::M64N128, s);
    eye(s_eye, s);
    gemm_f64_run(gs, b, TileShape::M64N128, s, false);
    gj_inverse(inv, d_status, s);
    gemm_f64_run(c1, b, TileShape::M64N128, s, false);
    gemm_f64_run(c2, b, TileShape::M64N128, s, false);
    dev_free(Ps, s);
  }
  dev_free(tmp, s);
  int st = 0;
  HB_CUDA(cudaMemcpyAsync(&st, d_status, sizeof(int), cudaMemcpyDeviceToHost, s));
  HB_CUDA(cudaStreamSynchronize(s));
  cudaFreeAsync(d_status, s);
  if (st) *status = INPUT_ERROR;
  return f;
}

void hodlr_solve(HodlrFactor &f, const double *B, int k, long long ldb, double *X,
                 long long ldx, cudaStream_t s) {
  if (k <= 0 || f.tree->g.n == 0) return;
  SolvePlan &P = solve_plan(f, k, ldb, ldx, s);
  const GemmBases b = solver_bases(f, X, B, P.T, P.Z);
  gemm_plan_run(P.leaves, b, s);
  for (int l = f.tree->g.h - 1; l >= 0; --l) {
    gemm_plan_run(*P.vt[l], b, s);
    gemm_plan_run(*P.cz[l], b, s);
    gemm_plan_run(*P.wx[l], b, s);
  }
}

}  // namespace hb
