// HODLR factorisation and solve (see solve.h for the algebra).
//
// The capacitance matrix of a node, C = [I, P; Q, I] with P = V_tr^T W2 and
// Q = V_bl^T W1, has identity diagonal blocks, so only its Schur complement
// S = I - Q P (order s_bl) is inverted: C^-1 [t1; t2] = [t1 - P y2; y2] with
// y2 = S^-1 (t2 - Q t1).  Per node the factor keeps P, Q and S^-1.
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
enum Slot { kS_Arena = 0, kS_Buf = 1, kS_X = 2, kS_T = 3, kS_Y = 4, kS_Tmp = 5 };

struct NodeParts {
  long long p_off, q_off, sinv_off;   // in the factor buffer
};

}  // namespace

HodlrFactor::~HodlrFactor() {
  if (buf) cudaFree(buf);
}

namespace {

// Per-node offsets of P, Q, S^-1 (kept beside cinv_off's vector layout).
struct Layout {
  std::vector<NodeParts> parts;
};

// x <- (I + W_l V_l^T)^-1 x for every depth-l node, x with k columns (ld ldx,
// slot kS_X of `bases`).  Scratch: t (sum (s_tr + s_bl) k) and y (sum s_bl k).
void apply_level(const HodlrFactor &f, const Layout &L, int l, double *X, int k, long long ldx,
                 cudaStream_t s) {
  const DeviceTree &t = *f.tree;
  const Geometry &g = t.g;
  std::vector<long long> t_off(1 << l), y_off(1 << l);
  long long tt = 0, yy = 0;
  for (int j = 0; j < (1 << l); ++j) {
    const BlockDesc &tr = g.blocks[block_index(l, j, 1)], &bl = g.blocks[block_index(l, j, 2)];
    t_off[j] = tt;
    tt += align_up((long long)(tr.s + bl.s) * k);
    y_off[j] = yy;
    yy += align_up((long long)bl.s * k);
  }
  if (tt == 0) return;
  double *T = dev_alloc(tt, s), *Y = dev_alloc(yy, s);
  GemmBases b{};
  b.p[kS_Arena] = t.arena;
  b.p[kS_Buf] = f.buf;
  b.p[kS_X] = X;
  b.p[kS_T] = T;
  b.p[kS_Y] = Y;
  b.p[kS_Tmp] = T;
  const long long wl = f.w_off[l];
  // 1. t1 = V_tr^T x[child 2], t2 = V_bl^T x[child 1]
  GemmBatch g1;
  for (int j = 0; j < (1 << l); ++j) {
    const BlockDesc &tr = g.blocks[block_index(l, j, 1)], &bl = g.blocks[block_index(l, j, 2)];
    const int q = tr.s + bl.s;
    if (tr.s) {
      int p = g1.add(kS_T, t_off[j], q, tr.s, k);
      g1.seg(p, kS_Arena, tr.v_off, tr.n, 1, kS_X, tr.c0, ldx, 0, tr.n);
    }
    if (bl.s) {
      int p = g1.add(kS_T, t_off[j] + tr.s, q, bl.s, k);
      g1.seg(p, kS_Arena, bl.v_off, bl.n, 1, kS_X, bl.c0, ldx, 0, bl.n);
    }
  }
  gemm_f64_run(g1, b, TileShape::M64N128, s);
  // 2. t2 -= Q t1;  3. y = S^-1 t2;  4. t1 -= P y
  GemmBatch g2, g3, g4;
  for (int j = 0; j < (1 << l); ++j) {
    const BlockDesc &tr = g.blocks[block_index(l, j, 1)], &bl = g.blocks[block_index(l, j, 2)];
    const int q = tr.s + bl.s;
    const NodeParts &np = L.parts[node_index(l, j)];
    if (tr.s && bl.s) {
      int p = g2.add(kS_T, t_off[j] + tr.s, q, bl.s, k, -1.0, 1.0);
      g2.seg(p, kS_Buf, np.q_off, bl.s, 0, kS_T, t_off[j], q, 0, tr.s);
    }
    if (bl.s) {
      int p = g3.add(kS_Y, y_off[j], bl.s, bl.s, k);
      g3.seg(p, kS_Buf, np.sinv_off, bl.s, 0, kS_T, t_off[j] + tr.s, q, 0, bl.s);
    }
    if (tr.s && bl.s) {
      int p = g4.add(kS_T, t_off[j], q, tr.s, k, -1.0, 1.0);
      g4.seg(p, kS_Buf, np.p_off, tr.s, 0, kS_Y, y_off[j], bl.s, 0, bl.s);
    }
  }
  gemm_f64_run(g2, b, TileShape::M64N128, s, false);
  gemm_f64_run(g3, b, TileShape::M64N128, s, false);
  gemm_f64_run(g4, b, TileShape::M64N128, s, false);
  // 5. x[child 1] -= W1 t1, x[child 2] -= W2 y
  GemmBatch g5;
  for (int j = 0; j < (1 << l); ++j) {
    const BlockDesc &tr = g.blocks[block_index(l, j, 1)], &bl = g.blocks[block_index(l, j, 2)];
    const int q = tr.s + bl.s;
    if (tr.s) {
      int p = g5.add(kS_X, tr.r0, ldx, tr.m, k, -1.0, 1.0);
      g5.seg(p, kS_Buf, wl + tr.r0, g.n, 0, kS_T, t_off[j], q, 0, tr.s);
    }
    if (bl.s) {
      int p = g5.add(kS_X, bl.r0, ldx, bl.m, k, -1.0, 1.0);
      g5.seg(p, kS_Buf, wl + bl.r0, g.n, 0, kS_Y, y_off[j], bl.s, 0, bl.s);
    }
  }
  gemm_f64_run(g5, b, TileShape::M128N64, s, false);
  dev_free(T, s);
  dev_free(Y, s);
}

// X = D^-1 B, one block-diagonal GEMM launch (X and B distinct).
void apply_leaves(const HodlrFactor &f, const double *B, long long ldb, double *X, long long ldx,
                  int k, cudaStream_t s) {
  const DeviceTree &t = *f.tree;
  GemmBases b{};
  b.p[kS_Arena] = t.arena;
  b.p[kS_Buf] = f.buf;
  b.p[kS_X] = X;
  b.p[kS_T] = const_cast<double *>(B);
  b.p[kS_Y] = X;
  b.p[kS_Tmp] = X;
  GemmBatch gb;
  for (int i = 0; i < t.g.nleaf(); ++i) {
    const LeafDesc &L = t.leaves[i];
    if (L.m == 0) continue;
    int p = gb.add(kS_X, L.r0, ldx, L.m, k);
    gb.seg(p, kS_Buf, f.dinv_off + f.leaf_inv_off[i], L.m, 0, kS_T, L.r0, ldb, 0, L.m);
  }
  gemm_f64_run(gb, b, TileShape::M128N64, s);
}

// The layouts are rebuilt from the factor's geometry when needed.
Layout layout_of(const HodlrFactor &f) {
  Layout L;
  const Geometry &g = f.tree->g;
  L.parts.resize(g.nblock() / 2 + 1);
  long long o = f.cinv_off.empty() ? 0 : f.cinv_off[0];
  for (int d = 0; d < g.h; ++d)
    for (int j = 0; j < (1 << d); ++j) {
      const BlockDesc &tr = g.blocks[block_index(d, j, 1)], &bl = g.blocks[block_index(d, j, 2)];
      NodeParts &np = L.parts[node_index(d, j)];
      np.p_off = f.cinv_off[node_index(d, j)];
      np.q_off = np.p_off + align_up((long long)tr.s * bl.s);
      np.sinv_off = np.q_off + align_up((long long)bl.s * tr.s);
      (void)o;
    }
  return L;
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
  f->dinv_off = 0;
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
      const int s1 = g.blocks[block_index(d, j, 1)].s, s2 = g.blocks[block_index(d, j, 2)].s;
      f->cinv_off[node_index(d, j)] = total;
      f->q[node_index(d, j)] = s1 + s2;
      total += align_up((long long)s1 * s2) * 2 + align_up((long long)s2 * s2);
    }
  HB_CUDA(cudaMalloc(&f->buf, sizeof(double) * std::max<long long>(total, 1)));
  HB_CUDA(cudaMemsetAsync(f->buf, 0, sizeof(double) * std::max<long long>(total, 1), s));
  const Layout L = layout_of(*f);
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
                             f->buf + f->dinv_off + f->leaf_inv_off[i], lf.m});
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
    apply_leaves(*f, tmp, n, Wl, n, w, s);
    for (int lev = h - 1; lev > l; --lev) apply_level(*f, L, lev, Wl, w, n, s);
    // P = V_tr^T W2, Q = V_bl^T W1, S = I - Q P, S^-1
    GemmBases b{};
    b.p[kS_Arena] = t.arena;
    b.p[kS_Buf] = f->buf;
    for (int i = 2; i < kGemmBases; ++i) b.p[i] = f->buf;
    GemmBatch gpq, gs;
    std::vector<EyeDesc> eyes;
    std::vector<GjProb> inv;
    double *S = nullptr;
    long long stot = 0;
    std::vector<long long> s_off(1 << l, 0);
    for (int j = 0; j < (1 << l); ++j) {
      const int s2 = g.blocks[block_index(l, j, 2)].s;
      s_off[j] = stot;
      stot += align_up((long long)s2 * s2);
    }
    S = dev_alloc(stot, s);
    b.p[kS_Tmp] = S;
    for (int j = 0; j < (1 << l); ++j) {
      const BlockDesc &tr = g.blocks[block_index(l, j, 1)], &bl = g.blocks[block_index(l, j, 2)];
      const NodeParts &np = L.parts[node_index(l, j)];
      if (tr.s && bl.s) {
        int p = gpq.add(kS_Buf, np.p_off, tr.s, tr.s, bl.s);          // P: s_tr x s_bl
        gpq.seg(p, kS_Arena, tr.v_off, tr.n, 1, kS_Buf, f->w_off[l] + bl.r0, n, 0, tr.n);
        int q = gpq.add(kS_Buf, np.q_off, bl.s, bl.s, tr.s);          // Q: s_bl x s_tr
        gpq.seg(q, kS_Arena, bl.v_off, bl.n, 1, kS_Buf, f->w_off[l] + tr.r0, n, 0, bl.n);
        int sp = gs.add(kS_Tmp, s_off[j], bl.s, bl.s, bl.s, -1.0, 1.0);
        gs.seg(sp, kS_Buf, np.q_off, bl.s, 0, kS_Buf, np.p_off, tr.s, 0, tr.s);
      }
      if (bl.s) {
        eyes.push_back(EyeDesc{S + s_off[j], bl.s, bl.s});
        inv.push_back(GjProb{S + s_off[j], bl.s, bl.s, nullptr, f->buf + np.sinv_off, bl.s});
      }
    }
    gemm_f64_run(gpq, b, TileShape::M64N128, s);
    eye(eyes, s);
    gemm_f64_run(gs, b, TileShape::M64N128, s, false);
    gj_inverse(inv, d_status, s);
    dev_free(S, s);
  }
  dev_free(tmp, s);
  int st = 0;
  HB_CUDA(cudaMemcpyAsync(&st, d_status, sizeof(int), cudaMemcpyDeviceToHost, s));
  HB_CUDA(cudaStreamSynchronize(s));
  cudaFreeAsync(d_status, s);
  if (st) *status = INPUT_ERROR;
  return f;
}

void hodlr_solve(const HodlrFactor &f, const double *B, int k, long long ldb, double *X,
                 long long ldx, cudaStream_t s) {
  if (k <= 0 || f.tree->g.n == 0) return;
  const Layout L = layout_of(f);
  apply_leaves(f, B, ldb, X, ldx, k, s);
  for (int l = f.tree->g.h - 1; l >= 0; --l) apply_level(f, L, l, X, k, ldx, s);
}

}  // namespace hb
