// HODLR x HODLR with recompression on the device (replaces hmat_lib
// src/hodlr_algebra.c: multiply_hodlr_hodlr :1452, compute_diagonal :1267,
// add_off_diagonal_contribution :1189, compute_inner_off_diagonal :780,
// compute_other_off_diagonal :1057, compute_higher_level_contributions_off_diagonal
// :467, recompress :97, recompress_large_s :280).
//
// For output block (d, j, c) the exact product is a sum of low-rank terms:
//  * one per ancestor (dd, jj): U_A(anc)[rows] (V_A(anc)^T U_B(anc')) V_B(anc')[cols]^T,
//    where anc / anc' are A's and B's off-diagonal blocks of (dd, jj) on the
//    two sides of the output block;
//  * two inside the node: (A's diagonal subtree) U_B(d, j, c) V_B(d, j, c)^T and
//    U_A(d, j, c) ((B's diagonal subtree)^T V_A(d, j, c))^T.
// The subtree products of all nodes of one depth are one masked HODLR product
// (only leaves and blocks below that depth) on a stacked right-hand side.  The
// concatenated factors of every output block are then recompressed at once:
// blocked Householder QR of U and V (BCGS2 + TSQR panels), SVD of
// R_U R_V^T (Jacobi), absolute truncation, U = Q_U W Sigma, V = Q_V Z; or,
// when the concatenated rank reaches min(m, n) on a small block, an SVD of the
// dense product (the reference's recompress_large_s).  Diagonal leaves are
// D_A D_B plus every ancestor's term, accumulated in one segmented GEMM.
#include <algorithm>

#include "hxh.h"
#include "jacobi.h"
#include "products.h"
#include "tsqr.h"

namespace hb {

namespace {

enum Slot { kA = 0, kB = 1, kWork = 2, kOut = 3 };

template <class T>
T *upload_vec(const std::vector<T> &v, cudaStream_t s) {
  T *d = nullptr;
  HB_CUDA(cudaMallocAsync((void **)&d, sizeof(T) * std::max<size_t>(v.size(), 1), s));
  if (!v.empty())
    HB_CUDA(cudaMemcpyAsync(d, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice, s));
  return d;
}

void run_copies(const std::vector<CopyDesc> &c, cudaStream_t s) {
  if (c.empty()) return;
  CopyDesc *d = upload_vec(c, s);
  copy2d_batched(d, (int)c.size(), s);
  cudaFreeAsync(d, s);
}

// Blocked Householder QR of Y (m x S), Q written over Y, R (S x S, zeroed by
// the caller) accumulated: 32-column panels, each orthogonalised against the
// previous columns twice (coefficients added into R) and then factored by
// TSQR.  Columns that carry no new direction get an R row of (near) zero.
struct BlockQr {
  double *Y;
  long long ldy;
  int m, S;
  double *R;
  long long ldr;
  double *C;   // scratch S x kPanel (ld S)
};

void block_qr(const std::vector<BlockQr> &probs, double *base, cudaStream_t s) {
  int max_panels = 0;
  for (auto &p : probs) max_panels = std::max(max_panels, (p.S + kPanel - 1) / kPanel);
  GemmBases gb{};
  for (int i = 0; i < kGemmBases; ++i) gb.p[i] = base;
  auto off = [&](const double *p) { return (long long)(p - base); };
  for (int q = 0; q < max_panels; ++q) {
    std::vector<const BlockQr *> pa;
    for (auto &p : probs)
      if (q * kPanel < p.S) pa.push_back(&p);
    for (int rep = 0; rep < 2; ++rep) {
      GemmBatch gc, gu;
      std::vector<CopyDesc> acc;
      for (const BlockQr *p : pa) {
        const int p0 = q * kPanel, pw = std::min(kPanel, p->S - p0);
        if (p0 == 0) continue;
        const double *panel = p->Y + (long long)p0 * p->ldy;
        double *ctarget = rep == 0 ? p->R + (long long)p0 * p->ldr : p->C;
        const long long cld = rep == 0 ? p->ldr : p->S;
        int pr = gc.add(0, off(ctarget), cld, p0, pw);
        gc.seg(pr, 0, off(p->Y), p->ldy, 1, 0, off(panel), p->ldy, 0, p->m);
        int pu = gu.add(0, off(panel), p->ldy, p->m, pw, -1.0, 1.0);
        gu.seg(pu, 0, off(p->Y), p->ldy, 0, 0, off(ctarget), cld, 0, p0);
        if (rep == 1)
          acc.push_back(CopyDesc{p->C, p->S, p->R + (long long)p0 * p->ldr, p->ldr, p0, pw});
      }
      gemm_f64_run(gc, gb, TileShape::M64N128, s);
      gemm_f64_run(gu, gb, TileShape::M128N64, s, false);
      if (!acc.empty()) {
        CopyDesc *d = upload_vec(acc, s);
        add2d_batched(d, (int)acc.size(), 1.0, s);
        cudaFreeAsync(d, s);
      }
    }
    std::vector<TsqrProb> tp;
    for (const BlockQr *p : pa) {
      const int p0 = q * kPanel, pw = std::min(kPanel, p->S - p0);
      tp.push_back(TsqrProb{p->Y + (long long)p0 * p->ldy, p->ldy, p->m, pw,
                            p->R + p0 + (long long)p0 * p->ldr, p->ldr});
    }
    tsqr_batched(tp, s);
  }
}

// ---- recompression of concatenated factors --------------------------------------
// hmat_lib recompress (src/hodlr_algebra.c:97-211) and recompress_large_s
// (:280-343), batched over blocks: blocked Householder QR of U and of V, SVD
// of R_U R_V^T by Jacobi, absolute truncation (:160-163), U' = Q_U W Sigma,
// V' = Q_V Z; a job marked dense decomposes U V^T itself instead.
struct RecompJob {
  int m = 0, n = 0, S = 0;   // block rows, columns, concatenated rank
  long long u = 0, v = 0;    // workspace offsets of U (m x S, ld m) and V (n x S, ld n)
  bool dense = false;        // SVD of the dense m x n product (recompress_large_s)
  long long ru = 0, rv = 0, mm = 0, cs = 0, jws = 0, jo_u = 0, jo_v = 0, jsig = 0, dmat = 0;
  bool active() const { return std::min(m, n) > 0 && S > 0; }
};

// Workspace of every job (`take(e)` returns the offset of e doubles);
// returns the widest Jacobi problem.
template <class Take>
int recomp_layout(std::vector<RecompJob> &jobs, Take take) {
  int max_c = 1;
  for (RecompJob &j : jobs) {
    const int mn = std::min(j.m, j.n);
    if (mn == 0) continue;
    const int Sb = std::max(j.S, 1);
    if (j.dense) {
      j.dmat = take((long long)j.m * j.n);
      j.jws = take(jacobi_workspace(j.m, j.n));
      j.jo_u = take((long long)j.m * mn);
      j.jo_v = take((long long)j.n * mn);
      j.jsig = take(mn);
      max_c = std::max(max_c, mn);
    } else {
      j.ru = take((long long)Sb * Sb);
      j.rv = take((long long)Sb * Sb);
      j.mm = take((long long)Sb * Sb);
      j.cs = take((long long)Sb * kPanel);
      j.jws = take(jacobi_workspace(Sb, Sb));
      j.jo_u = take((long long)Sb * Sb);
      j.jo_v = take((long long)Sb * Sb);
      j.jsig = take(Sb);
      max_c = std::max(max_c, Sb);
    }
  }
  return max_c;
}

// Runs the QRs, the dense products and the Jacobi SVDs of every job (the R
// blocks of the workspace must be zero); returns each job's rank (0 for
// inactive jobs) and the Jacobi status in *status.  Synchronises.
std::vector<int> recomp_run(const std::vector<RecompJob> &jobs, double *work, double tol,
                            int max_c, cudaStream_t s, int *status) {
  GemmBases gb{};
  for (int i = 0; i < kGemmBases; ++i) gb.p[i] = work;
  const int nj = (int)jobs.size();
  std::vector<BlockQr> qr_u, qr_v;
  GemmBatch gd;   // dense products U V^T of the dense jobs
  for (const RecompJob &j : jobs) {
    if (!j.active()) continue;
    if (j.dense) {
      int p = gd.add(kWork, j.dmat, j.m, j.m, j.n);
      gd.seg(p, kWork, j.u, j.m, 0, kWork, j.v, j.n, 1, j.S);
    } else {
      // the two QRs of a job share its C scratch: U's and V's run separately
      qr_u.push_back(BlockQr{work + j.u, j.m, j.m, j.S, work + j.ru, j.S, work + j.cs});
      qr_v.push_back(BlockQr{work + j.v, j.n, j.n, j.S, work + j.rv, j.S, work + j.cs});
    }
  }
  gemm_f64_run(gd, gb, TileShape::M128N64, s);
  block_qr(qr_u, work, s);
  block_qr(qr_v, work, s);
  {
    GemmBatch gm;   // M = R_U R_V^T
    for (const RecompJob &j : jobs) {
      if (!j.active() || j.dense) continue;
      int p = gm.add(kWork, j.mm, j.S, j.S, j.S);
      gm.seg(p, kWork, j.ru, j.S, 0, kWork, j.rv, j.S, 1, j.S);
    }
    gemm_f64_run(gm, gb, TileShape::M64N128, s);
  }
  std::vector<JacobiProb> jp;
  int *d_int = nullptr;
  HB_CUDA(cudaMallocAsync((void **)&d_int, sizeof(int) * (nj + 1), s));
  HB_CUDA(cudaMemsetAsync(d_int, 0, sizeof(int) * (nj + 1), s));
  for (int i = 0; i < nj; ++i) {
    const RecompJob &j = jobs[i];
    if (!j.active()) continue;
    JacobiProb p{};
    p.transA = 0;
    if (j.dense) {
      p.A = work + j.dmat;
      p.lda = j.m;
      p.m = j.m;
      p.n = j.n;
      p.ldu = j.m;
      p.ldv = j.n;
    } else {
      p.A = work + j.mm;
      p.lda = j.S;
      p.m = j.S;
      p.n = j.S;
      p.ldu = j.S;
      p.ldv = j.S;
    }
    const long long R = std::max(p.m, p.n), C = std::min(p.m, p.n);
    p.G = work + j.jws;
    p.W = p.G + align_up(R * C);
    p.U = work + j.jo_u;
    p.V = work + j.jo_v;
    p.sigma = work + j.jsig;
    p.rank = d_int + i;
    p.sweeps = nullptr;
    jp.push_back(p);
  }
  if (!jp.empty()) {
    JacobiParams prm;
    prm.tol = tol;
    prm.trunc = Truncation::Absolute;
    prm.scale_u = 1;
    prm.max_sweeps = (int)option("jacobi_max_sweeps", 60);
    JacobiProb *d_jp = upload_vec(jp, s);
    jacobi_svd_batched(d_jp, (int)jp.size(), prm, d_int + nj, max_c, s);
    cudaFreeAsync(d_jp, s);
  }
  std::vector<int> ints(nj + 1, 0);
  HB_CUDA(cudaMemcpyAsync(ints.data(), d_int, sizeof(int) * (nj + 1), cudaMemcpyDeviceToHost, s));
  HB_CUDA(cudaStreamSynchronize(s));
  dev_free(d_int, s);
  *status = ints[nj];
  ints.resize(nj);
  for (int i = 0; i < nj; ++i)
    if (!jobs[i].active()) ints[i] = 0;
  return ints;
}

// Writes job i's recompressed factors, U' (m x r, ld m) at out + uo[i] and
// V' (n x r, ld n) at out + vo[i], r = ranks[i].
void recomp_finish(const std::vector<RecompJob> &jobs, const std::vector<int> &ranks,
                   double *work, double *out, const std::vector<long long> &uo,
                   const std::vector<long long> &vo, cudaStream_t s) {
  GemmBases gb{};
  for (int i = 0; i < kGemmBases; ++i) gb.p[i] = work;
  gb.p[kOut] = out;
  std::vector<CopyDesc> cp;
  GemmBatch gf;
  for (size_t i = 0; i < jobs.size(); ++i) {
    const RecompJob &j = jobs[i];
    const int r = ranks[i];
    if (r == 0) continue;
    if (j.dense) {
      cp.push_back(CopyDesc{work + j.jo_u, j.m, out + uo[i], j.m, j.m, r});
      cp.push_back(CopyDesc{work + j.jo_v, j.n, out + vo[i], j.n, j.n, r});
    } else {
      int pu = gf.add(kOut, uo[i], j.m, j.m, r);
      gf.seg(pu, kWork, j.u, j.m, 0, kWork, j.jo_u, j.S, 0, j.S);
      int pv = gf.add(kOut, vo[i], j.n, j.n, r);
      gf.seg(pv, kWork, j.v, j.n, 0, kWork, j.jo_v, j.S, 0, j.S);
    }
  }
  run_copies(cp, s);
  gemm_f64_run(gf, gb, TileShape::M128N64, s, false);
}

struct Term {        // one low-rank term of an output block
  int kind;          // 0 ancestor, 1 in-node "subtree x U_B", 2 in-node "U_A"
  int a_block, b_block;
  int core;          // index into the cores (ancestor terms)
  int cols;          // columns this term contributes
};

}  // namespace

std::shared_ptr<DeviceTree> hxh_multiply(DeviceTree &A, DeviceTree &B, double tol,
                                         cudaStream_t s, int *status) {
  *status = SUCCESS;
  const Geometry &ga = A.g, &gbg = B.g;
  HB_REQUIRE(ga.h == gbg.h && ga.leaf_m == gbg.leaf_m, INPUT_ERROR,
             "multiply_hodlr_hodlr: trees of different heights or block sizes");
  const int h = ga.h, nb = ga.nblock(), nleaf = ga.nleaf(), n = ga.n;
  const int dense_max = (int)option("hxh_dense_max", 256);
  // option hxh_precision = 1: the subtree products (the bulk of the product's
  // multiply-adds) on the int8 tensor cores; cores, recompression and leaves
  // stay FP64.  Needs leaves that are multiples of 32.
  bool mixed = option("hxh_precision", 0.0) == 1.0;
  for (int m : ga.leaf_m) mixed = mixed && (m % 32 == 0);

  // ---- workspace layout --------------------------------------------------------
  long long ws = 0;
  auto take = [&](long long e) {
    const long long o = ws;
    ws += align_up(std::max<long long>(e, 1));
    return o;
  };
  // cores of every internal node: core[2k] = V_A(k,1)^T U_B(k,2), core[2k+1] = V_A(k,2)^T U_B(k,1)
  const int ninternal = (1 << h) - 1;
  std::vector<long long> core_off(2 * ninternal);
  std::vector<int> core_m(2 * ninternal), core_n(2 * ninternal);
  for (int k = 0; k < ninternal; ++k)
    for (int side = 0; side < 2; ++side) {
      const BlockDesc &a = ga.blocks[2 * k + side];
      const BlockDesc &b = gbg.blocks[2 * k + (1 - side)];
      core_m[2 * k + side] = a.s;
      core_n[2 * k + side] = b.s;
      core_off[2 * k + side] = take((long long)a.s * b.s);
    }
  // stacked subtree-product operands per depth
  std::vector<int> smax_b(h, 0), smax_a(h, 0);
  for (int b = 0; b < nb; ++b) {
    smax_b[ga.blocks[b].depth] = std::max(smax_b[ga.blocks[b].depth], gbg.blocks[b].s);
    smax_a[ga.blocks[b].depth] = std::max(smax_a[ga.blocks[b].depth], ga.blocks[b].s);
  }
  std::vector<long long> xd(h), yd(h), xpd(h), ypd(h);
  for (int d = 0; d < h; ++d) {
    xd[d] = take((long long)n * smax_b[d]);
    yd[d] = take((long long)n * smax_b[d]);
    xpd[d] = take((long long)n * smax_a[d]);
    ypd[d] = take((long long)n * smax_a[d]);
  }
  // terms and concatenated factors of every output block
  std::vector<std::vector<Term>> terms(nb);
  std::vector<int> S(nb, 0);
  std::vector<long long> ucat(nb), vcat(nb);
  for (int b = 0; b < nb; ++b) {
    const BlockDesc &o = ga.blocks[b];
    const int d = o.depth, j = (b / 2) - ((1 << d) - 1), c = (b % 2) + 1;
    for (int dd = d - 1; dd >= 0; --dd) {
      const int jj = j >> (d - dd);
      const int side = (j >> (d - dd - 1)) & 1;     // 0: output lies in the top half
      const int k = (1 << dd) - 1 + jj;
      Term t{0, 2 * k + side, 2 * k + (1 - side), 2 * k + side, ga.blocks[2 * k + side].s};
      if (t.cols > 0 && gbg.blocks[t.b_block].s > 0) terms[b].push_back(t);
    }
    (void)c;
    if (gbg.blocks[b].s > 0) terms[b].push_back(Term{1, b, b, -1, gbg.blocks[b].s});
    if (ga.blocks[b].s > 0) terms[b].push_back(Term{2, b, b, -1, ga.blocks[b].s});
    for (auto &t : terms[b]) S[b] += t.cols;
    ucat[b] = take((long long)o.m * std::max(S[b], 1));
    vcat[b] = take((long long)o.n * std::max(S[b], 1));
  }
  // recompression jobs, one per output block
  std::vector<RecompJob> jobs(nb);
  for (int b = 0; b < nb; ++b) {
    const BlockDesc &o = ga.blocks[b];
    RecompJob &j = jobs[b];
    j.m = o.m;
    j.n = o.n;
    j.S = S[b];
    j.u = ucat[b];
    j.v = vcat[b];
    const int mn = std::min(o.m, o.n);
    j.dense = mn > 0 && S[b] >= mn && mn <= dense_max;
  }
  const int max_c = recomp_layout(jobs, take);
  // diagonal leaves: products and ancestor intermediates T = U_A[rows] core
  std::vector<long long> leaf_out(nleaf), tmat;
  std::vector<std::vector<std::pair<int, long long>>> leaf_terms(nleaf);
  for (int i = 0; i < nleaf; ++i) {
    const int m = ga.leaf_m[i];
    leaf_out[i] = take((long long)m * m);
    for (int dd = h - 1; dd >= 0; --dd) {
      const int jj = i >> (h - dd);
      const int side = (i >> (h - dd - 1)) & 1;
      const int k = (1 << dd) - 1 + jj;
      if (ga.blocks[2 * k + side].s == 0 || gbg.blocks[2 * k + 1 - side].s == 0) continue;
      leaf_terms[i].push_back({2 * k + side, take((long long)m * gbg.blocks[2 * k + 1 - side].s)});
    }
  }
  double *work = dev_alloc(ws, s);
  HB_CUDA(cudaMemsetAsync(work, 0, ws * sizeof(double), s));
  GemmBases gb{};
  gb.p[kA] = A.arena;
  gb.p[kB] = B.arena;
  gb.p[kWork] = work;
  gb.p[kOut] = work;
  gb.p[4] = work;
  gb.p[5] = work;

  // ---- 1. cores -------------------------------------------------------------------
  {
    GemmBatch g;
    for (int k = 0; k < ninternal; ++k)
      for (int side = 0; side < 2; ++side) {
        const BlockDesc &a = ga.blocks[2 * k + side];
        const BlockDesc &bb = gbg.blocks[2 * k + 1 - side];
        if (a.s == 0 || bb.s == 0) continue;
        // V_A^T (s_a x len) U_B (len x s_b), len = the half both blocks share
        int p = g.add(kWork, core_off[2 * k + side], a.s, a.s, bb.s);
        g.seg(p, kA, a.v_off, a.n, 1, kB, bb.u_off, bb.m, 0, a.n);
      }
    gemm_f64_run(g, gb, TileShape::M64N128, s);
  }

  // ---- 2. subtree products per depth ------------------------------------------------
  for (int d = 0; d < h; ++d) {
    std::vector<CopyDesc> cp;
    for (int j = 0; j < (1 << d); ++j)
      for (int c = 1; c <= 2; ++c) {
        const int b = block_index(d, j, c);
        const BlockDesc &bo = gbg.blocks[b];   // rows of this block = the subtree's rows
        const BlockDesc &ao = ga.blocks[b];
        if (bo.s > 0)
          cp.push_back(CopyDesc{B.arena + bo.u_off, bo.m, work + xd[d] + bo.r0, n, bo.m, bo.s});
        // the other side: V_A of the mirrored block, placed at its columns' rows
        if (ao.s > 0)
          cp.push_back(CopyDesc{A.arena + ao.v_off, ao.n, work + xpd[d] + ao.c0, n, ao.n, ao.s});
      }
    run_copies(cp, s);
    if (smax_b[d] > 0) {
      if (mixed)
        product_mixed_op(A, ProdOp::N, work + xd[d], smax_b[d], n, work + yd[d], n, s, d + 1);
      else
        product_f64(A, ProdOp::N, work + xd[d], smax_b[d], n, work + yd[d], n, s, d + 1);
    }
    if (smax_a[d] > 0) {
      if (mixed)
        product_mixed_op(B, ProdOp::T, work + xpd[d], smax_a[d], n, work + ypd[d], n, s, d + 1);
      else
        product_f64(B, ProdOp::T, work + xpd[d], smax_a[d], n, work + ypd[d], n, s, d + 1);
    }
  }

  // ---- 3. concatenated factors ---------------------------------------------------------
  {
    std::vector<CopyDesc> cp;
    GemmBatch gv;
    for (int b = 0; b < nb; ++b) {
      const BlockDesc &o = ga.blocks[b];
      long long col = 0;
      for (const Term &t : terms[b]) {
        double *u = work + ucat[b] + col * o.m;
        double *v = work + vcat[b] + col * o.n;
        if (t.kind == 0) {
          const BlockDesc &a = ga.blocks[t.a_block];
          const BlockDesc &bb = gbg.blocks[t.b_block];
          cp.push_back(CopyDesc{A.arena + a.u_off + (o.r0 - a.r0), a.m, u, o.m, o.m, a.s});
          // V_B[cols] core^T : (n x s_b) (s_b x s_a)
          int p = gv.add(kWork, vcat[b] + col * o.n, o.n, o.n, a.s);
          gv.seg(p, kB, bb.v_off + (o.c0 - bb.c0), bb.n, 0, kWork, core_off[t.core], a.s, 1,
                 bb.s);
        } else if (t.kind == 1) {
          const BlockDesc &bb = gbg.blocks[b];
          // (A subtree) U_B sits in Y_d at the block's rows; V_B as is
          cp.push_back(CopyDesc{work + yd[o.depth] + o.r0, n, u, o.m, o.m, bb.s});
          cp.push_back(CopyDesc{B.arena + bb.v_off, bb.n, v, o.n, o.n, bb.s});
        } else {
          const BlockDesc &a = ga.blocks[b];
          // U_A as is; (B subtree)^T V_A sits in Y'_d at the block's columns
          cp.push_back(CopyDesc{A.arena + a.u_off, a.m, u, o.m, o.m, a.s});
          cp.push_back(CopyDesc{work + ypd[o.depth] + o.c0, n, v, o.n, o.n, a.s});
        }
        col += t.cols;
      }
    }
    run_copies(cp, s);
    gemm_f64_run(gv, gb, TileShape::M128N64, s, false);
  }

  // ---- 4. recompression ----------------------------------------------------------------
  const std::vector<int> ranks = recomp_run(jobs, work, tol, max_c, s, status);

  // ---- 5. diagonal leaves ----------------------------------------------------------------
  {
    GemmBatch gt;   // T = U_A[rows] core
    for (int i = 0; i < nleaf; ++i)
      for (auto &lt : leaf_terms[i]) {
        const BlockDesc &a = ga.blocks[lt.first];
        const int kb = lt.first;
        const int m = ga.leaf_m[i];
        const int sb = core_n[kb];
        int p = gt.add(kWork, lt.second, m, m, sb);
        gt.seg(p, kA, a.u_off + (ga.leaf_off[i] - a.r0), a.m, 0, kWork, core_off[kb], a.s, 0, a.s);
      }
    gemm_f64_run(gt, gb, TileShape::M128N64, s);
    GemmBatch gl;   // leaf = D_A D_B + sum T V_B[cols]^T
    for (int i = 0; i < nleaf; ++i) {
      const int m = ga.leaf_m[i];
      if (m == 0) continue;
      int p = gl.add(kWork, leaf_out[i], m, m, m);
      gl.seg(p, kA, A.leaves[i].off, m, 0, kB, B.leaves[i].off, m, 0, m);
      for (auto &lt : leaf_terms[i]) {
        const int kb = lt.first;
        const int bb_index = (kb % 2 == 0) ? kb + 1 : kb - 1;
        const BlockDesc &bb = gbg.blocks[bb_index];
        gl.seg(p, kWork, lt.second, m, 0, kB, bb.v_off + (ga.leaf_off[i] - bb.c0), bb.n, 1, bb.s);
      }
    }
    gemm_f64_run(gl, gb, TileShape::M128N64, s, false);
  }

  // ---- 6. output tree ----------------------------------------------------------------------
  Geometry go = ga;
  for (int b = 0; b < nb; ++b) go.blocks[b].s = ranks[b];
  std::shared_ptr<DeviceTree> out = dtree_create(go, s);
  std::vector<CopyDesc> cp;
  for (int i = 0; i < nleaf; ++i) {
    const int m = go.leaf_m[i];
    if (m) cp.push_back(CopyDesc{work + leaf_out[i], m, out->arena + out->leaves[i].off, m, m, m});
  }
  run_copies(cp, s);
  std::vector<long long> uo(nb), vo(nb);
  for (int b = 0; b < nb; ++b) {
    uo[b] = out->g.blocks[b].u_off;
    vo[b] = out->g.blocks[b].v_off;
  }
  recomp_finish(jobs, ranks, work, out->arena, uo, vo, s);
  HB_CUDA(cudaStreamSynchronize(s));
  dev_free(work, s);
  HB_CUDA(cudaStreamSynchronize(s));
  return out;
}

int recompress_one(int m, int n, int S, const double *d_u, int ldu, const double *d_v, int ldv,
                   double tol, bool dense, double *d_uo, double *d_vo, int *rank,
                   cudaStream_t s) {
  HB_REQUIRE(m >= 0 && n >= 0 && S >= 0 && ldu >= std::max(m, 1) && ldv >= std::max(n, 1),
             INPUT_ERROR, "recompress: negative size or leading dimension below the rows");
  *rank = 0;
  if (std::min(m, n) == 0 || S == 0) return SUCCESS;
  HB_REQUIRE(d_u && d_v && d_uo && d_vo, INPUT_ERROR, "recompress: NULL buffer");
  long long ws = 0;
  auto take = [&](long long e) {
    const long long o = ws;
    ws += align_up(std::max<long long>(e, 1));
    return o;
  };
  std::vector<RecompJob> jobs(1);
  RecompJob &j = jobs[0];
  j.m = m;
  j.n = n;
  j.S = S;
  j.dense = dense;
  j.u = take((long long)m * S);
  j.v = take((long long)n * S);
  const int max_c = recomp_layout(jobs, take);
  const int cap = std::max(S, std::min(m, n));
  const long long uo = take((long long)m * cap), vo = take((long long)n * cap);
  double *work = dev_alloc(ws, s);
  HB_CUDA(cudaMemsetAsync(work, 0, ws * sizeof(double), s));
  HB_CUDA(cudaMemcpy2DAsync(work + j.u, sizeof(double) * m, d_u, sizeof(double) * ldu,
                            sizeof(double) * m, S, cudaMemcpyDeviceToDevice, s));
  HB_CUDA(cudaMemcpy2DAsync(work + j.v, sizeof(double) * n, d_v, sizeof(double) * ldv,
                            sizeof(double) * n, S, cudaMemcpyDeviceToDevice, s));
  int status = SUCCESS;
  const std::vector<int> ranks = recomp_run(jobs, work, tol, max_c, s, &status);
  recomp_finish(jobs, ranks, work, work, {uo}, {vo}, s);
  *rank = ranks[0];
  if (ranks[0] > 0) {
    HB_CUDA(cudaMemcpyAsync(d_uo, work + uo, sizeof(double) * (size_t)m * ranks[0],
                            cudaMemcpyDeviceToDevice, s));
    HB_CUDA(cudaMemcpyAsync(d_vo, work + vo, sizeof(double) * (size_t)n * ranks[0],
                            cudaMemcpyDeviceToDevice, s));
  }
  HB_CUDA(cudaStreamSynchronize(s));
  dev_free(work, s);
  return status;
}

}  // namespace hb
