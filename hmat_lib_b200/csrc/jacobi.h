// Batched FP64 one-sided Jacobi SVD and batched 2-D copies.
#pragma once

#include "common.h"
#include "kernelspec.cuh"

namespace hb {

// One SVD problem.  The input block A (m x n, column-major, ld lda) is read
// only.  With R = max(m, n) and C = min(m, n) the kernel orthogonalises the C
// columns of the tall orientation in G (R x C, ld R) while accumulating the
// rotations in W (C x C, ld C).
struct JacobiProb {
  const double *A;  // element (i, j) at A[i + j lda], or A[j + i lda] if transA
  long long lda;
  int transA;
  int m, n;
  double *G;        // workspace R x C
  double *W;        // workspace C x C
  double *U;        // out: m x C, ld ldu (left vectors, times sigma if scale_u)
  long long ldu;
  double *V;        // out: n x C, ld ldv (right vectors)
  long long ldv;
  double *sigma;    // out: C singular values, descending
  int *rank;        // out: truncation rank (>= 1 unless the block is empty)
  int *sweeps;      // out (optional): sweeps used; max_sweeps + 1 if not converged
  int gen_r0 = -1;  // >= 0: A is the block of the launch's kernel matrix with origin
  int gen_c0 = 0;   //   (gen_r0, gen_c0) (element (i, j) computed, A / lda unused)
  double skip_abs = 0.0;   // pairs with a column norm at or below this are neither
                           // rotated nor tested (on top of the truncation's own rule)
  double conv_scale = 0.0; // > 0: a pair also counts as orthogonal when
                           // |g_p . g_q| <= conv_tol conv_scale max(||g_p||, ||g_q||)
};

enum class Truncation : int {
  Relative = 0,   // keep while s[k] >= tol * s[0]; one if s[0] <= tol
                  // (hmat_lib src/constructors.c:329-336)
  Absolute = 1,   // stop at the first k >= 1 with s[k] <= tol
                  // (hmat_lib src/hodlr_algebra.c:160-163, 305-308)
  None = 2,       // keep all C values
};

struct JacobiParams {
  double tol = 0.0;
  Truncation trunc = Truncation::Relative;
  int scale_u = 1;          // write U * Sigma (hmat_lib stores scaled U)
  int max_sweeps = 60;      // bounded: exceeding it sets the status word
  double conv_tol = 1e-15;  // |g_p . g_q| <= conv_tol ||g_p|| ||g_q||
  // problems without their own conv_scale take ||A||_F: a pair also counts as
  // orthogonal when |g_p . g_q| <= conv_tol ||A||_F max(||g_p||, ||g_q||)
  int norm_stop = 0;
};

// Workspace doubles needed by problem (m, n): G + W.
inline long long jacobi_workspace(int m, int n) {
  const long long R = m > n ? m : n, C = m < n ? m : n;
  return align_up(R * C) + align_up(C * C);
}

// status: device int, set to SVD_FAILURE by any problem that did not
// converge within max_sweeps (left untouched otherwise).
void jacobi_svd_batched(const JacobiProb *d_probs, int nprobs, const JacobiParams &prm,
                        int *d_status, int max_c, cudaStream_t stream,
                        const KernelSpec &gen = KernelSpec());

struct CopyDesc {
  const double *src;
  long long lds;
  double *dst;
  long long ldd;
  int rows, cols;
};

void copy2d_batched(const CopyDesc *d_descs, int n, cudaStream_t stream);

// dst += alpha * src for every descriptor (same shape rules as CopyDesc).
void add2d_batched(const CopyDesc *d_descs, int n, double alpha, cudaStream_t stream);

}  // namespace hb
