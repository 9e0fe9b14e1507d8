// Block one-sided Jacobi SVD for wide square problems: the sketched cores of
// the build, up to thousands of columns (hmat_lib runs LAPACK dgesdd on the
// whole block instead, src/lapack_wrapper.c:8-59).
#pragma once

#include <vector>

#include "common.h"

namespace hb {

// One problem: the L x L matrix A with element (i, j) at A[j + i lda] (the
// transpose of a column-major L x L matrix, as the build stores its cores).
struct BjProb {
  const double *A;
  long long lda;
  int L;
  double *U;       // out: L x L (ld L), left vectors times sigma, descending sigma
  double *V;       // out: L x L (ld L), right vectors
  double *sigma;   // out: L singular values, descending
  int *rank;       // out (device int): hmat_lib's relative truncation rank
  int *sweeps;     // out (device int, optional): sweeps used; max_sweeps + 1 if not converged
};

// Columns of A are taken 32 at a time (blocks); every round pairs each block
// with another (round-robin over the blocks), and for each pair of 64 columns
// one cluster of CTAs forms the pair's Gram matrix on the FP64 tensor cores,
// diagonalises it by two-sided Jacobi in shared memory and rotates the pair's
// columns and the accumulated right rotations by its eigenvectors: one launch
// per round for all pairs of all problems, so every round streams the
// columns through all SMs instead of the pairwise rotations of the one-CTA /
// one-cluster solver, which stream the whole matrix through a few SMs.  A
// sweep ends when every block met every other; a problem stops once a whole
// sweep applied no rotation.  Pairs of columns whose norm is below
// 1e-3 tol ||A||_F / L are not rotated (the same rule as the scalar solver, so
// no kept singular value moves by more than 0.1% of the truncation
// threshold).  The rank follows hmat_lib's relative rule
// (src/constructors.c:329-336).  A problem that has not converged after
// max_sweeps sweeps sets *d_status to SVD_FAILURE.
// Synchronises with `stream`.
void block_jacobi_svd(const std::vector<BjProb> &probs, double tol, int max_sweeps,
                      int *d_status, cudaStream_t stream);

}  // namespace hb
