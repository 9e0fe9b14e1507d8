// Batched tall-skinny Householder QR (TSQR) of panels of at most 32 columns,
// with the explicit orthonormal factor written over the input.
#pragma once

#include <memory>
#include <vector>

#include "common.h"

namespace hb {

constexpr int kPanel = 32;       // panel width
constexpr int kChunk = 256;      // rows per CTA-level QR

struct TsqrProb {
  double *Y;        // m x w panel (ld ldy), overwritten by Q
  long long ldy;
  int m, w;         // w <= kPanel
  double *R;        // out: w x w upper triangular (ld ldr)
  long long ldr;
};

// Q R = Y for every problem.  Rank-deficient panels still get an orthonormal
// Q (Householder), R then has (near-)zero diagonal entries.
void tsqr_batched(const std::vector<TsqrProb> &probs, cudaStream_t stream);

// The same as a reusable plan: made once for fixed panel and R addresses,
// run whenever the panels hold new values (one launch per tree level).
struct TsqrPlan;
struct TsqrPlanDeleter {
  void operator()(TsqrPlan *p) const;
};
std::unique_ptr<TsqrPlan, TsqrPlanDeleter> tsqr_plan(const std::vector<TsqrProb> &probs,
                                                     cudaStream_t stream);
void tsqr_run(const TsqrPlan &plan, cudaStream_t stream);

// Zeroes the columns of a freshly orthonormalised sketch panel whose R
// diagonal is at rounding level, |R_jj| <= rel * max_c ||Y_c||, where ||Y_c||
// are the panel's column norms before projection.  A Gaussian sketch of a
// residual of rank r < w has its r independent columns first, so these are
// the trailing columns that carry no new direction; left in place they would
// not be orthogonal to the existing basis.
struct CleanDesc {
  double *Q;
  long long ldq;
  int rows, w;
  const double *R;
  long long ldr;
  const double *prenorm2;
};
void panel_clean(const std::vector<CleanDesc> &descs, double rel, cudaStream_t stream);

// Gaussian N(0, 1) entries from a counter-based hash (splitmix64 + Box-Muller):
// entry (i, j) of matrix `id` depends only on (seed, id, i, j).
struct RandDesc {
  double *X;
  long long ld;
  int rows, cols;
  unsigned long long id;
};
void gaussian_fill(const std::vector<RandDesc> &descs, unsigned long long seed,
                   cudaStream_t stream);

// Squared column norms of many matrices: out[c] = ||X[:, c]||^2.
struct NormDesc {
  const double *X;
  long long ld;
  int rows, cols;
  double *out;
};
void column_norms2(const std::vector<NormDesc> &descs, cudaStream_t stream);

}  // namespace hb
