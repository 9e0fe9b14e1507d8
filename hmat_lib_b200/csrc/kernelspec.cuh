// Kernel matrices defined by a point set: A_ij = k(|p_i - p_j|) + diag
// delta_ij.  The same device function fills a dense matrix
// (hodlr_b200_kernel_matrix_dev) and feeds the matrix-free build, where the
// GEMM loaders, the Jacobi initialisation and the leaf copies compute the
// entries they need instead of reading them.
#pragma once

#include "common.h"

namespace hb {

struct KernelSpec {
  const double *pts = nullptr;   // n x dim, column-major: coordinate a of point i at pts[i + a n]
  int n = 0, dim = 0;
  int kind = 0;                  // 0 Gaussian, 1 Matern-3/2, 2 exponential
  double length = 1.0, diag = 0.0;
};

#ifdef __CUDACC__
__device__ __forceinline__ double kernel_entry(const KernelSpec &K, int i, int j) {
  double r2 = 0.0;
  for (int a = 0; a < K.dim; ++a) {
    const double d = K.pts[i + (long long)a * K.n] - K.pts[j + (long long)a * K.n];
    r2 = fma(d, d, r2);
  }
  const double r = sqrt(r2);
  double v;
  if (K.kind == 0) {
    v = exp(-r2 / (2.0 * K.length * K.length));          // Gaussian
  } else if (K.kind == 1) {
    const double t = 1.7320508075688772 * r / K.length;   // Matern-3/2
    v = (1.0 + t) * exp(-t);
  } else {
    v = exp(-r / K.length);                               // exponential
  }
  if (i == j) v += K.diag;
  return v;
}
#endif

// Base slot of a generated GEMM operand: its offset packs the block's first
// row (high 32 bits) and first column (low 32 bits) in the kernel matrix.
constexpr unsigned char kGenSlot = 255;
inline long long gen_offset(int row0, int col0) {
  return ((long long)row0 << 32) | (unsigned int)col0;
}

}  // namespace hb
