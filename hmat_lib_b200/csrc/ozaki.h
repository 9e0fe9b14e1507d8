// Mixed-precision products on the 5th-generation tensor cores: FP64 matrices
// split into int8 slices, products of slices accumulated exactly in int32 by
// tcgen05.mma kind::i8, recombined in FP64.
//
// Splitting (error-free, after Ozaki et al., "Error-free transformations of
// matrix multiplication by using fast routines of matrix multiplication and
// its applications", Numer. Algorithms 2012, with integer slices): each row r
// of A is scaled by 2^-e_r so that |A_rk 2^-e_r| <= 127/128, then written as
// sum_p a^(p) 2^(-7p) with integers a^(1) in [-127, 127] and a^(p) in
// [-64, 64] for p > 1 (round to nearest at every step, so each slice carries
// 7 new bits); columns of B likewise with 2^-f_j.  Then
//   (A B)_rj ~= 2^(e_r + f_j) sum_{t=2}^{S+1} 2^(-7t) sum_{p+q=t} (a^(p) b^(q))_rj
// keeping the S(S+1)/2 slice products with p + q <= S + 1.  Each inner sum is
// one int32 TMEM accumulator (exact: |sum| < 2^31 for K <= 8192).  With S = 6
// the truncation error is about 2^-42 relative to |A_r|_max |B_j|_max per term.
#pragma once

#include <cstdint>
#include <vector>

#include "common.h"

namespace hb {

constexpr int kOzSlices = 6;         // S
constexpr int kOzM = 128;            // tile rows (one MMA M)
constexpr int kOzN = 64;             // tile columns (one MMA N)
constexpr int kOzKStage = 64;        // K bytes per pipeline stage (2 MMA k-steps of 32)
constexpr int kOzStages = 3;
constexpr int kOzMaxK = 8192;        // K per tile and segment, keeps int32 exact

// int8 slices of one operand: slice p at base + p * slice_stride; element
// (row, k) of an A-type operand at row * ld + k (rows K-major); element
// (col, k) of a B-type operand at col * ld + k.  One exponent per row (A) or
// column (B).
struct OzOperand {
  const int8_t *base;
  long long slice_stride;
  int ld;
  const int *exp;
};

// One K segment of a tile: A rows [0, rows) and B columns [0, cols) relative
// to the descriptors' bases, K in [0, K) (K a multiple of 32; the slices are
// zero-padded up to it).
struct OzSeg {
  OzOperand a, b;
  int K;
};

struct OzTile {
  int seg0, nseg;
  int rows, cols;   // valid extent of the output tile (<= 128 x 64)
  long long c_off;  // output tile origin (column-major) relative to the launch's base
  long long ldc;
  int atomic;       // 1: atomically add into C (split K)
};

// Runs the tiles (one CTA each).  `status` (device int) receives
// SVD_FAILURE-style error code 1 if a bounded barrier wait ran out.
void ozaki_gemm(const OzSeg *d_segs, const OzTile *d_tiles, int ntiles, double *cbase,
                int *d_status, cudaStream_t stream);

// Slicing.  `rowwise`: scale and slice the rows of a column-major m x k
// matrix, write row-major slices (ld kpad) -> an A-type operand.
// `colwise`: scale and slice the columns -> column-contiguous slices (ld
// mpad) for a B-type operand, or for an A-type operand whose rows are the
// columns (V^T).  shift: extra power of two applied to every value (exact).
struct SliceJob {
  const double *src;
  long long ld;
  int m, k;          // source rows, columns
  int8_t *dst;
  long long slice_stride;
  int dld;           // destination leading dimension (kpad for rowwise, mpad for colwise)
  int *exp;          // exponents: m (rowwise) or k (colwise)
  int rowwise;
};
void ozaki_slice(const std::vector<SliceJob> &jobs, cudaStream_t stream);

}  // namespace hb
