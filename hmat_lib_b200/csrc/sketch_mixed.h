// The build's sketch products on the int8 tensor cores: Y = A_b Omega and
// B^T = A_b^T Q for the blocks of a dense input, with the split-precision
// scheme and kernel of the mixed products (ozaki.h: six int8 slices per
// value, 21 slice products accumulated exactly in int32, FP64 recombination,
// about 42 bits).  Each block of the input is sliced once per build in both
// orientations (rows for A Omega, columns for A^T Q); the test matrices and
// the new basis columns are sliced per round.
#pragma once

#include <vector>

#include "common.h"
#include "ozaki.h"

namespace hb {

struct SketchMixedBlock {
  const double *A;   // m x n block of the input, column-major, leading dimension lda
  long long lda;
  int m, n;          // multiples of 32
};

class SketchMixed {
 public:
  SketchMixed(const std::vector<SketchMixedBlock> &blocks, cudaStream_t s);
  ~SketchMixed();
  SketchMixed(const SketchMixed &) = delete;
  SketchMixed &operator=(const SketchMixed &) = delete;

  // One product: Y (rows x w, ld ldy) = op(A_block) X with X (K x w, ld ldx);
  // op N: rows = m, K = n; op T: rows = n, K = m.
  struct Call {
    int block;
    const double *X;
    long long ldx;
    int w;
    double *Y;
    long long ldy;
  };
  // All calls of one op in one launch of the int8 kernel (plus the slicing
  // of every X).  Y is overwritten.
  void multiply(bool transA, const std::vector<Call> &calls, cudaStream_t s);
  // SVD_FAILURE if a kernel gave up waiting on a barrier since the last check.
  int status(cudaStream_t s);

 private:
  std::vector<SketchMixedBlock> blocks_;
  std::vector<long long> row_off_, col_off_;   // slice bytes of each block, both orientations
  std::vector<long long> rexp_off_, cexp_off_; // exponents of its rows / columns
  uint8_t *slices_ = nullptr;
  int *exps_ = nullptr;
  int *status_ = nullptr;
  cudaStream_t stream_ = nullptr;
  std::vector<void *> keep_;   // job arrays of launches in flight, freed with the object
};

}  // namespace hb
