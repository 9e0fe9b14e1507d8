// Dense -> HODLR construction on the device.
#pragma once

#include "dtree.h"

namespace hb {

struct BuildStats {
  int exact_blocks = 0;        // blocks compressed by full Jacobi SVD
  int sketched_blocks = 0;     // blocks compressed by the randomized path
  int sketch_rounds = 0;       // adaptive growth rounds of the randomized path
  double seconds = 0.0;
  int cap_hit = 0;             // a sketch reached its column cap
  int max_sweeps_exact = 0, max_sweeps_sketch = 0;
  int failed_exact = 0, failed_sketch = 0;
  int max_sketch = 0;          // largest sketch (columns)
};

// Statistics of the most recent build on the calling thread.
const BuildStats &last_build_stats();

// Compresses every off-diagonal block of the n x n matrix d_A (ld lda, device)
// following the block sizes of `g` (ranks ignored) with hmat_lib's relative
// truncation rule at `tol`.  `svd_status` receives SUCCESS or SVD_FAILURE.
std::shared_ptr<DeviceTree> build_from_dense(const Geometry &g, const double *d_A, long long lda,
                                             double tol, cudaStream_t stream, int *svd_status,
                                             BuildStats *stats = nullptr);

}  // namespace hb
