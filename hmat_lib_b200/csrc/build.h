// Dense -> HODLR construction on the device.
#pragma once

#include <vector>

#include "dtree.h"
#include "kernelspec.cuh"

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
  // device time (ms) of the build's stages, from events on the build stream
  double ms_exact = 0.0;       // Jacobi SVDs of the small blocks
  double ms_rounds = 0.0;      // sketch rounds (products, orthonormalisation, decisions)
  double ms_core_svd = 0.0;    // Jacobi SVDs of the sketched cores R_B^T
  double ms_finish = 0.0;      // arena, leaf copies, U = Q U_R S, V = P V_R
  int learned_fallbacks = 0;   // one-shot sketches that failed the error check
  double ms_features = 0.0;    // rank-model features and prediction (host clock)
  double gemm_flops = 0.0;     // FP64 GEMM work of the build (2 M N K summed)
  double input_elems = 0.0;    // entries of the input matrices (n^2 per tree)
  double ms_host_setup = 0.0;  // host clock from the call to the first stage event
  double ms_host_total = 0.0;  // host clock from the call to the return
  double ms_host_plans = 0.0;  // host clock spent making GEMM and TSQR plans
};

// Statistics of the most recent build on the calling thread.
const BuildStats &last_build_stats();

// Per sketched block of the most recent build that computed features: the 8
// rank-model features, final rank, predicted rank (-1: no model), first
// sketch width, fallback flag (1: the one-shot sketch failed its error
// check), final sketch width, Frobenius epsilon-rank (fewest leading singular
// values whose discarded tail has Frobenius norm <= tol * s_0; the rank
// model's training target).
constexpr int kFeatureRow = 14;
const std::vector<float> &last_build_features();

// Compresses every off-diagonal block of the n x n matrix d_A (ld lda, device)
// following the block sizes of `g` (ranks ignored) with hmat_lib's relative
// truncation rule at `tol`.  `svd_status` receives SUCCESS or SVD_FAILURE.
// With `gen` set, the matrix is the kernel matrix it defines and is never
// formed: every entry the build needs is computed where it is used (d_A and
// lda are then ignored).
std::shared_ptr<DeviceTree> build_from_dense(const Geometry &g, const double *d_A, long long lda,
                                             double tol, cudaStream_t stream, int *svd_status,
                                             BuildStats *stats = nullptr,
                                             const KernelSpec *gen = nullptr);

// One tree of a batch build: its block sizes and its n x n input (ld lda).
struct BuildInput {
  Geometry g;
  const double *A;
  long long lda;
};

// Builds many trees at once: the blocks of every tree share the launches of
// every stage (exact Jacobi SVDs, sketch rounds, core SVDs, finishing), and
// each tree gets the same random test matrices, so the same ranks, as when
// built alone.  `svd_status` is SVD_FAILURE if any tree's build failed.  With
// `gen` the batch must hold one tree.
std::vector<std::shared_ptr<DeviceTree>> build_batch(const std::vector<BuildInput> &in,
                                                     double tol, cudaStream_t stream,
                                                     int *svd_status, BuildStats *stats = nullptr,
                                                     const KernelSpec *gen = nullptr);

}  // namespace hb
