// HODLR x dense products on the device (FP64).
#pragma once

#include <string>

#include "dtree.h"

namespace hb {

enum class ProdOp : int {
  N = 0,  // Y = H X        (hmat_lib src/dense_algebra.c:361)
  T = 1,  // Y = H^T X      (hmat_lib src/dense_algebra.c:617)
  L = 2,  // Y = X H        (hmat_lib src/dense_algebra.c:957), X is k x n
};

enum class Precision : int {
  FP64 = 0,     // DFMA throughout
  MIXED = 1,    // split-precision tensor-core products (products_mixed.cu)
};

// Two launches per product: phase 1 projects the input onto every block's
// factor (W_b = V_b^T X_b, split along the long dimension with atomics);
// phase 2 writes each output row band once, accumulating the leaf product and
// one U_b W_b term per level in registers.
struct ProductPlan {
  ProdOp op = ProdOp::N;
  int k = 0;
  long long ldx = 0, ldy = 0;
  GemmPlan phase1, phase2;
  double *w = nullptr;            // sum_b s_b k doubles of projected input
  long long w_elems = 0;
  ProductPlan() = default;
  ProductPlan(const ProductPlan &) = delete;
  ProductPlan &operator=(const ProductPlan &) = delete;
  ~ProductPlan();
};

// Algorithmic traffic / work of one product (for roofline reporting).
struct ProductWork {
  double elements;   // sum m_leaf^2 + sum s (m + n)
  double flops;      // 2 k elements
  double bytes;      // 8 elements + 16 n k
};
ProductWork product_work(const DeviceTree &t, int k);

// Runs Y = op(H, X) with X, Y device pointers (column-major, ld given).
// With min_depth > 0 only the diagonal leaves and the off-diagonal blocks of
// depth >= min_depth take part: the block-diagonal product of all subtrees
// rooted at that depth (used by HODLR x HODLR).
void product_f64(DeviceTree &t, ProdOp op, const double *X, int k, long long ldx, double *Y,
                 long long ldy, cudaStream_t stream, int min_depth = 0);
// The same, always launched directly (product_f64 replays a captured graph
// when a call repeats an earlier one's tree, op, sizes, buffers and stream).
void product_f64_direct(DeviceTree &t, ProdOp op, const double *X, int k, long long ldx,
                        double *Y, long long ldy, cudaStream_t stream, int min_depth = 0);

// Mixed-precision Y = H X (op N) on the int8 tensor cores (products_mixed.cu).
// With min_depth > 0 only the leaves and the blocks of depth >= min_depth
// take part (as for product_f64).
void product_mixed(DeviceTree &t, const double *X, int k, long long ldx, double *Y,
                   long long ldy, cudaStream_t stream, int min_depth = 0);
// Mixed-precision Y = op(H, X) for every op: H^T X is the op-N product of the
// cached transposed tree (leaves D^T, each block the transpose of its
// sibling), X H = (H^T X^T)^T with X and the result transposed through
// device scratch.
void product_mixed_op(DeviceTree &t, ProdOp op, const double *X, int k, long long ldx,
                      double *Y, long long ldy, cudaStream_t stream, int min_depth = 0);
// Error word of the tree's mixed-precision kernels (0: none), read and reset.
int mixed_status(DeviceTree &t, cudaStream_t stream);

// Mixed-precision products of many trees with one launch per step (each
// tree at most once per batch: the tree's cached scratch is reused).
struct MixedItem {
  DeviceTree *t;
  const double *X;
  int k;
  long long ldx;
  double *Y;
  long long ldy;
};
struct MixedBatch;
struct MixedBatchDeleter {
  void operator()(MixedBatch *b) const;
};
std::unique_ptr<MixedBatch, MixedBatchDeleter> mixed_batch_build(const std::vector<MixedItem> &items,
                                                                 cudaStream_t stream);
void mixed_batch_run(MixedBatch &b, cudaStream_t stream);
int mixed_batch_status(MixedBatch &b, cudaStream_t stream);

// Y_i = op(H_i) X_i for every i with one launch per phase (batched.cu).
void batched_product(const std::vector<std::shared_ptr<DeviceTree>> &trees, ProdOp op,
                     Precision prec, const std::vector<const double *> &X,
                     const std::vector<int> &k, const std::vector<long long> &ldx,
                     const std::vector<double *> &Y, const std::vector<long long> &ldy,
                     cudaStream_t stream);
int batched_status();            // worst error word of the cached mixed batches (read, reset)
std::string batched_tuning();    // configuration the autotuner chose for the latest plan
void batched_release();          // drops every cached batch plan

// Events around the two phases of a product when option
// "record_phase_times" is set (mark(1) after phase 1, mark(2) at the end),
// and optionally around the main GEMM launch of each phase (kernel(p, false)
// just before it, kernel(p, true) just after) when a phase also runs other
// kernels.
struct PhaseTimer {
  cudaStream_t stream;
  bool on = false;
  bool kmarks = false;
  cudaEvent_t e[3] = {};
  cudaEvent_t k[4] = {};
  explicit PhaseTimer(cudaStream_t s);
  void kernel(int phase, bool end);
  void mark(int i);
};

// Accumulated per-phase device times (ms) of products run with option
// "record_phase_times" set: out[0] phase 1, out[1] phase 2, out[2] count,
// out[3] / out[4] the GEMM launch of phase 1 / 2 alone.  Resets the
// accumulators.
int phase_times(double *out, int cap);

// y = H x for one vector (op N) by the dedicated projection and row kernels
// (matvec.cu); y and x distinct, both of length n.
void matvec_f64(DeviceTree &t, const double *x, double *y, cudaStream_t stream);

// Base slots and element offsets of one product's operands inside a GEMM
// batch: a single tree uses its own slots with zero offsets; a batch of trees
// addresses every operand from one common base.
struct ProductSlots {
  int arena, x, y, w;
  long long arena_off, x_off, y_off, w_off;
};

// Appends one product's phase-1 and phase-2 problems (W laid out by w_off).
void append_product(GemmBatch &p1, GemmBatch &p2, const DeviceTree &t, ProdOp op, int k,
                    long long ldx, long long ldy, const ProductSlots &slots,
                    const std::vector<long long> &w_off, int min_depth = 0);
// Offsets of every block's W (s_b x k, or k x s_b for op L); returns the total.
long long product_w_layout(const DeviceTree &t, int k, std::vector<long long> &w_off);
// Tile shape used by the single-tree product for a phase (1 or 2).
TileShape default_shape(ProdOp op, int k, int phase);

// Builds (and caches on the tree) the plan for this shape without running it.
ProductPlan &product_plan(DeviceTree &t, ProdOp op, int k, long long ldx, long long ldy,
                          cudaStream_t stream, int min_depth = 0);

}  // namespace hb
