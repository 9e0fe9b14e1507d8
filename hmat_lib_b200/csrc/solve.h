// Direct solver for a HODLR matrix (hodlr_b200_factorize_dev /
// hodlr_b200_solve_dev).  hmat_lib has no solver; this is the step after the
// products.
//
// With A^(l) the tree restricted to its blocks of depth >= l (block diagonal
// over the subtrees rooted at depth l; A^(h) = D, the leaves) and U_l V_l^T the
// depth-l off-diagonal blocks,
//   A^(l) = A^(l+1) (I + W_l V_l^T),   W_l = (A^(l+1))^-1 U_l,
// so A = D (I + W_{h-1} V_{h-1}^T) ... (I + W_0 V_0^T) and
//   A^-1 b = (I + W_0 V_0^T)^-1 ... (I + W_{h-1} V_{h-1}^T)^-1 D^-1 b.
// Each factor is block diagonal over the depth-l nodes; for a node with
// top-right block U_tr V_tr^T and bottom-left block U_bl V_bl^T,
//   W = diag(W1, W2),  W1 = K1^-1 U_tr,  W2 = K2^-1 U_bl  (K_i: the child subtree),
//   (I + W V^T)^-1 = I - W C^-1 V^T,  C = [I, P; Q, I],
//   P = V_tr^T W2,  Q = V_bl^T W1,
// a Woodbury step with a capacitance matrix of order q = s_tr + s_bl.  With
// the Schur complement S = I - Q P,
//   C^-1 = [I + P S^-1 Q, -P S^-1; -S^-1 Q, S^-1],
// which the factor stores explicitly, so applying a level is three batched
// launches: t = V^T x, z = C^-1 t, x -= W z.
// Factorising computes the leaf inverses, then from the deepest level up W_l
// (the level's U blocks solved through the leaves and every deeper factor;
// the deeper factors act within each child's rows, so W_l is one n x max-rank
// matrix whose row bands use their own columns) and C^-1 of every node.  Every
// product is a batched launch of the segmented FP64 GEMM; S^-1 and the leaf
// inverses come from a batched Gauss-Jordan kernel with partial pivoting.
#pragma once

#include "dtree.h"

namespace hb {

struct SolvePlan;

struct HodlrFactor {
  std::shared_ptr<DeviceTree> tree;
  double *buf = nullptr;                  // leaf inverses, W of every level, C^-1 of every node
  std::vector<long long> leaf_inv_off;    // leaf i's inverse (m_i x m_i, ld m_i)
  std::vector<long long> w_off;           // per depth: W_l (n x w_cols[l], ld n)
  std::vector<int> w_cols;
  std::vector<long long> cinv_off;        // per node (index 2^d - 1 + j): C^-1 (q x q, ld q)
  std::vector<int> q;                     // per node: s_tr + s_bl
  // Launch plans and scratch of hodlr_solve, per (k, ldb, ldx, stream).
  std::map<std::tuple<int, long long, long long, cudaStream_t>, std::unique_ptr<SolvePlan>> plans;
  std::mutex plan_mutex;
  HodlrFactor();
  ~HodlrFactor();
};

// Factorises the tree; `status` receives SUCCESS or INPUT_ERROR when a leaf or
// a capacitance matrix is singular to working precision.
std::unique_ptr<HodlrFactor> hodlr_factorize(std::shared_ptr<DeviceTree> t, cudaStream_t stream,
                                             int *status);

// X = A^-1 B for k right-hand sides (device, column-major; X and B distinct).
// The first call for a (k, ldb, ldx, stream) builds its launch plans and
// scratch (synchronously); later calls only launch 1 + 3h GEMMs.
void hodlr_solve(HodlrFactor &f, const double *B, int k, long long ldb, double *X,
                 long long ldx, cudaStream_t stream);

}  // namespace hb
