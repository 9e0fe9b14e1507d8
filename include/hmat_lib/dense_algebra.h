/* HODLR x dense products (hmat_lib include/hmat_lib/dense_algebra.h:4-80,
 * src/dense_algebra.c).  Host pointers, column-major, leading dimensions as
 * in hmat_lib. */
#pragma once

#ifdef __cplusplus
extern "C" {
#endif

struct TreeHODLR;
struct HODLRInternalNode;

/* max rank * matrix_a (hmat_lib src/dense_algebra.c:39). */
int compute_multiply_hodlr_dense_workspace(
  const struct TreeHODLR *hodlr,
  const int matrix_a
);

/* out = H * matrix, matrix is m x matrix_n (hmat_lib src/dense_algebra.c:361). */
double *multiply_hodlr_dense(
  const struct TreeHODLR *hodlr,
  const double *matrix,
  const int matrix_n,
  const int matrix_ld,
  double *out,
  const int out_ld,
  int *ierr
);

/* out = H^T * matrix (hmat_lib src/dense_algebra.c:617). */
double *multiply_hodlr_transpose_dense(
  const struct TreeHODLR *hodlr,
  const double *matrix,
  const int matrix_n,
  const int matrix_ld,
  double *out,
  const int out_ld,
  int *ierr
);

/* out = matrix * H, matrix is matrix_m x m (hmat_lib src/dense_algebra.c:957). */
double *multiply_dense_hodlr(
  const struct TreeHODLR *hodlr,
  const double *matrix,
  const int matrix_m,
  const int matrix_ld,
  double *out,
  const int out_ld,
  int *ierr
);

/* Subtree products: `internal` is the root of a subtree of the given height;
 * `queue` and `workspace` are accepted for ABI compatibility and not used
 * (the work runs on the device).  out is overwritten.
 * (hmat_lib src/dense_algebra.c:492, 710, 1087.) */
void multiply_internal_node_dense(
  const struct HODLRInternalNode *internal,
  const int height,
  const double *matrix,
  const int matrix_n,
  const int matrix_ld,
  const struct HODLRInternalNode **queue,
  double *workspace,
  double *out,
  const int out_ld
);

void multiply_internal_node_transpose_dense(
  const struct HODLRInternalNode *internal,
  const int height,
  const double *matrix,
  const int matrix_n,
  const int matrix_ld,
  const struct HODLRInternalNode **queue,
  double *workspace,
  double *out,
  const int out_ld
);

void multiply_dense_internal_node(
  const struct HODLRInternalNode *internal,
  const int height,
  const double *matrix,
  const int matrix_m,
  const int matrix_ld,
  const struct HODLRInternalNode **queue,
  double *workspace,
  double *out,
  const int out_ld
);

#ifdef __cplusplus
}
#endif
