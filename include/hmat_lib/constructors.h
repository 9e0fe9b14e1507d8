/* Dense -> HODLR construction (hmat_lib include/hmat_lib/constructors.h:3-14,
 * src/constructors.c:629).  The compression runs on the GPU; `matrix` is a
 * host pointer to an m x m column-major matrix.  Unlike hmat_lib the input is
 * left unchanged (hmat_lib documents it as overwritten, so callers may not
 * rely on its contents afterwards either way). */
#pragma once

#ifdef __cplusplus
extern "C" {
#endif

struct TreeHODLR;

int dense_to_tree_hodlr(
  struct TreeHODLR *hodlr,
  const int m,
  const int *ms,
  double *matrix,
  const double svd_threshold,
  int *ierr
);

#ifdef __cplusplus
}
#endif
