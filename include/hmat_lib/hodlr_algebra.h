/* HODLR x HODLR with recompression (hmat_lib
 * include/hmat_lib/hodlr_algebra.h:4-10, src/hodlr_algebra.c:1452).
 * `out` must be an allocated, empty tree of the same height. */
#pragma once

#ifdef __cplusplus
extern "C" {
#endif

struct TreeHODLR;

int multiply_hodlr_hodlr(
  const struct TreeHODLR *hodlr1,
  const struct TreeHODLR *hodlr2,
  struct TreeHODLR *out,
  const double svd_threshold,
  int *ierr
);

#ifdef __cplusplus
}
#endif
