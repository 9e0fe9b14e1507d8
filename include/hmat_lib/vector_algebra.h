/* HODLR x vector (hmat_lib include/hmat_lib/vector_algebra.h:3-8,
 * src/vector_algebra.c:131).  Host pointers; out == NULL makes the library
 * malloc the result, which the caller then free()s. */
#pragma once

#ifdef __cplusplus
extern "C" {
#endif

struct TreeHODLR;

double *multiply_vector(
  const struct TreeHODLR *hodlr,
  const double *vector,
  double *out,
  int *ierr
);

#ifdef __cplusplus
}
#endif
