/*
 * A plain C caller of hmat_lib's public API, compiled with gcc against
 * the headers of include/hmat_lib and linked to libhodlr_b200.so instead of hmat_lib:
 * the drop-in swap a C user makes (same headers, same calls, same ownership:
 * results returned for out == NULL are the caller's to free()).
 *
 * It follows hmat_lib's own calling pattern (allocate a tree, build it from a
 * dense matrix that the constructor may overwrite, multiply, free) on a
 * Gaussian kernel matrix of sorted points, and checks every product against a
 * naive dense product computed here.  Prints one line per check; exits 0
 * only if all pass.
 *
 *   cc -std=c11 -I include tests/c_dropin_caller.c -L hmat_lib_b200 \
 *      -lhodlr_b200 -Wl,-rpath,hmat_lib_b200 -lm && ./a.out
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "hmat_lib/allocators.h"
#include "hmat_lib/constructors.h"
#include "hmat_lib/dense_algebra.h"
#include "hmat_lib/error.h"
#include "hmat_lib/hodlr.h"
#include "hmat_lib/hodlr_algebra.h"
#include "hmat_lib/utils.h"
#include "hmat_lib/vector_algebra.h"

static int failures = 0;

static void check(const char *what, double err, double bound) {
  const int ok = err <= bound;
  printf("%-34s rel err %.3e (bound %.0e) %s\n", what, err, bound, ok ? "ok" : "FAIL");
  if (!ok) failures++;
}

/* relative Frobenius difference of two m x k column-major arrays */
static double rel_diff(int m, int k, const double *a, int lda, const double *b, int ldb) {
  double num = 0.0, den = 0.0;
  for (int j = 0; j < k; j++)
    for (int i = 0; i < m; i++) {
      const double d = a[i + (size_t)j * lda] - b[i + (size_t)j * ldb];
      num += d * d;
      den += b[i + (size_t)j * ldb] * b[i + (size_t)j * ldb];
    }
  return sqrt(num / den);
}

/* C = A B (A m x p, B p x k), column-major */
static void gemm(int m, int p, int k, const double *a, const double *b, double *c) {
  for (int j = 0; j < k; j++) {
    for (int i = 0; i < m; i++) c[i + (size_t)j * m] = 0.0;
    for (int l = 0; l < p; l++) {
      const double blj = b[l + (size_t)j * p];
      for (int i = 0; i < m; i++) c[i + (size_t)j * m] += a[i + (size_t)l * m] * blj;
    }
  }
}

/* stored doubles of a tree, walking its structs as a C caller would */
static long storage(const struct TreeHODLR *t) {
  long total = 0;
  const long nleaf = 1L << t->height;
  for (long i = 0; i < nleaf; i++) {
    const int m = t->innermost_leaves[i]->data.diagonal.m;
    total += (long)m * m;
  }
  /* internal nodes breadth first from the root */
  const struct HODLRInternalNode **q = malloc(sizeof(*q) * (size_t)nleaf);
  long head = 0, tail = 0;
  q[tail++] = t->root;
  for (int d = 0; d < t->height; d++) {
    const long count = tail - head;
    for (long c = 0; c < count; c++) {
      const struct HODLRInternalNode *node = q[head++];
      for (int ch = 1; ch <= 2; ch++) {
        const struct NodeOffDiagonal *od = &node->children[ch].leaf->data.off_diagonal;
        total += (long)od->s * (od->m + od->n);
      }
      if (d + 1 < t->height) {
        q[tail++] = node->children[0].internal;
        q[tail++] = node->children[3].internal;
      }
    }
    /* compact the queue */
    memmove(q, q + head, sizeof(*q) * (size_t)(tail - head));
    tail -= head;
    head = 0;
  }
  free(q);
  return total;
}

int main(void) {
  const int n = 2048, height = 4, k = 5;
  const double tol = 1e-10;
  int ierr = -1;

  /* Gaussian kernel exp(-(x_i - x_j)^2 / (2 0.2^2)) + I on sorted points */
  double *x = malloc(sizeof(double) * n);
  srand(11);
  for (int i = 0; i < n; i++) x[i] = (double)rand() / RAND_MAX;
  for (int i = 1; i < n; i++) {      /* insertion sort */
    const double v = x[i];
    int j = i - 1;
    while (j >= 0 && x[j] > v) { x[j + 1] = x[j]; j--; }
    x[j + 1] = v;
  }
  double *a = malloc(sizeof(double) * (size_t)n * n);
  for (int j = 0; j < n; j++)
    for (int i = 0; i < n; i++) {
      const double d = x[i] - x[j];
      a[i + (size_t)j * n] = exp(-d * d / (2.0 * 0.2 * 0.2)) + (i == j ? 1.0 : 0.0);
    }
  double *a_keep = malloc(sizeof(double) * (size_t)n * n);
  memcpy(a_keep, a, sizeof(double) * (size_t)n * n);

  struct TreeHODLR *h = allocate_tree_monolithic(height, &ierr);
  if (h == NULL || ierr != SUCCESS) { printf("allocate_tree_monolithic failed: %d\n", ierr); return 1; }
  const int info = dense_to_tree_hodlr(h, n, NULL, a, tol, &ierr);
  if (ierr != SUCCESS || info != 0) { printf("dense_to_tree_hodlr failed: %d\n", ierr); return 1; }
  const int top_rank = h->root->children[1].leaf->data.off_diagonal.s;
  const int highest = get_highest_s(h);
  const long stored = storage(h);
  printf("built n=%d height=%d: root block rank %d, highest rank %d, %ld stored doubles\n", n,
         height, top_rank, highest, stored);
  if (highest < top_rank || top_rank < 1) { printf("rank query FAIL\n"); failures++; }
  if (compute_multiply_hodlr_dense_workspace(h, k) != highest * k) {
    printf("workspace size FAIL\n");
    failures++;
  }

  /* H v, result allocated by the library (out == NULL) */
  double *v = malloc(sizeof(double) * n);
  for (int i = 0; i < n; i++) v[i] = sin(0.37 * i);
  double *hv = multiply_vector(h, v, NULL, &ierr);
  if (hv == NULL || ierr != SUCCESS) { printf("multiply_vector failed: %d\n", ierr); return 1; }
  double *av = malloc(sizeof(double) * n);
  gemm(n, n, 1, a_keep, v, av);
  check("multiply_vector", rel_diff(n, 1, hv, n, av, n), 1e-9);
  free(hv);

  /* H X, H^T X and X H with leading dimensions larger than the sizes */
  const int ldx = n + 3;
  double *xm = malloc(sizeof(double) * (size_t)ldx * n);
  for (size_t i = 0; i < (size_t)ldx * n; i++) xm[i] = cos(0.011 * (double)i);
  double *ref = malloc(sizeof(double) * (size_t)n * k);
  double *xc = malloc(sizeof(double) * (size_t)n * k);
  for (int j = 0; j < k; j++) memcpy(xc + (size_t)j * n, xm + (size_t)j * ldx, sizeof(double) * n);
  double *out = malloc(sizeof(double) * (size_t)ldx * k);
  if (multiply_hodlr_dense(h, xm, k, ldx, out, ldx, &ierr) != out || ierr != SUCCESS) {
    printf("multiply_hodlr_dense failed: %d\n", ierr);
    return 1;
  }
  gemm(n, n, k, a_keep, xc, ref);
  check("multiply_hodlr_dense", rel_diff(n, k, out, ldx, ref, n), 1e-9);
  /* the kernel matrix is symmetric, so H^T X approximates A X as well */
  double *outt = multiply_hodlr_transpose_dense(h, xm, k, ldx, NULL, ldx, &ierr);
  if (outt == NULL || ierr != SUCCESS) { printf("multiply_hodlr_transpose_dense failed\n"); return 1; }
  check("multiply_hodlr_transpose_dense", rel_diff(n, k, outt, ldx, ref, n), 1e-9);
  free(outt);
  /* X H with X k x n (ld k + 2): compare (X A) against the transposed A X^T */
  const int ldl = k + 2;
  double *xl = malloc(sizeof(double) * (size_t)ldl * n);
  for (int j = 0; j < n; j++)
    for (int i = 0; i < ldl; i++) xl[i + (size_t)j * ldl] = (i < k) ? xc[j + (size_t)i * n] : 0.0;
  double *outl = multiply_dense_hodlr(h, xl, k, ldl, NULL, ldl, &ierr);
  if (outl == NULL || ierr != SUCCESS) { printf("multiply_dense_hodlr failed\n"); return 1; }
  double *outl_t = malloc(sizeof(double) * (size_t)n * k);
  for (int j = 0; j < n; j++)
    for (int i = 0; i < k; i++) outl_t[j + (size_t)i * n] = outl[i + (size_t)j * ldl];
  check("multiply_dense_hodlr", rel_diff(n, k, outl_t, n, ref, n), 1e-9);
  free(outl);

  /* H H with recompression, then (H H) X against A (A X) */
  struct TreeHODLR *hh = allocate_tree(height, &ierr);
  if (hh == NULL || ierr != SUCCESS) { printf("allocate_tree failed\n"); return 1; }
  multiply_hodlr_hodlr(h, h, hh, 1e-10, &ierr);
  if (ierr != SUCCESS) { printf("multiply_hodlr_hodlr failed: %d\n", ierr); return 1; }
  double *hhx = multiply_hodlr_dense(hh, xc, k, n, NULL, n, &ierr);
  if (hhx == NULL || ierr != SUCCESS) { printf("multiply_hodlr_dense (H H) failed\n"); return 1; }
  double *aax = malloc(sizeof(double) * (size_t)n * k);
  gemm(n, n, k, a_keep, ref, aax);
  check("multiply_hodlr_hodlr", rel_diff(n, k, hhx, n, aax, n), 1e-8);
  free(hhx);

  /* errors: NULL input and out == x are INPUT_ERROR, as in hmat_lib */
  ierr = SUCCESS;
  if (multiply_vector(h, NULL, NULL, &ierr) != NULL || ierr != INPUT_ERROR) {
    printf("NULL vector not rejected FAIL\n");
    failures++;
  }
  double *same = malloc(sizeof(double) * n);
  memcpy(same, v, sizeof(double) * n);
  ierr = SUCCESS;
  if (multiply_vector(h, same, same, &ierr) != NULL || ierr != INPUT_ERROR) {
    printf("out == x not rejected FAIL\n");
    failures++;
  }

  free_tree_hodlr(&hh);
  free_tree_hodlr(&h);
  if (h != NULL) { printf("free_tree_hodlr did not clear the pointer FAIL\n"); failures++; }
  free(same); free(aax); free(outl_t); free(xl); free(out); free(xc); free(ref); free(xm);
  free(av); free(v); free(a_keep); free(a); free(x);
  printf("%s\n", failures == 0 ? "ALL OK" : "FAILED");
  return failures == 0 ? 0 : 1;
}
