/*
 * A C program written against the reference's public API as a user of
 * gooseberry would (include/gooseberry.h names, argument order, status
 * codes), linked with libgooseberry_b200.so instead of libgooseberry:
 * SpMV with one and with three right-hand sides, CG, the Cuthill-McKee order
 * and sparse and dense permutations on a small tridiagonal system.  Exits 0 and prints
 * "dropin ok" when every result is right.
 */
#define GOOSEBERRY_DOUBLE_REALS 1
#include "gooseberry.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>

#define N 64

static int fail(const char * what, int rc) {
  fprintf(stderr, "%s failed (%d): %s\n", what, rc, gb_last_error());
  return 1;
}

int main(void) {
  ind_t rowptr[N + 1];
  dim_t rowind[3 * N];
  real_t rowval[3 * N];
  real_t x[3 * N], y[3 * N], b[N], sol[N];
  dim_t perm[N];
  ind_t k = 0;
  dim_t i;
  int rc;
  size_t iters = 0;
  double rnorm = 0.0;
  /* tridiag(-1, 2, -1) */
  for (i = 0; i < N; ++i) {
    rowptr[i] = k;
    if (i > 0) { rowind[k] = i - 1; rowval[k++] = -1.0; }
    rowind[k] = i; rowval[k++] = 2.0;
    if (i + 1 < N) { rowind[k] = i + 1; rowval[k++] = -1.0; }
  }
  rowptr[N] = k;
  /* y = A x with x = 1..N: the rows sum to 0 except at the ends */
  for (i = 0; i < N; ++i) x[i] = (real_t)(i + 1);
  rc = gooseberry_spmult(N, N, 1, rowptr, rowind, rowval, x, y, NULL, 0);
  if (rc != GOOSEBERRY_SUCCESS) return fail("gooseberry_spmult", rc);
  for (i = 0; i < N; ++i) {
    const real_t want = (i == N - 1) ? (real_t)(N + 1) : 0.0;
    if (y[i] != want) { fprintf(stderr, "y[%u] = %g\n", i, y[i]); return 1; }
  }
  /* three right-hand sides at once: column j is (j + 1) * x */
  for (i = 0; i < 3 * N; ++i) x[i] = (real_t)((i / N) + 1) * (real_t)((i % N) + 1);
  rc = gooseberry_spmult(N, N, 3, rowptr, rowind, rowval, x, y, NULL, 0);
  if (rc != GOOSEBERRY_SUCCESS) return fail("gooseberry_spmult (3 columns)", rc);
  if (y[3 * (N - 1) + 2] != 3.0 * (N + 1)) { fprintf(stderr, "spmm\n"); return 1; }
  /* CG on A sol = b with b = A * 1 */
  for (i = 0; i < N; ++i) b[i] = (i == 0 || i == N - 1) ? 1.0 : 0.0;
  rc = gooseberry_cgd(N, rowptr, rowind, rowval, b, sol, 1e-12, 1000, &iters, &rnorm, NULL, 0);
  if (rc != GOOSEBERRY_SUCCESS) return fail("gooseberry_cgd", rc);
  for (i = 0; i < N; ++i)
    if (fabs(sol[i] - 1.0) > 1e-9) { fprintf(stderr, "sol[%u] = %g\n", i, sol[i]); return 1; }
  /* the band is already minimal: Cuthill-McKee keeps it banded */
  rc = gooseberry_permute_cuthillmckee(N, N, rowptr, rowind, rowval, NULL, 0, perm);
  if (rc != GOOSEBERRY_SUCCESS) return fail("gooseberry_permute_cuthillmckee", rc);
  rc = gooseberry_permute_sparse(N, N, rowptr, rowind, rowval, perm, perm);
  if (rc != GOOSEBERRY_SUCCESS) return fail("gooseberry_permute_sparse", rc);
  for (i = 0; i < N; ++i) {
    for (k = rowptr[i]; k < rowptr[i + 1]; ++k)
      if (rowind[k] + 1 < i || rowind[k] > i + 1) { fprintf(stderr, "band\n"); return 1; }
  }
  /* the right-hand side follows the reorder and comes back with its reverse */
  rc = gooseberry_permute_dense(N, 1, b, perm, NULL);
  if (rc != GOOSEBERRY_SUCCESS) return fail("gooseberry_permute_dense", rc);
  rc = gooseberry_permute_dense_rev(N, 1, b, perm, NULL);
  if (rc != GOOSEBERRY_SUCCESS) return fail("gooseberry_permute_dense_rev", rc);
  if (b[0] != 1.0 || b[N - 1] != 1.0 || b[1] != 0.0) { fprintf(stderr, "dense\n"); return 1; }
  /* a bad call comes back as the reference's error code */
  if (gooseberry_permute_cuthillmckee(N, N + 1, rowptr, rowind, rowval, NULL, 0, perm) !=
      GOOSEBERRY_ERROR_INVALIDINPUT) { fprintf(stderr, "error code\n"); return 1; }
  printf("dropin ok: cg %zu iterations\n", iters);
  return 0;
}
