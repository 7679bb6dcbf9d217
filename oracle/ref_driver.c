#define _POSIX_C_SOURCE 200809L
/*
 * ref_driver.c -- flat C entry points into the REFERENCE's own hot path,
 * compiled together with the unmodified reference sources src/blas.c,
 * src/cgd.c and src/matrix.c into oracle/_ref/libgbref_{f64,f32}.so.
 *
 * TEST INFRASTRUCTURE ONLY (the checker and the CPU baseline).  Nothing in the
 * product links it.  `real_t` is double when built with
 * -DGOOSEBERRY_DOUBLE_REALS=1 and float otherwise, exactly as in the reference
 * (include/gooseberry.h:73-79).
 *
 * - gbref_spmult: forwards to blas_spmult (src/blas.c:552-606), the body of
 *   gooseberry_spmult (src/gooseberry.c:53-67).
 * - gbref_dot:    forwards to blas_dot (src/blas.c:413-430).
 * - gbref_add / gbref_sub: forward to blas_add / blas_sub (src/blas.c:275-290,
 *   321-336) on an n x 1 dense vector; c may alias a or b, as cgd uses it.
 * - gbref_spdot:  forwards to blas_spdot (src/blas.c:433-451).
 * - gbref_read_sparse / _read_dense / _write_sparse / _write_dense: forward
 *   to the reference's src/io.c readers and writers (CSR and grid formats,
 *   src/io.c:145-239,369-498,1195-1275); gbref_free releases their arrays.
 * - gbref_pagerank: the pagerank command's loop (src/gooseberry_bin.c:
 *   2610-2741) lives in the CLI's main file, which does not build as a
 *   library; it is restated here around the reference's own blas_spmult,
 *   blas_scale and blas_add_scalar -- the calls the command makes through
 *   gooseberry_spmult / _scale / _add_scalar (src/gooseberry.c:35-67).
 * - gbref_cgd:    wraps cgd (src/cgd.c:40-129) for raw CSR arrays.  cgd prints
 *   one "ITER: k RMSE: v" line per iteration (src/cgd.c:116) and returns no
 *   iteration count, so stdout is redirected to a temporary file for the call
 *   and the ITER lines are parsed back into (iterations, last norm, history).
 * - gbref_cuthillmckee / gbref_permute_sparse / gbref_permute_dense: forward
 *   to permute_cuthillmckee (src/permute.c:288-337), permute_sparse
 *   (src/permute.c:120-205) and permute_dense / permute_dense_rev
 *   (src/permute.c:208-283), compiled from src/permute.c against the shim's
 *   priority queue (oracle/shim/dlpq_headers.h), which breaks equal-degree
 *   ties by the smaller vertex id.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

#include "matrix.h"
#include "blas.h"
#include "cgd.h"
#include "io.h"
#include "permute.h"
#include <omp.h>

int gbref_real_size(void);
void gbref_set_threads(int n);
int gbref_spmult(dim_t anrows, dim_t ancols, dim_t bncols,
    const ind_t * arowptr, const dim_t * arowind, const real_t * arowval,
    const real_t * bcolval, real_t * crowval, const dim_t * blocks,
    dim_t nblocks);
double gbref_dot(dim_t n, const real_t * a, const real_t * b);
int gbref_add(dim_t n, const real_t * a, const real_t * b, real_t * c);
int gbref_sub(dim_t n, const real_t * a, const real_t * b, real_t * c);
double gbref_spdot(dim_t nnz, const dim_t * ind, const real_t * val, const real_t * x);
int gbref_cgd(dim_t n, ind_t * rowptr, dim_t * rowind, real_t * rowval,
    real_t * b, real_t * x, double error, size_t niter, size_t * iters,
    double * last_norm, double * history, size_t history_len);
size_t gbref_pagerank(dim_t n, const ind_t * rowptr, const dim_t * rowind,
    const real_t * rowval, double damping, double minerror, size_t niter, real_t * result,
    double * error);
int gbref_read_sparse(int type, const char * file, dim_t * nrows, dim_t * ncols,
    ind_t ** rowptr, dim_t ** rowind, real_t ** rowval);
int gbref_read_dense(int type, const char * file, dim_t * nrows, dim_t * ncols,
    real_t ** rowval);
int gbref_write_sparse(int type, const char * file, dim_t nrows, dim_t ncols,
    const ind_t * rowptr, const dim_t * rowind, const real_t * rowval);
int gbref_write_dense(int type, const char * file, dim_t nrows, dim_t ncols,
    const real_t * rowval);
void gbref_free(void * p);
int gbref_cuthillmckee(dim_t nrows, dim_t ncols, const ind_t * rowptr,
    const dim_t * rowind, const dim_t * blocks, dim_t nblocks, dim_t * perm);
int gbref_permute_sparse(dim_t nrows, dim_t ncols, ind_t * rowptr,
    dim_t * rowind, real_t * rowval, const dim_t * rowperm,
    const dim_t * colperm);
int gbref_permute_dense(dim_t nrows, dim_t ncols, real_t * rowval,
    const dim_t * rowperm, const dim_t * colperm, int reverse);

/* OpenMP thread count of the reference's parallel regions.  With 1 thread
 * blas_dot sums in index order, which makes cgd bit-reproducible. */
void gbref_set_threads(int n)
{
  omp_set_num_threads(n > 0 ? n : 1);
}

int gbref_real_size(void)
{
  return (int)sizeof(real_t);
}

int gbref_spmult(dim_t anrows, dim_t ancols, dim_t bncols,
    const ind_t * arowptr, const dim_t * arowind, const real_t * arowval,
    const real_t * bcolval, real_t * crowval, const dim_t * blocks,
    dim_t nblocks)
{
  return blas_spmult(anrows, ancols, bncols, arowptr, arowind, arowval,
      bcolval, crowval, blocks, nblocks);
}

double gbref_dot(dim_t n, const real_t * a, const real_t * b)
{
  return (double)blas_dot(n, a, b);
}

int gbref_add(dim_t n, const real_t * a, const real_t * b, real_t * c)
{
  return blas_add(n, 1, a, b, c);
}

int gbref_sub(dim_t n, const real_t * a, const real_t * b, real_t * c)
{
  return blas_sub(n, 1, a, b, c);
}

/* blas_spdot (src/blas.c:433-451) takes its indices as real_t values; they
 * are converted here (exact below 2^24 for the float build, 2^53 for double). */
double gbref_spdot(dim_t nnz, const dim_t * ind, const real_t * val, const real_t * x)
{
  dim_t i;
  double s;
  real_t * rind = malloc(sizeof(real_t) * (nnz ? nnz : 1));
  if (!rind) {
    return 0.0;
  }
  for (i = 0; i < nnz; ++i) {
    rind[i] = (real_t)ind[i];
  }
  s = (double)blas_spdot(nnz, rind, val, x);
  free(rind);
  return s;
}

int gbref_cgd(dim_t n, ind_t * rowptr, dim_t * rowind, real_t * rowval,
    real_t * b, real_t * x, double error, size_t niter, size_t * iters,
    double * last_norm, double * history, size_t history_len)
{
  matrix_t a, bv, xv;
  FILE * tmp;
  int saved, rv;
  char line[256];
  size_t count = 0, k;
  double v, last = -1.0;

  memset(&a, 0, sizeof(a));
  memset(&bv, 0, sizeof(bv));
  memset(&xv, 0, sizeof(xv));
  a.type = MATRIX_TYPE_SPARSE_MATRIX;
  a.nrows = n;
  a.ncols = n;
  a.rowptr = rowptr;
  a.rowind = rowind;
  a.rowval = rowval;
  bv.type = MATRIX_TYPE_DENSE_VECTOR;
  bv.nrows = n;
  bv.ncols = 1;
  bv.rowval = bv.colval = b;
  xv.type = MATRIX_TYPE_DENSE_VECTOR;
  xv.nrows = n;
  xv.ncols = 1;
  xv.rowval = xv.colval = x;

  tmp = tmpfile();
  if (!tmp) {
    return -1;
  }
  fflush(stdout);
  saved = dup(STDOUT_FILENO);
  if (saved < 0 || dup2(fileno(tmp), STDOUT_FILENO) < 0) {
    fclose(tmp);
    return -1;
  }
  rv = cgd(&a, &bv, &xv, (real_t)error, niter);
  fflush(stdout);
  dup2(saved, STDOUT_FILENO);
  close(saved);

  rewind(tmp);
  while (fgets(line, sizeof(line), tmp)) {
    if (sscanf(line, "ITER: %zu RMSE: %lf", &k, &v) == 2) {
      if (history && count < history_len) {
        history[count] = v;
      }
      ++count;
      last = v;
    }
  }
  fclose(tmp);
  *iters = count;
  *last_norm = last;
  return rv;
}

size_t gbref_pagerank(dim_t n, const ind_t * rowptr, const dim_t * rowind,
    const real_t * rowval, double damping, double minerror, size_t niter, real_t * result,
    double * error)
{
  dim_t k, nsinks = 0;
  ind_t l;
  size_t i;
  real_t err = 0.0, dist, diff;
  const ind_t nnz = rowptr[n];
  real_t * indeg = calloc(n ? n : 1, sizeof(real_t));
  real_t * val = malloc(sizeof(real_t) * (nnz ? nnz : 1));
  dim_t * sinks = malloc(sizeof(dim_t) * (n ? n : 1));
  real_t * rank = malloc(sizeof(real_t) * (n ? n : 1));
  real_t * out = malloc(sizeof(real_t) * (n ? n : 1));
  real_t * tmp;
  int done = 0;
  for (k = 0; k < n; ++k) {
    if (rowptr[k] == rowptr[k + 1]) {
      sinks[nsinks++] = k;
    } else {
      for (l = rowptr[k]; l < rowptr[k + 1]; ++l) indeg[rowind[l]] += rowval[l];
    }
  }
  for (l = 0; l < nnz; ++l) val[l] = rowval[l] / indeg[rowind[l]];
  for (k = 0; k < n; ++k) rank[k] = 1.0 / n;
  for (i = 0; niter == 0 || i < niter; ++i) {
    blas_spmult(n, n, 1, rowptr, rowind, val, rank, out, NULL, 0);
    blas_scale(n, out, damping);
    dist = 0;
    for (k = 0; k < nsinks; ++k) dist += rank[sinks[k]];
    blas_add_scalar(n, out, ((1.0 - damping) / n) + dist);
    if (i % 10 == 0) {
      err = 0.0;
      for (k = 0; k < n; ++k) {
        diff = rank[k] - out[k];
        err += diff * diff;
      }
      if (err <= minerror * minerror) {
        ++i;
        done = 1;
        break;
      }
    }
    tmp = rank;
    rank = out;
    out = tmp;
  }
  if (!done) {
    err = 0.0;
    for (k = 0; k < n; ++k) {
      diff = rank[k] - out[k];
      err += diff * diff;
    }
  }
  *error = sqrt(err);
  memcpy(result, out, sizeof(real_t) * n);
  free(indeg);
  free(val);
  free(sinks);
  free(rank);
  free(out);
  return i;
}

int gbref_read_sparse(int type, const char * file, dim_t * nrows, dim_t * ncols,
    ind_t ** rowptr, dim_t ** rowind, real_t ** rowval)
{
  return read_sparse_matrix(type, file, nrows, ncols, rowptr, rowind, rowval);
}

int gbref_read_dense(int type, const char * file, dim_t * nrows, dim_t * ncols,
    real_t ** rowval)
{
  return read_dense_matrix(type, file, nrows, ncols, rowval);
}

int gbref_write_sparse(int type, const char * file, dim_t nrows, dim_t ncols,
    const ind_t * rowptr, const dim_t * rowind, const real_t * rowval)
{
  return write_sparse_matrix(type, file, nrows, ncols, rowptr, rowind, rowval);
}

int gbref_write_dense(int type, const char * file, dim_t nrows, dim_t ncols,
    const real_t * rowval)
{
  return write_dense_matrix(type, file, nrows, ncols, rowval);
}

void gbref_free(void * p)
{
  free(p);
}

/* The bandwidth-reducing order (src/permute.c:288-337): perm[new] = old; per
 * block when `blocks` (nblocks+1 boundaries) is given.  The values are not
 * read by the ordering. */
int gbref_cuthillmckee(dim_t nrows, dim_t ncols, const ind_t * rowptr,
    const dim_t * rowind, const dim_t * blocks, dim_t nblocks, dim_t * perm)
{
  return permute_cuthillmckee(nrows, ncols, rowptr, rowind, NULL, blocks,
      nblocks, perm);
}

/* In-place sparse permutation (src/permute.c:120-205): new row i is old row
 * rowperm[i]; old column colperm[j] becomes column j. */
int gbref_permute_sparse(dim_t nrows, dim_t ncols, ind_t * rowptr,
    dim_t * rowind, real_t * rowval, const dim_t * rowperm,
    const dim_t * colperm)
{
  return permute_sparse(nrows, ncols, rowptr, rowind, rowval, rowperm, colperm);
}

/* In-place dense permutation (src/permute.c:208-242) or its reverse
 * (src/permute.c:248-283), row-major nrows x ncols. */
int gbref_permute_dense(dim_t nrows, dim_t ncols, real_t * rowval,
    const dim_t * rowperm, const dim_t * colperm, int reverse)
{
  return reverse ? permute_dense_rev(nrows, ncols, rowval, rowperm, colperm)
                 : permute_dense(nrows, ncols, rowval, rowperm, colperm);
}

