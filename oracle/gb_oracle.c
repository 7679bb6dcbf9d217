/*
 * gb_oracle.c -- CPU restatement of gooseberry's SpMV / BLAS-1 / CG hot path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA path and the "port" CPU
 * baseline.  The product never links, loads or calls it.  Compiled with
 * -ffp-contract=off so no multiply-add is fused, like the reference's x86-64
 * build (no FMA in the baseline ISA).
 *
 * Each function states the reference lines it follows.  With one thread the
 * results are bit-identical to the reference built from its own sources
 * (oracle/_ref), which the CPU tests check.
 */
#include <math.h>
#include <stddef.h>
#include <stdint.h>
#include <string.h>
#include <stdlib.h>

typedef uint32_t dim_t;
typedef uint32_t ind_t;

/*
 * C = A*B for CSR A and column-major dense B (bcolval[j*ancols + l]), output
 * row-major (crowval[i*bncols + j]).  Per row and column: the sum starts at 0
 * and adds val[k]*B[ind[k]] for k ascending -- src/blas.c:82-91
 * (__sparse_mult_dense_block).  `blocks` (nblocks+1 row boundaries) restricts
 * the computed rows to the union of [blocks[c], blocks[c+1]) exactly as the
 * blocks branch of blas_spmult (src/blas.c:576-595); rows outside stay
 * untouched.  `nthreads` > 1 splits rows over OpenMP threads (src/blas.c:565,
 * 597-601); the split never changes a row's result.
 */
#define GB_ORACLE_SPMM(NAME, REAL)                                             \
  void NAME(dim_t anrows, dim_t ancols, dim_t bncols, const ind_t * rowptr,   \
      const dim_t * rowind, const REAL * rowval, const REAL * bcolval,         \
      REAL * crowval, const dim_t * blocks, dim_t nblocks, int nthreads);      \
  static void NAME##_block(dim_t start, dim_t end, dim_t ancols,              \
      dim_t bncols, const ind_t * rowptr, const dim_t * rowind,                \
      const REAL * rowval, const REAL * bcolval, REAL * crowval)               \
  {                                                                            \
    dim_t i, j;                                                                \
    ind_t k;                                                                   \
    for (i = start; i < end; ++i) {                                            \
      for (j = 0; j < bncols; ++j) {                                           \
        REAL acc = 0;                                                          \
        for (k = rowptr[i]; k < rowptr[i + 1]; ++k) {                          \
          acc += rowval[k] *                                                   \
              bcolval[(size_t)j * (size_t)ancols + (size_t)rowind[k]];         \
        }                                                                      \
        crowval[(size_t)i * (size_t)bncols + (size_t)j] = acc;                 \
      }                                                                        \
    }                                                                          \
  }                                                                            \
  void NAME(dim_t anrows, dim_t ancols, dim_t bncols, const ind_t * rowptr,   \
      const dim_t * rowind, const REAL * rowval, const REAL * bcolval,         \
      REAL * crowval, const dim_t * blocks, dim_t nblocks, int nthreads)       \
  {                                                                            \
    if (nthreads < 1) {                                                        \
      nthreads = 1;                                                            \
    }                                                                          \
    if (blocks) {                                                              \
      long c;                                                                  \
      _Pragma("omp parallel for num_threads(nthreads) schedule(static,1)")     \
      for (c = 0; c < (long)nblocks; ++c) {                                    \
        NAME##_block(blocks[c], blocks[c + 1], ancols, bncols, rowptr, rowind, \
            rowval, bcolval, crowval);                                         \
      }                                                                        \
    } else {                                                                   \
      long c;                                                                  \
      long const nchunk = (long)nthreads * 8;                                  \
      _Pragma("omp parallel for num_threads(nthreads) schedule(static,1)")     \
      for (c = 0; c < nchunk; ++c) {                                           \
        size_t const q = anrows / (size_t)nchunk, r = anrows % (size_t)nchunk; \
        size_t const s = (size_t)c * q + ((size_t)c < r ? (size_t)c : r);      \
        size_t const e = s + q + ((size_t)c < r ? 1 : 0);                      \
        NAME##_block((dim_t)s, (dim_t)e, ancols, bncols, rowptr, rowind,       \
            rowval, bcolval, crowval);                                         \
      }                                                                        \
    }                                                                          \
  }

GB_ORACLE_SPMM(oracle_spmm_f64, double)
GB_ORACLE_SPMM(oracle_spmm_f32, float)

/* sum_i a[i]*b[i], i ascending, accumulated in REAL -- src/blas.c:413-430
 * (blas_dot) as it runs on one OpenMP thread. */
#define GB_ORACLE_DOT(NAME, REAL)                                              \
  REAL NAME(size_t n, const REAL * a, const REAL * b);                         \
  REAL NAME(size_t n, const REAL * a, const REAL * b)                          \
  {                                                                            \
    size_t i;                                                                  \
    REAL x = 0;                                                                \
    for (i = 0; i < n; ++i) {                                                  \
      x += a[i] * b[i];                                                        \
    }                                                                          \
    return x;                                                                  \
  }
GB_ORACLE_DOT(oracle_dot_f64, double)
GB_ORACLE_DOT(oracle_dot_f32, float)

/* sum_k val[k]*x[ind[k]], k ascending, accumulated in REAL -- src/blas.c:433-451
 * (blas_spdot) as it runs on one OpenMP thread.  The reference passes the
 * indices as real_t values (src/blas.h:218-222); here they are integers. */
#define GB_ORACLE_SPDOT(NAME, REAL)                                            \
  REAL NAME(size_t nnz, const uint32_t * ind, const REAL * val, const REAL * x); \
  REAL NAME(size_t nnz, const uint32_t * ind, const REAL * val, const REAL * x)  \
  {                                                                            \
    size_t i;                                                                  \
    REAL s = 0;                                                                \
    for (i = 0; i < nnz; ++i) {                                                \
      s += val[i] * x[ind[i]];                                                 \
    }                                                                          \
    return s;                                                                  \
  }
GB_ORACLE_SPDOT(oracle_spdot_f64, double)
GB_ORACLE_SPDOT(oracle_spdot_f32, float)

/* v[i] *= s -- src/blas.c:244-257 (blas_scale); v[i] += s --
 * src/blas.c:397-410 (blas_add_scalar). */
void oracle_scale_f64(size_t n, double * v, double s);
void oracle_scale_f64(size_t n, double * v, double s)
{
  size_t i;
  for (i = 0; i < n; ++i) v[i] *= s;
}
void oracle_add_scalar_f64(size_t n, double * v, double s);
void oracle_add_scalar_f64(size_t n, double * v, double s)
{
  size_t i;
  for (i = 0; i < n; ++i) v[i] += s;
}
void oracle_scale_f32(size_t n, float * v, float s);
void oracle_scale_f32(size_t n, float * v, float s)
{
  size_t i;
  for (i = 0; i < n; ++i) v[i] *= s;
}
void oracle_add_scalar_f32(size_t n, float * v, float s);
void oracle_add_scalar_f32(size_t n, float * v, float s)
{
  size_t i;
  for (i = 0; i < n; ++i) v[i] += s;
}

/*
 * Unpreconditioned CG with exactly the update order of cgd (src/cgd.c:81-119):
 *   x = 0; r = b; p = r; dr = r.r
 *   loop iter = 0.. while iter < niter or niter == 0:
 *     ap = A p; alpha = dr / (p.ap)
 *     p *= alpha; nx = x + p                      (cgd.c:92-93)
 *     ap *= alpha; nr = r - ap                    (cgd.c:96-97)
 *     dnr = nr.nr; beta = dnr / dr                (cgd.c:100-101)
 *     p *= beta/alpha; p = nr + p                 (cgd.c:104-105)
 *     x = nx; r = nr; dr = dnr                    (cgd.c:108-112)
 *     rmse = sqrt(dr); record; stop if rmse <= error   (cgd.c:115-119)
 * `error` is the reference's ABSOLUTE bound on ||r||_2.  Returns the number of
 * iterations run (the reference's ITER line count); history[k] (if given)
 * receives rmse after iteration k.  Dots are sequential (one-thread blas_dot);
 * the SpMV uses `nthreads` threads (row split only, results unchanged).
 * niter == 0 is unbounded, as in the reference; the tests never pass it.
 */
#define GB_ORACLE_CGD(NAME, REAL, SPMM, DOT)                                   \
  size_t NAME(dim_t n, const ind_t * rowptr, const dim_t * rowind,             \
      const REAL * rowval, const REAL * b, REAL * x, REAL error, size_t niter, \
      double * history, size_t history_len, double * last_norm,                \
      int nthreads);                                                           \
  size_t NAME(dim_t n, const ind_t * rowptr, const dim_t * rowind,             \
      const REAL * rowval, const REAL * b, REAL * x, REAL error, size_t niter, \
      double * history, size_t history_len, double * last_norm, int nthreads)  \
  {                                                                            \
    size_t iter, i, count = 0;                                                 \
    REAL alpha, beta, rmse, dr, dnr;                                           \
    REAL * r = (REAL *)malloc(sizeof(REAL) * (n ? n : 1));                     \
    REAL * p = (REAL *)malloc(sizeof(REAL) * (n ? n : 1));                     \
    REAL * nr = (REAL *)malloc(sizeof(REAL) * (n ? n : 1));                    \
    REAL * nx = (REAL *)malloc(sizeof(REAL) * (n ? n : 1));                    \
    REAL * ap = (REAL *)malloc(sizeof(REAL) * (n ? n : 1));                    \
    *last_norm = -1.0;                                                         \
    for (i = 0; i < n; ++i) {                                                  \
      x[i] = 0;                                                                \
      r[i] = b[i];                                                             \
      p[i] = r[i];                                                             \
    }                                                                          \
    dr = DOT(n, r, r);                                                         \
    for (iter = 0; iter < niter || niter == 0; ++iter) {                       \
      SPMM(n, n, 1, rowptr, rowind, rowval, p, ap, NULL, 0, nthreads);         \
      alpha = dr / DOT(n, p, ap);                                              \
      for (i = 0; i < n; ++i) p[i] *= alpha;                                   \
      for (i = 0; i < n; ++i) nx[i] = x[i] + p[i];                             \
      for (i = 0; i < n; ++i) ap[i] *= alpha;                                  \
      for (i = 0; i < n; ++i) nr[i] = r[i] - ap[i];                            \
      dnr = DOT(n, nr, nr);                                                    \
      beta = dnr / dr;                                                         \
      {                                                                        \
        REAL const s = beta / alpha;                                           \
        for (i = 0; i < n; ++i) p[i] *= s;                                     \
      }                                                                        \
      for (i = 0; i < n; ++i) p[i] = nr[i] + p[i];                             \
      memcpy(x, nx, sizeof(REAL) * n);                                         \
      memcpy(r, nr, sizeof(REAL) * n);                                         \
      dr = dnr;                                                                \
      rmse = (REAL)sqrt((double)dr);                                           \
      if (history && count < history_len) history[count] = (double)rmse;      \
      ++count;                                                                 \
      *last_norm = (double)rmse;                                               \
      if (rmse <= error) {                                                     \
        break;                                                                 \
      }                                                                        \
    }                                                                          \
    free(r);                                                                   \
    free(p);                                                                   \
    free(nr);                                                                  \
    free(nx);                                                                  \
    free(ap);                                                                  \
    return count;                                                              \
  }
GB_ORACLE_CGD(oracle_cgd_f64, double, oracle_spmm_f64, oracle_dot_f64)
GB_ORACLE_CGD(oracle_cgd_f32, float, oracle_spmm_f32, oracle_dot_f32)

/* PageRank power iteration -- the reference's `pagerank` command,
 * src/gooseberry_bin.c:2610-2741, for a square CSR matrix already read in
 * (no permutation file, one run), with sequential sums (one OpenMP thread):
 *   - normalise: indeg[c] = sum of the values in column c, accumulated in row
 *     order; every value is divided by its column's indeg; rows without
 *     entries are sinks (2611-2630);
 *   - rank = 1/n; per iteration i: out = A rank; out *= damping;
 *     dist = sum of rank over the sinks, in sink order; out += (1-damping)/n
 *     + dist (2668-2689);
 *   - when i % 10 == 0: err = sum (rank - out)^2; err <= minerror^2 stops
 *     with i + 1 iterations and out the newest iterate (2691-2712);
 *   - otherwise rank and out swap (2714); niter == 0 means no limit;
 *   - at the limit err is taken between rank (newest) and out (the iterate
 *     before), and out -- the second-to-last iterate -- is the result
 *     (2716-2737, the output written at 2767).
 * rowval is not modified (the reference normalises its own copy in place).
 * Writes the result to result[n]; returns the iteration count. */
size_t oracle_pagerank_f64(uint32_t n, const uint32_t * rowptr, const uint32_t * rowind,
    const double * rowval, double damping, double minerror, size_t niter,
    double * result, double * error);
size_t oracle_pagerank_f64(uint32_t n, const uint32_t * rowptr, const uint32_t * rowind,
    const double * rowval, double damping, double minerror, size_t niter,
    double * result, double * error)
{
  uint32_t k, nsinks = 0;
  size_t l, i;
  double err = 0.0, dist, diff;
  const uint32_t nnz = rowptr[n];
  double * indeg = calloc(n ? n : 1, sizeof(double));
  double * val = malloc(sizeof(double) * (nnz ? nnz : 1));
  uint32_t * sinks = malloc(sizeof(uint32_t) * (n ? n : 1));
  double * rank = malloc(sizeof(double) * (n ? n : 1));
  double * out = malloc(sizeof(double) * (n ? n : 1));
  double * tmp;
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
    oracle_spmm_f64(n, n, 1, rowptr, rowind, val, rank, out, NULL, 0, 1);
    oracle_scale_f64(n, out, damping);
    dist = 0;
    for (k = 0; k < nsinks; ++k) dist += rank[sinks[k]];
    oracle_add_scalar_f64(n, out, ((1.0 - damping) / n) + dist);
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
  memcpy(result, out, sizeof(double) * n);
  free(indeg);
  free(val);
  free(sinks);
  free(rank);
  free(out);
  return i;
}

/*
 * Cuthill-McKee order -- src/permute.c:45-104 (__cuthillmckee_block) and
 * :288-337 (permute_cuthillmckee).  perm[new] = old.
 *
 * Per diagonal block [start, end) (the whole matrix when blocks is NULL):
 *   - deg[v] = entries of row v whose column lies in [start, end) (:66-77);
 *   - a new component starts at the remaining vertex of least degree
 *     (:81-84, the `rem` queue);
 *   - breadth-first from it: for each ordered vertex in turn, its still
 *     remaining in-block columns are taken out of `rem` and appended in
 *     ascending degree (:86-101, the `q` queue).
 * Positions start at `start`, so each block orders its own slice of perm.
 * Equal degrees are taken smaller vertex id first.  The reference's queues
 * come from domlib's dlpq (not vendored); this tie order is the one the oracle
 * shim's queue gives the compiled reference, so the two agree exactly.
 *
 * Written as a sort, not a queue: the least-degree remaining vertex is the
 * first unvisited entry of all vertices sorted by (degree, id), and a
 * vertex's children leave `q` in (degree, id) order.  Returns 0, or -1 when
 * nrows != ncols (the reference's GOOSEBERRY_ERROR_INVALIDINPUT).
 */
static int oracle_u64_cmp(const void * a, const void * b)
{
  const uint64_t x = *(const uint64_t *)a, y = *(const uint64_t *)b;
  return x < y ? -1 : (x > y ? 1 : 0);
}

static void oracle_cm_block(uint32_t start, uint32_t end, const uint32_t * rowptr,
    const uint32_t * rowind, uint32_t * perm)
{
  const uint32_t m = end - start;
  uint32_t v, j, nordered = start, sr = start, next = 0, maxdeg = 0, nc;
  uint32_t * deg = calloc(m ? m : 1, sizeof(uint32_t));
  uint32_t * order = malloc(sizeof(uint32_t) * (m ? m : 1));
  uint32_t * count;
  unsigned char * seen = calloc(m ? m : 1, 1);
  uint64_t * child = malloc(sizeof(uint64_t) * (m ? m : 1));
  for (v = start; v < end; ++v) {
    uint32_t d = 0;
    for (j = rowptr[v]; j < rowptr[v + 1]; ++j) {
      if (rowind[j] >= start && rowind[j] < end) ++d;
    }
    deg[v - start] = d;
    if (d > maxdeg) maxdeg = d;
  }
  /* stable counting sort by degree: (degree, id) order */
  count = calloc((size_t)maxdeg + 2, sizeof(uint32_t));
  for (v = 0; v < m; ++v) ++count[deg[v] + 1];
  for (v = 0; v <= maxdeg; ++v) count[v + 1] += count[v];
  for (v = 0; v < m; ++v) order[count[deg[v]]++] = start + v;
  free(count);
  while (nordered < end) {
    while (seen[order[next] - start]) ++next;
    v = order[next];
    seen[v - start] = 1;
    perm[nordered++] = v;
    while (sr < nordered) {
      v = perm[sr++];
      nc = 0;
      for (j = rowptr[v]; j < rowptr[v + 1]; ++j) {
        const uint32_t k = rowind[j];
        if (k >= start && k < end && !seen[k - start]) {
          seen[k - start] = 1;
          child[nc++] = ((uint64_t)deg[k - start] << 32) | k;
        }
      }
      qsort(child, nc, sizeof(uint64_t), oracle_u64_cmp);
      for (j = 0; j < nc; ++j) perm[nordered++] = (uint32_t)child[j];
    }
  }
  free(deg);
  free(order);
  free(seen);
  free(child);
}

int oracle_cuthillmckee(uint32_t nrows, uint32_t ncols, const uint32_t * rowptr,
    const uint32_t * rowind, const uint32_t * blocks, uint32_t nblocks, uint32_t * perm);
int oracle_cuthillmckee(uint32_t nrows, uint32_t ncols, const uint32_t * rowptr,
    const uint32_t * rowind, const uint32_t * blocks, uint32_t nblocks, uint32_t * perm)
{
  uint32_t c;
  if (nrows != ncols) return -1;
  if (blocks) {
    for (c = 0; c < nblocks; ++c) oracle_cm_block(blocks[c], blocks[c + 1], rowptr, rowind, perm);
  } else {
    oracle_cm_block(0, nrows, rowptr, rowind, perm);
  }
  return 0;
}

/*
 * Sparse permutation -- src/permute.c:120-205 (permute_sparse), out of place:
 * new row i is old row rowperm[i] (identity when NULL) with its entries in
 * their stored order; an old column c becomes the j with colperm[j] == c
 * (unchanged when colperm is NULL).  Columns are not re-sorted.
 */
void oracle_permute_sparse_f64(uint32_t nrows, uint32_t ncols, const uint32_t * rowptr,
    const uint32_t * rowind, const double * rowval, const uint32_t * rowperm,
    const uint32_t * colperm, uint32_t * prowptr, uint32_t * prowind, double * prowval);
void oracle_permute_sparse_f64(uint32_t nrows, uint32_t ncols, const uint32_t * rowptr,
    const uint32_t * rowind, const double * rowval, const uint32_t * rowperm,
    const uint32_t * colperm, uint32_t * prowptr, uint32_t * prowind, double * prowval)
{
  uint32_t i, j, v, k = 0;
  uint32_t * rename = NULL;
  if (colperm) {
    rename = malloc(sizeof(uint32_t) * (ncols ? ncols : 1));
    for (j = 0; j < ncols; ++j) rename[colperm[j]] = j;
  }
  prowptr[0] = 0;
  for (i = 0; i < nrows; ++i) {
    v = rowperm ? rowperm[i] : i;
    for (j = rowptr[v]; j < rowptr[v + 1]; ++j, ++k) {
      prowind[k] = rename ? rename[rowind[j]] : rowind[j];
      prowval[k] = rowval[j];
    }
    prowptr[i + 1] = k;
  }
  free(rename);
}

/*
 * Dense permutation -- src/permute.c:208-242 (permute_dense) and :248-283
 * (permute_dense_rev), out of place, row-major nrows x ncols:
 *   forward: out[i][j] = in[rowperm[i]][colperm[j]]
 *   reverse: out[rowperm[i]][colperm[j]] = in[i][j]
 * with a NULL permutation meaning identity.
 */
void oracle_permute_dense_f64(uint32_t nrows, uint32_t ncols, const double * in, double * out,
    const uint32_t * rowperm, const uint32_t * colperm, int reverse);
void oracle_permute_dense_f64(uint32_t nrows, uint32_t ncols, const double * in, double * out,
    const uint32_t * rowperm, const uint32_t * colperm, int reverse)
{
  uint32_t i, j;
  for (i = 0; i < nrows; ++i) {
    const size_t v = rowperm ? rowperm[i] : i;
    for (j = 0; j < ncols; ++j) {
      const size_t u = colperm ? colperm[j] : j;
      if (reverse) out[v * ncols + u] = in[(size_t)i * ncols + j];
      else out[(size_t)i * ncols + j] = in[v * ncols + u];
    }
  }
}
