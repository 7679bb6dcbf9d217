/*
 * gooseberry.h -- drop-in C API of the gooseberry sparse hot path, served by
 * the B200 library libgooseberry_b200.so.
 *
 * Declares the same types, status codes and entry points that the reference's
 * public header declares for this path (reference include/gooseberry.h), so a
 * C or C++ program that calls gooseberry_spmult / gooseberry_scale /
 * gooseberry_add_scalar recompiles against this header unchanged.  Unlike the
 * reference header (include/gooseberry.h:117, `extern 'C'`), this one also
 * compiles as C++.
 *
 * Precision follows the reference's build-time rule
 * (include/gooseberry.h:73-79): real_t is float unless GOOSEBERRY_DOUBLE_REALS
 * is defined.  The library exports both widths: the unsuffixed symbols take
 * float (the reference's default ABI) and the `_f64` symbols take double; with
 * GOOSEBERRY_DOUBLE_REALS defined the unsuffixed names below are mapped onto
 * the `_f64` symbols by macro, so callers write the reference's names either
 * way.
 *
 * All pointers here are HOST pointers owned by the caller, as in the
 * reference: each call copies its inputs to the GPU, runs there and copies the
 * result back before returning (synchronous, like the OpenMP original).  For
 * device-resident matrices, streams and the solvers see gooseberry_b200.h.
 */
#ifndef GOOSEBERRY_H
#define GOOSEBERRY_H

#include <stddef.h>
#include <stdint.h>
#include <inttypes.h>

#define GOOSEBERRY_VER_MAJOR 0
#define GOOSEBERRY_VER_MINOR 1
#define GOOSEBERRY_VER_SUBMINOR 7

/* Index and value types (reference include/gooseberry.h:43-82).  Only the
 * default 32-bit unsigned dim_t / ind_t layout is served by this library. */
#ifndef BOWSTRING_TYPES_DEFINED
#if defined(GOOSEBERRY_SIGNED_TYPES) || defined(GOOSEBERRY_64BIT_DIMENSIONS) || \
    defined(GOOSEBERRY_64BIT_INDICES)
#error "libgooseberry_b200 serves the default uint32 dim_t/ind_t layout only"
#endif
typedef uint64_t gooseberry_int64_t;
typedef uint32_t gooseberry_int32_t;
#define PF_BSINT64_T "%" PRIu64
#define PF_BSINT32_T "%" PRIu32
typedef gooseberry_int32_t dim_t;
typedef gooseberry_int32_t ind_t;
#define PF_DIM_T PF_BSINT32_T
#define PF_IND_T PF_BSINT32_T
#ifdef GOOSEBERRY_DOUBLE_REALS
typedef double real_t;
#define PF_REAL_T "%lf"
#else
typedef float real_t;
#define PF_REAL_T "%f"
#endif
#define PF_MINREAL_T "%g"
#endif

/* Status codes (reference include/gooseberry.h:85-94).  Success is 1. */
typedef enum gooseberry_error_t {
  GOOSEBERRY_SUCCESS = 1,
  GOOSEBERRY_ERROR_UNIMPLEMENTED,
  GOOSEBERRY_ERROR_INVALIDINPUT,
  GOOSEBERRY_ERROR_READ,
  GOOSEBERRY_ERROR_WRITE,
  GOOSEBERRY_ERROR_FILENOTFOUND,
  GOOSEBERRY_ERROR_PERMISSIONDENIED,
  GOOSEBERRY_ERROR_UNKNOWN
} gooseberry_error_t;

/* File formats, numbered as the reference (include/gooseberry.h:97-106).
 * CSR and GRID are read and written here; the others are reported as
 * GOOSEBERRY_ERROR_UNIMPLEMENTED. */
typedef enum gooseberry_format_t {
  GOOSEBERRY_FORMAT_RAW,
  GOOSEBERRY_FORMAT_GRID,
  GOOSEBERRY_FORMAT_CSR,
  GOOSEBERRY_FORMAT_POINT,
  GOOSEBERRY_FORMAT_SVM,
  GOOSEBERRY_FORMAT_GRAPH,
  GOOSEBERRY_FORMAT_CLU,
  GOOSEBERRY_FORMAT_MATRIXMARKET
} gooseberry_format_t;

/* Symbols exported by the shared library (hidden visibility otherwise). */
#if defined(__GNUC__)
#define GOOSEBERRY_API __attribute__((visibility("default")))
#else
#define GOOSEBERRY_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#ifdef GOOSEBERRY_DOUBLE_REALS
#define gooseberry_scale gooseberry_scale_f64
#define gooseberry_add_scalar gooseberry_add_scalar_f64
#define gooseberry_spmult gooseberry_spmult_f64
#define gooseberry_cgd gooseberry_cgd_f64
#define gooseberry_pagerank gooseberry_pagerank_f64
#define gooseberry_read_sparse_matrix gooseberry_read_sparse_matrix_f64
#define gooseberry_read_dense_matrix gooseberry_read_dense_matrix_f64
#define gooseberry_write_sparse_matrix gooseberry_write_sparse_matrix_f64
#define gooseberry_write_dense_matrix gooseberry_write_dense_matrix_f64
#define gooseberry_permute_sparse gooseberry_permute_sparse_f64
#define gooseberry_permute_dense gooseberry_permute_dense_f64
#define gooseberry_permute_dense_rev gooseberry_permute_dense_rev_f64
#endif

/* Message of the last failed call on this thread (no reference counterpart:
 * the reference prints its errors).  Also declared in gooseberry_b200.h. */
GOOSEBERRY_API const char * gb_last_error(void);

/*
 * val[i] *= s for i < n.
 * Replaces gooseberry_scale (reference include/gooseberry.h:134-137,
 * src/gooseberry.c:35-41 -> src/blas.c:244-257).
 */
GOOSEBERRY_API int gooseberry_scale(ind_t n, real_t * val, real_t s);
GOOSEBERRY_API int gooseberry_scale_f64(ind_t n, double * val, double s);

/*
 * val[i] += s for i < n.
 * Replaces gooseberry_add_scalar (reference include/gooseberry.h:150-153,
 * src/gooseberry.c:44-50 -> src/blas.c:397-410).
 */
GOOSEBERRY_API int gooseberry_add_scalar(ind_t n, real_t * val, real_t s);
GOOSEBERRY_API int gooseberry_add_scalar_f64(ind_t n, double * val, double s);

/*
 * C = A * B with A an anrows x ancols CSR matrix (arowptr[anrows+1],
 * arowind[nnz], arowval[nnz]), B dense ancols x bncols stored column-major
 * (bcolval[j*ancols + l]) and C dense anrows x bncols stored row-major
 * (crowval[i*bncols + j]).  bncols == 1 is SpMV.  When blocks != NULL only the
 * rows of [blocks[c], blocks[c+1]) for c < nblocks are computed and every
 * other row of C is left untouched, as in the reference's blocks branch.
 * Returns GOOSEBERRY_ERROR_INVALIDINPUT for NULL arrays or column indices
 * >= ancols, GOOSEBERRY_ERROR_UNKNOWN for a CUDA failure (see
 * gb_last_error()).
 * Replaces gooseberry_spmult (reference include/gooseberry.h:174-184,
 * src/gooseberry.c:53-67 -> src/blas.c:552-606).
 */
GOOSEBERRY_API int gooseberry_spmult(dim_t anrows, dim_t ancols, dim_t bncols,
    const ind_t * arowptr, const dim_t * arowind, const real_t * arowval,
    const real_t * bcolval, real_t * crowval, const dim_t * blocks,
    dim_t nblocks);
GOOSEBERRY_API int gooseberry_spmult_f64(dim_t anrows, dim_t ancols, dim_t bncols,
    const ind_t * arowptr, const dim_t * arowind, const double * arowval,
    const double * bcolval, double * crowval, const dim_t * blocks,
    dim_t nblocks);

/*
 * Unpreconditioned conjugate gradient on the n x n CSR matrix A: x0 = 0, stop
 * when ||r||_2 <= error (ABSOLUTE, as the reference) or after niter
 * iterations (niter == 0: no iteration limit).  On return x holds the
 * solution, *iterations (if non-NULL) the number of iterations run -- the
 * count of ITER lines the reference prints -- and *rnorm (if non-NULL) the
 * final ||r||_2.  history (if non-NULL) receives ||r||_2 after each iteration,
 * up to history_len entries.
 * Exports cgd (reference src/cgd.h:29-34, src/cgd.c:40-129), which the
 * reference keeps internal, over raw CSR arrays instead of matrix_t.
 * Returns GOOSEBERRY_ERROR_INVALIDINPUT for NULL arrays or bad indices.
 */
GOOSEBERRY_API int gooseberry_cgd(dim_t n, const ind_t * rowptr, const dim_t * rowind,
    const real_t * rowval, const real_t * b, real_t * x, real_t error,
    size_t niter, size_t * iterations, double * rnorm, double * history,
    size_t history_len);
GOOSEBERRY_API int gooseberry_cgd_f64(dim_t n, const ind_t * rowptr, const dim_t * rowind,
    const double * rowval, const double * b, double * x, double error,
    size_t niter, size_t * iterations, double * rnorm, double * history,
    size_t history_len);

/*
 * PageRank of the square n x n CSR graph (rowptr/rowind/rowval), the
 * reference's `pagerank` command (src/gooseberry_bin.c:2610-2741) over arrays
 * already in memory.  Values are normalised by their column sums; rows with no
 * entries are sinks.  Starting from rank = 1/n, every iteration computes
 * out = damping * (A rank) + (1 - damping)/n + (sum of rank over the sinks); on
 * iterations 0, 10, 20, ... the squared change sum (rank - out)^2 is compared
 * with minerror^2 and the run stops when it is not larger.  niter == 0 means
 * no iteration limit (a graph with sinks never converges: the reference adds
 * the whole sink mass to every entry).  On return rank[n] holds the result --
 * the newest iterate on convergence, the one before it when niter ended the
 * run, as the reference writes -- *iterations (if non-NULL) the iteration
 * count and *error (if non-NULL) the 2-norm of the last change.  The float
 * form computes in double and rounds rank to float.
 */
GOOSEBERRY_API int gooseberry_pagerank(dim_t n, const ind_t * rowptr, const dim_t * rowind,
    const real_t * rowval, real_t damping, real_t minerror, size_t niter, real_t * rank,
    size_t * iterations, double * error);
GOOSEBERRY_API int gooseberry_pagerank_f64(dim_t n, const ind_t * rowptr,
    const dim_t * rowind, const double * rowval, double damping, double minerror,
    size_t niter, double * rank, size_t * iterations, double * error);

/*
 * Text files (reference include/gooseberry.h:389-421, src/io.c:1467-1545),
 * parsed by all host threads with the reference's rules: CSR rows of
 * "column value" pairs (1-based columns unless a 0 appears; ncols = largest -
 * smallest column + 1; blank lines are empty rows; lines starting with
 * # % ' " / are comments) and GRID rows of values.  Output arrays are
 * malloc'ed; the caller frees them with free().  Writers print values with
 * %g, CSR columns 1-based.  Errors: GOOSEBERRY_ERROR_FILENOTFOUND /
 * _PERMISSIONDENIED / _READ / _WRITE, _INVALIDINPUT for a ragged grid or an
 * unknown format, _UNIMPLEMENTED for the formats other than CSR and GRID.
 */
GOOSEBERRY_API int gooseberry_read_sparse_matrix(int type, const char * file, dim_t * nrows,
    dim_t * ncols, ind_t ** rowptr, dim_t ** rowind, real_t ** rowval);
GOOSEBERRY_API int gooseberry_read_sparse_matrix_f64(int type, const char * file,
    dim_t * nrows, dim_t * ncols, ind_t ** rowptr, dim_t ** rowind, double ** rowval);
GOOSEBERRY_API int gooseberry_read_dense_matrix(int type, const char * file, dim_t * nrows,
    dim_t * ncols, real_t ** rowval);
GOOSEBERRY_API int gooseberry_read_dense_matrix_f64(int type, const char * file,
    dim_t * nrows, dim_t * ncols, double ** rowval);
GOOSEBERRY_API int gooseberry_write_dense_matrix(int type, const char * file, dim_t nrows,
    dim_t ncols, const real_t * rowval);
GOOSEBERRY_API int gooseberry_write_dense_matrix_f64(int type, const char * file,
    dim_t nrows, dim_t ncols, const double * rowval);
GOOSEBERRY_API int gooseberry_write_sparse_matrix(int type, const char * file, dim_t nrows,
    dim_t ncols, const ind_t * rowptr, const dim_t * rowind, const real_t * rowval);
GOOSEBERRY_API int gooseberry_write_sparse_matrix_f64(int type, const char * file,
    dim_t nrows, dim_t ncols, const ind_t * rowptr, const dim_t * rowind,
    const double * rowval);

/*
 * Bandwidth-reducing order: replaces permute_cuthillmckee (reference
 * src/permute.h:40-48, src/permute.c:288-337), which the CLI calls for
 * `permute -p bandwidth` (src/gooseberry_bin.c:986-993) and `blas -b`
 * (:1655-1676).  perm[new] = old.  With `blocks` (nblocks+1 row boundaries)
 * every diagonal block is ordered on its own within its slice of perm; edges
 * leaving a block are ignored.  Equal degrees go smaller row first.  rowval is
 * not read.  nrows != ncols gives GOOSEBERRY_ERROR_INVALIDINPUT as in the
 * reference; so do blocks that do not cover [0, nrows) (the reference leaves
 * the uncovered part of perm unwritten).  Runs on the GPU; host arrays.
 */
GOOSEBERRY_API int gooseberry_permute_cuthillmckee(dim_t nrows, dim_t ncols,
    const ind_t * rowptr, const dim_t * rowind, const void * rowval, const dim_t * blocks,
    dim_t nblocks, dim_t * perm);

/*
 * In-place sparse permutation: replaces permute_sparse (reference
 * src/permute.h:30-37, src/permute.c:120-205).  New row i is old row
 * rowperm[i]; old column colperm[j] becomes column j; either may be NULL (no
 * change); the entries of a row keep their stored order.  Differences: a
 * rowperm / colperm that is not a permutation, a decreasing rowptr or a column
 * >= ncols gives GOOSEBERRY_ERROR_INVALIDINPUT and leaves the arrays as they
 * were (the reference reads or writes out of bounds).  Runs on the GPU.
 */
GOOSEBERRY_API int gooseberry_permute_sparse(dim_t nrows, dim_t ncols, ind_t * rowptr,
    dim_t * rowind, real_t * rowval, const dim_t * rowperm, const dim_t * colperm);
GOOSEBERRY_API int gooseberry_permute_sparse_f64(dim_t nrows, dim_t ncols, ind_t * rowptr,
    dim_t * rowind, double * rowval, const dim_t * rowperm, const dim_t * colperm);

/*
 * In-place dense permutation of a row-major nrows x ncols matrix: replaces
 * permute_dense (reference src/permute.h:51-56, src/permute.c:208-242;
 * row[i][j] <- row[rowperm[i]][colperm[j]]) and permute_dense_rev (:59-64,
 * :248-283; row[rowperm[i]][colperm[j]] <- row[i][j]), which matrix_permute
 * applies to dense vectors and matrices (src/matrix.c:256-342), e.g. the
 * right-hand side after a Cuthill-McKee reorder (src/gooseberry_bin.c:1674).
 * NULL permutations mean identity.  A rowperm / colperm that is not a
 * permutation gives GOOSEBERRY_ERROR_INVALIDINPUT (the reference does not
 * check).  Runs on the GPU.
 */
GOOSEBERRY_API int gooseberry_permute_dense(dim_t nrows, dim_t ncols, real_t * rowval,
    const dim_t * rowperm, const dim_t * colperm);
GOOSEBERRY_API int gooseberry_permute_dense_f64(dim_t nrows, dim_t ncols, double * rowval,
    const dim_t * rowperm, const dim_t * colperm);
GOOSEBERRY_API int gooseberry_permute_dense_rev(dim_t nrows, dim_t ncols, real_t * rowval,
    const dim_t * rowperm, const dim_t * colperm);
GOOSEBERRY_API int gooseberry_permute_dense_rev_f64(dim_t nrows, dim_t ncols, double * rowval,
    const dim_t * rowperm, const dim_t * colperm);

#ifdef __cplusplus
}
#endif

#endif /* GOOSEBERRY_H */
