/*
 * domlib.h -- minimal stand-in for the un-vendored `domlib` submodule of
 * gooseberry (reference .gitmodules:1-3, src/base.h:19).
 *
 * TEST INFRASTRUCTURE ONLY.  It exists so the reference's own hot-path sources
 * (src/blas.c, src/cgd.c, src/matrix.c, src/io.c with dlfile_shim.h, and
 * src/permute.c with dlpq_headers.h) can be compiled unmodified into the CPU
 * oracle under oracle/_ref.  It supplies only the helpers those files call:
 * typed alloc/calloc/set/copy/init_alloc, exclusive prefix sums, even
 * chunking of an index range over threads, free/swap/min and the
 * eprintf/wprintf message macros.  Written for this project from the call
 * sites; it is not domlib's code.
 */
#ifndef GB_ORACLE_DOMLIB_SHIM_H
#define GB_ORACLE_DOMLIB_SHIM_H

#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <stdint.h>
#include <stddef.h>
#include <math.h>

#define PF_SIZE_T "%zu"

#define DLTYPE_FLOAT 1
#define DLTYPE_INTEGRAL 2

#define eprintf(...) fprintf(stderr, __VA_ARGS__)
#define wprintf(...) fprintf(stderr, __VA_ARGS__)

#define dl_free(p) free(p)
#define dl_min(a, b) ((a) < (b) ? (a) : (b))
#define dl_swap(a, b)                                                          \
  do {                                                                         \
    __typeof__(a) dl_swap_tmp_ = (a);                                          \
    (a) = (b);                                                                 \
    (b) = dl_swap_tmp_;                                                        \
  } while (0)

/* Token pasting with one level of expansion, so PREFIX macros expand first. */
#define DLSHIM_CAT2(a, b) a##_##b
#define DLSHIM_CAT(a, b) DLSHIM_CAT2(a, b)

/* Even split of `n` items over `nchunks` workers: the first n%nchunks workers
 * get one extra item.  Only decides which thread owns which rows; it never
 * changes an SpMV result because every row is summed by a single thread. */
static inline size_t size_chunksize(size_t id, size_t nchunks, size_t n)
{
  return n / nchunks + (id < n % nchunks ? 1 : 0);
}
static inline size_t size_chunkstart(size_t id, size_t nchunks, size_t n)
{
  size_t const r = n % nchunks;
  return id * (n / nchunks) + (id < r ? id : r);
}
#define dim_chunksize(id, nchunks, n) size_chunksize((id), (nchunks), (n))
#define dim_chunkstart(id, nchunks, n) size_chunkstart((id), (nchunks), (n))

static inline int * int_calloc(size_t n)
{
  return (int *)calloc(n ? n : 1, sizeof(int));
}

#include "dlfile_shim.h"

#endif
