/*
 * gooseberry_b200.h -- device-resident extension API of libgooseberry_b200.so.
 *
 * The reference keeps everything in host memory and re-reads the matrix on
 * every call (src/blas.c:552-606, src/cgd.c:40-129).  On a GPU the matrix and
 * the Krylov vectors should stay in HBM across calls, so this header adds
 * opaque device-resident handles beside the drop-in API of gooseberry.h:
 *
 *   gb_csr_t  a CSR matrix in HBM (owned copy or borrowed device arrays) plus
 *             its SpMV tile plan and schedule;
 *   gb_cg_t   a CG solver workspace bound to one gb_csr_t.
 *
 * Conventions
 *   - Return GOOSEBERRY_SUCCESS (1) or a gooseberry_error_t code; on failure
 *     gb_last_error() returns a message (thread-local).
 *   - `stream` is a cudaStream_t passed as void*; NULL is the legacy default
 *     stream.  Calls taking device pointers are asynchronous on `stream`
 *     unless stated otherwise.
 *   - Index layout is gooseberry's CSR: uint32 rowptr[nrows+1] (row i holds
 *     rowptr[i]..rowptr[i+1]-1), uint32 rowind[nnz] column indices, values
 *     rowval[nnz] (src/matrix.h:37-45).
 *   - The current CUDA device of the calling thread is used.
 */
#ifndef GOOSEBERRY_B200_H
#define GOOSEBERRY_B200_H

#include "gooseberry.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct gb_csr gb_csr_t;
typedef struct gb_cg gb_cg_t;
typedef void * gb_stream_t;

/* ---- errors -------------------------------------------------------------- */

/* Message describing the last failed call on this thread ("" if none).
 * No reference counterpart (the reference prints with eprintf). */
GOOSEBERRY_API const char * gb_last_error(void);

/* ---- matrices ------------------------------------------------------------ */

/* gb_csr_create flags */
#define GB_CSR_VALUES_F64 0x1u      /* keep double values on the device      */
#define GB_CSR_VALUES_F32 0x2u      /* keep float values (rounded from f64)   */
#define GB_CSR_DEVICE_POINTERS 0x4u /* arrays are device memory; borrow them  */

/* Row-length summary and chosen SpMV schedule of a matrix. */
typedef struct gb_csr_info {
  dim_t nrows, ncols;
  ind_t nnz;
  uint32_t ntiles;       /* row-aligned tiles of the SpMV plan               */
  uint32_t nlong;        /* rows split across several tiles                  */
  uint32_t max_row;      /* longest row                                      */
  double mean_row;       /* nnz / nrows                                      */
  uint32_t row_p50, row_p90, row_p99; /* row-length quantiles               */
  int schedule;          /* gb_schedule_t of the f64 SpMV                    */
  int schedule_f32;      /* gb_schedule_t of the f32 SpMV                    */
  uint32_t tile_items;   /* rows + nnz per tile                              */
} gb_csr_info_t;

/* How the SpMV kernel reduces the products of one tile (a run of whole rows
 * holding at most tile_items rows + nonzeros, staged in shared memory) into
 * row sums. */
typedef enum gb_schedule {
  GB_SCHED_AUTO = 0,     /* autotuner decides (default)                      */
  GB_SCHED_THREAD = 1,   /* one thread per row                               */
  GB_SCHED_GROUP4 = 2,   /* 4 lanes per row                                  */
  GB_SCHED_GROUP8 = 3,   /* 8 lanes per row                                  */
  GB_SCHED_WARP = 4,     /* 32 lanes per row                                 */
  GB_SCHED_MERGE = 5,    /* merge-path split of rows+nnz over threads        */
  GB_SCHED_ROW = 6,      /* one thread per row straight from global memory,
                            no tile staging; sums each row in the reference's
                            order (k ascending, unfused multiply and add), so
                            its SpMV is bit-identical to the reference       */
  GB_SCHED_WTILE = 7,    /* per-WARP tiles (small tile_items, ~256): each
                            warp streams its next tile into its own shared
                            memory stage with cp.async while its lanes sum
                            the current tile's rows, one row per lane, in
                            the reference's order (bit-identical, like ROW) */
  GB_SCHED_WMERGE = 8,   /* per-WARP tiles of at most 128 items, no CTA
                            barrier: indices, values and x gathers are
                            prefetched into registers one tile ahead, and
                            rows are reduced along the merge path of (row
                            ends, nonzeros) with equal work per lane (for
                            skewed row lengths).  The CG solvers run a
                            matrix set to this schedule with MERGE. */
  GB_SCHED_SEG = 9       /* no tiles: one contiguous range of nonzeros per
                            warp (balanced on rows + nonzeros), read with
                            16-byte loads; each lane sums 4 consecutive
                            products and a segmented scan over the lanes
                            joins rows that span lanes, whatever the row
                            lengths.  Needs rowind and the values on
                            16-byte boundaries (always true for matrices
                            the library uploads).  Plain SpMV only: the CG
                            solvers run such a matrix with MERGE. */
} gb_schedule_t;

/*
 * Create a device-resident CSR matrix.  Without GB_CSR_DEVICE_POINTERS the
 * host arrays are uploaded into library-owned device memory; with it the
 * device arrays are borrowed (they must outlive the handle and stay
 * unchanged).  rowval64 is required for GB_CSR_VALUES_F64; rowval32 may be
 * NULL, in which case float values are rounded from rowval64 on the device.
 * Validates rowptr (non-decreasing, rowptr[nrows]-rowptr[0] == nnz) and every
 * column index (< ncols); builds the tile plan.  Synchronous.
 * Counterpart of matrix_init(MATRIX_TYPE_SPARSE_MATRIX, ...) followed by the
 * caller filling rowptr/rowind/rowval (reference src/matrix.c:44-143).
 */
GOOSEBERRY_API int gb_csr_create(dim_t nrows, dim_t ncols, ind_t nnz, const ind_t * rowptr,
    const dim_t * rowind, const double * rowval64, const float * rowval32,
    unsigned flags, gb_stream_t stream, gb_csr_t ** out);

/* Read a CSR text file (the format of gooseberry_read_sparse_matrix with
 * GOOSEBERRY_FORMAT_CSR, reference src/io.c:369-498) with all host threads
 * into host memory and create a device matrix from it (flags: the
 * value widths to keep, GB_CSR_VALUES_F64 and/or _F32).  Synchronous. */
GOOSEBERRY_API int gb_csr_read(const char * file, unsigned flags, gb_stream_t stream,
    gb_csr_t ** out);

/* Release a matrix (matrix_free, reference src/matrix.c:483-535). */
GOOSEBERRY_API int gb_csr_destroy(gb_csr_t * a);

/* Shape, row-length summary, tile plan and current schedules of a matrix
 * (host struct; no GPU work).  The reference's matrix_t exposes only the
 * shape and the arrays (src/matrix.h:37-45). */
GOOSEBERRY_API int gb_csr_get_info(const gb_csr_t * a, gb_csr_info_t * info);

/* Fix the SpMV schedule of one value width (GB_CSR_VALUES_F64 or _F32).
 * tile_items == 0 keeps the current tile size (for the per-warp schedules a
 * plan built for CTA tiles is rebuilt at their default tile size). */
GOOSEBERRY_API int gb_csr_set_schedule(gb_csr_t * a, unsigned value_width, int schedule,
    uint32_t tile_items);

/* Time every candidate schedule on this matrix and keep the fastest; the
 * choice is cached per process under a key of (row-length quantiles, nrows,
 * nnz, value width) so equal-shaped matrices skip the timing.  Synchronous. */
GOOSEBERRY_API int gb_csr_autotune(gb_csr_t * a, unsigned value_width, gb_stream_t stream);

/* Run the SpMV tile planner on a HOST rowptr (no GPU involved).  Writes the
 * tile and long-row counts; when tiles != NULL (room for max_tiles) also the
 * tiles, 4 uint32 each: {first row | long-row id, row count (0 marks a chunk
 * of a long row), first nonzero, nonzero count}.  Row-length quantiles go to
 * info (optional).  Used for inspection and host-side tests; no reference
 * counterpart (the reference splits rows evenly per thread,
 * src/blas.c:597-601). */
GOOSEBERRY_API int gb_plan_tiles_host(dim_t nrows, const ind_t * rowptr, ind_t nnz,
    uint32_t tile_items, uint32_t * tiles, size_t max_tiles, uint32_t * ntiles,
    uint32_t * nlong, gb_csr_info_t * info);

/* ---- SpMV / SpMM on device vectors ---------------------------------------- */

/* y = A x.  Device-resident counterpart of blas_spmult with bncols == 1
 * (reference src/blas.c:552-606, inner loop src/blas.c:82-91).  f64: double
 * values, x, y and accumulation.  f32: float values, x, y and accumulation. */
GOOSEBERRY_API int gb_spmv_f64(const gb_csr_t * a, const double * x, double * y,
    gb_stream_t stream);
GOOSEBERRY_API int gb_spmv_f32(const gb_csr_t * a, const float * x, float * y,
    gb_stream_t stream);

/* C = A B, B column-major ncols x bncols, C row-major nrows x bncols
 * (reference src/blas.c:82-91 with bncols > 1). */
GOOSEBERRY_API int gb_spmm_f64(const gb_csr_t * a, dim_t bncols, const double * b, double * c,
    gb_stream_t stream);

/* ---- reordering ------------------------------------------------------------ */

/* Cuthill-McKee order of a square device matrix into the DEVICE array perm
 * (perm[new] = old), as permute_cuthillmckee (reference src/permute.c:
 * 288-337) computes it; equal degrees go smaller row first.  blocks: HOST
 * array of nblocks+1 row boundaries covering [0, nrows) (each diagonal block
 * ordered on its own, edges leaving it ignored), or NULL.  Synchronous. */
GOOSEBERRY_API int gb_csr_cuthillmckee(const gb_csr_t * a, const dim_t * blocks, dim_t nblocks,
    dim_t * perm, gb_stream_t stream);

/* A new device matrix P_r A P_c^T: new row i is row rowperm[i] of a, old
 * column colperm[j] becomes column j (permute_sparse, reference
 * src/permute.c:120-205); both DEVICE arrays, NULL for identity; rows keep
 * their entry order.  The result holds the same value widths as a, owns its
 * memory and gets the default schedule.  Synchronous. */
GOOSEBERRY_API int gb_csr_permute(const gb_csr_t * a, const dim_t * rowperm,
    const dim_t * colperm, gb_stream_t stream, gb_csr_t ** out);

/* y[i] = x[perm[i]] (reverse = 0; permute_dense with one column, reference
 * src/permute.c:208-242) or y[perm[i]] = x[i] (reverse != 0;
 * permute_dense_rev, :245-280).  Device arrays; perm must be a permutation
 * of 0..n-1; x and y must not overlap. */
GOOSEBERRY_API int gb_permute_vector_f64(size_t n, const double * x, const dim_t * perm,
    int reverse, double * y, gb_stream_t stream);

/* ---- BLAS-1 on device vectors --------------------------------------------- */

/* *result = sum a[i]*b[i], accumulated in double, deterministic (fixed
 * reduction order).  result is a DEVICE pointer.  blas_dot, reference
 * src/blas.c:413-430. */
GOOSEBERRY_API int gb_dot_f64(size_t n, const double * a, const double * b, double * result,
    gb_stream_t stream);
GOOSEBERRY_API int gb_dot_f32(size_t n, const float * a, const float * b, double * result,
    gb_stream_t stream);

/* *result = sum_k val[k] * x[ind[k]] (a sparse vector . a dense vector of nx
 * entries), accumulated in double, deterministic (fixed reduction order).
 * Indices must be < nx.  result is a DEVICE pointer.  blas_spdot, reference
 * src/blas.c:433-451.  Run on a matrix's own (rowind, rowval) and x it streams
 * the same bytes and gathers the same x entries as that matrix's SpMV, without
 * the row reductions: its time is a floor for the SpMV on this GPU. */
GOOSEBERRY_API int gb_spdot_f64(size_t nnz, const dim_t * ind, const double * val,
    const double * x, size_t nx, double * result, gb_stream_t stream);
GOOSEBERRY_API int gb_spdot_f32(size_t nnz, const dim_t * ind, const float * val,
    const float * x, size_t nx, double * result, gb_stream_t stream);

/*
 * Allocation-free form of gb_dot_f64, for callers that must not allocate
 * device memory during a call: code whose device memory is entirely owned by
 * another allocator (a framework's caching pool holding all of HBM, where
 * cudaMalloc fails or forces that pool to release memory), and
 * latency-critical loops where cudaMalloc/cudaFree would synchronise the
 * device.  It computes the same sum as gb_dot_f64 (double accumulation,
 * fixed order; the grouping differs, so the last bits can too), but it keeps
 * its per-CTA partial sums in one fixed 64 KiB array in device memory,
 * declared in the library, instead of asking for memory.
 *   - n may be at most GB_DOT_NOALLOC_MAX_N; larger n is rejected with
 *     GOOSEBERRY_ERROR_INVALIDINPUT before anything runs.
 *   - The first call on each device looks up that array's device address
 *     (with that device current) and remembers it for the device's CUDA
 *     context: make that first call before any stream capture.  After a
 *     cudaDeviceReset the next call is again a first call (new context).
 *   - Every call on a device shares the one array, and it keeps the previous
 *     call's partial sums (each call writes every entry it reads first), so
 *     calls whose kernels overlap on the GPU (different streams, or threads
 *     racing) corrupt each other's result: serialise them.
 * The array stays allocated on every GPU that loaded the library until the
 * process exits.  No counterpart in the reference.
 */
#define GB_DOT_NOALLOC_MAX_N ((size_t)16384 * 8192)
GOOSEBERRY_API int gb_dot_f64_noalloc(size_t n, const double * a, const double * b,
    double * result, gb_stream_t stream);
/* v *= s (blas_scale, src/blas.c:244-257); v += s (blas_add_scalar,
 * src/blas.c:397-410); c = a + b (blas_add, src/blas.c:275-290);
 * c = a - b (blas_sub, src/blas.c:321-336).  c may alias a or b. */
GOOSEBERRY_API int gb_scale_f64(size_t n, double * v, double s, gb_stream_t stream);
GOOSEBERRY_API int gb_add_scalar_f64(size_t n, double * v, double s, gb_stream_t stream);
GOOSEBERRY_API int gb_add_f64(size_t n, const double * a, const double * b, double * c,
    gb_stream_t stream);
GOOSEBERRY_API int gb_sub_f64(size_t n, const double * a, const double * b, double * c,
    gb_stream_t stream);
GOOSEBERRY_API int gb_scale_f32(size_t n, float * v, float s, gb_stream_t stream);
GOOSEBERRY_API int gb_add_scalar_f32(size_t n, float * v, float s, gb_stream_t stream);

/* ---- conjugate gradient --------------------------------------------------- */

typedef enum gb_cg_mode {
  GB_CG_F64 = 0,   /* plain FP64 CG, the reference's algorithm             */
  GB_CG_MIXED = 1  /* FP32 values/vectors inside, FP64 residual refinement  */
} gb_cg_mode_t;

/* OR-ed into the mode of gb_cg_create: run the whole solve as ONE persistent
 * cooperative launch (CTAs own fixed rows; two grid barriers per iteration)
 * instead of the default two graph-replayed kernels per iteration.  Taken
 * only when every row fits a tile and the grid can be co-resident; it holds
 * every SM until the solve ends. */
#define GB_CG_PERSISTENT 0x100

/* The FP64 solver's SpMV on the row schedule normally reads a compressed copy
 * of the matrix entries that it builds at create time when the matrix allows:
 * columns as 16-bit distances from the row (every entry within 32767 of the
 * diagonal) and values as 8-bit codes into a table (at most 256 distinct
 * values) or as floats (every value exactly a float).  Decoding is exact, so
 * results are bit-identical to the plain arrays; only the bytes streamed per
 * iteration shrink.  OR this flag into the mode to read the plain CSR arrays
 * instead. */
#define GB_CG_PLAIN_ENTRIES 0x200

typedef enum gb_cg_status {
  GB_CG_CONVERGED = 0,  /* ||r|| <= tolerance                                 */
  GB_CG_MAXITER = 1,    /* iteration limit reached first                      */
  GB_CG_BREAKDOWN = 2,  /* p.Ap <= 0: matrix not SPD                          */
  GB_CG_NONFINITE = 3,  /* NaN or Inf appeared                                */
  GB_CG_CANCELLED = 4,  /* stopped by gb_cg_cancel / gb_server_cancel; x is
                           the iterate of the last finished iteration        */
  GB_CG_TIMEOUT = 5     /* a GB_CG_PERSISTENT solve gave up at a grid barrier
                           that not every CTA reached within the limit (2 s
                           unless set by gb_cg_set_barrier_fault); the call
                           returns GOOSEBERRY_ERROR_UNKNOWN with this status
                           in the result, rnorm NaN; x is not meaningful     */
} gb_cg_status_t;

typedef struct gb_cg_result {
  size_t iterations;    /* CG iterations run (inner iterations for MIXED)     */
  size_t refinements;   /* FP64 residual recomputations (MIXED)               */
  double rnorm;         /* final ||b - A x||_2 as tracked by the solver       */
  double bnorm;         /* ||b||_2                                            */
  int status;           /* gb_cg_status_t                                     */
  size_t kernel_launches; /* GPU kernels this solve launched                  */
} gb_cg_result_t;

/* Allocate the workspace of a CG solver for matrix a (the matrix must hold
 * the value widths the mode needs: F64 for GB_CG_F64, F64 and F32 for
 * GB_CG_MIXED).  Reference: the five work vectors cgd allocates per call
 * (src/cgd.c:67-77). */
GOOSEBERRY_API int gb_cg_create(const gb_csr_t * a, int mode, gb_cg_t ** out);
GOOSEBERRY_API int gb_cg_destroy(gb_cg_t * s);

/*
 * Solve A x = b from x0 = 0 with device vectors b, x.  Stops when
 * ||r||_2 <= tol (tol_relative == 0: absolute, the reference's rule,
 * src/cgd.c:115-119) or ||r||_2 <= tol * ||b||_2 (tol_relative != 0), or
 * after niter iterations (0: no limit).  history (optional, HOST pointer)
 * receives ||r||_2 after each iteration, up to history_len entries.
 * Synchronous on `stream` (returns after the solve finished).
 */
GOOSEBERRY_API int gb_cg_solve(gb_cg_t * s, const double * b, double * x, double tol,
    int tol_relative, size_t niter, double * history, size_t history_len,
    gb_cg_result_t * result, gb_stream_t stream);

/* Ask the solver's running gb_cg_solve (called on another thread) to stop.
 * Safe to call from any thread at any time.  The solve ends at its next
 * check -- between graph replays, or, for a GB_CG_PERSISTENT solve, at the
 * next iteration's first grid barrier, which every CTA then leaves -- and
 * reports GB_CG_CANCELLED with the iterations it finished.  A request made
 * while no solve runs stops the next solve at its first check; a solve that
 * stopped on a request clears it.  The reference's cgd cannot be stopped
 * (src/cgd.c:87-119); no counterpart. */
GOOSEBERRY_API int gb_cg_cancel(gb_cg_t * s);

/* Failure-path hook for GB_CG_PERSISTENT solves, for tests of the bounded
 * grid barrier: from the next gb_cg_solve on, CTA `drop_cta` (>= 0) does not
 * arrive at the solve's first grid barrier and leaves, so the other CTAs
 * wait out the barrier limit, raise the abort flag and leave too; the solve
 * returns GOOSEBERRY_ERROR_UNKNOWN with status GB_CG_TIMEOUT.  `limit_ms` sets the barrier limit (0 keeps 2000);
 * drop_cta < 0 turns the fault off.  Nothing waits without a limit, so the
 * device stays usable.  No reference counterpart (cgd runs on the host). */
GOOSEBERRY_API int gb_cg_set_barrier_fault(gb_cg_t * s, int drop_cta, unsigned limit_ms);

/*
 * Measurement hook: start a solve of A x = b and run its first `iterations`
 * iterations launch by launch, timing every launch with CUDA events on
 * `stream`.  ms[k] receives the mean duration in milliseconds of kernel k of
 * an iteration (k < nkernels; F64: 0 = SpMV+direction+p.Ap, 1 = x/r update +
 * r.r).  Returns the number of kernels per iteration in *nkernels.  Leaves
 * the solver ready for the next gb_cg_solve.  No reference counterpart (the
 * reference only has wall-clock phase timers, src/gooseberry_bin.c:2078-2113).
 */
GOOSEBERRY_API int gb_cg_profile(gb_cg_t * s, const double * b, size_t iterations,
    double * ms, size_t ms_len, size_t * nkernels, gb_stream_t stream);

/* Bytes per matrix entry the solver's SpMV streams: 12 for the plain arrays
 * (4-byte column, 8-byte value); 2 + the value bytes with 16-bit column
 * distances, F64 values as 8-bit codes (1), exact floats (4) or doubles (8)
 * (see GB_CG_PLAIN_ENTRIES); 0 on a pattern matrix (rows of at most 7 entries
 * forming at most 256 distinct lists of column offsets from the diagonal:
 * stencils), whose values the solver keeps in rows of fixed width (see
 * gb_cg_row_bytes).  No reference counterpart. */
GOOSEBERRY_API int gb_cg_entry_bytes(const gb_cg_t * s, size_t * bytes);

/* Bytes per row the solver's SpMV streams besides the entries: 4 (rowptr);
 * on a pattern matrix a pattern byte and the row's zero-padded values or
 * codes instead: 9 (8 codes), 33 (8 floats; MIXED, or exact floats), 49 or
 * 65 (6 or 8 doubles); 5 (rowptr and a pattern byte) for MIXED in builds
 * without its rows of values.  No reference counterpart. */
GOOSEBERRY_API int gb_cg_row_bytes(const gb_cg_t * s, size_t * bytes);

/* ---- batched solve server (continuous batching) ---------------------------- */

/*
 * Many independent CG solves of uneven sizes resident on one GPU at once.
 * Every gb_server_step runs `iters_per_step` CG iterations of EVERY resident
 * solve with one replay of a captured CUDA graph (the kernels walk a global
 * list of small row tiles covering all resident solves, so a 1k-row and a
 * 262k-row system advance together), retires the solves that finished
 * (their x is copied to the caller's buffer) and admits queued requests into
 * the freed slots and device memory.  Admission is by device-memory
 * footprint, bounded by pool_bytes.  No reference counterpart (the reference
 * runs one cgd call at a time, src/gooseberry_bin.c:2078-2091).
 *
 * Host memory: a server pins a staging arena of pool_bytes / 8, at least
 * 64 MiB and at most 2 GiB, for the life of the server.  Submitted requests
 * are copied there, so admission uploads them asynchronously; requests that
 * find the arena full are copied to ordinary memory instead.
 */
typedef struct gb_server gb_server_t;

typedef struct gb_server_config {
  size_t pool_bytes;        /* device memory for resident solves             */
  uint32_t max_slots;       /* resident solves at most                       */
  int mode;                 /* GB_CG_MIXED or GB_CG_F64                      */
  uint32_t iters_per_step;  /* CG iterations per gb_server_step (>= 1)       */
  uint32_t tile_rows;       /* rows per work tile (a power of two in
                               [256, 65536]), or 0: chosen per request by the
                               tile autotuner (gb_server_tuned_tile_rows)    */
} gb_server_config_t;

typedef struct gb_server_result {
  uint64_t id;
  size_t iterations;
  size_t refinements;
  double rnorm;             /* final ||b - A x||_2 (FP64, true residual for
                               GB_CG_MIXED; recurrence residual for F64)     */
  double bnorm;
  int status;               /* gb_cg_status_t                                */
  double t_submit, t_admit, t_done;  /* seconds on the server clock        */
} gb_server_result_t;

GOOSEBERRY_API int gb_server_create(const gb_server_config_t * cfg, gb_server_t ** out);
GOOSEBERRY_API int gb_server_destroy(gb_server_t * s);

/* Queue one solve of A x = b (square CSR, host arrays, copied at once) to
 * relative residual tol_rel or niter iterations.  x_out (host, n doubles)
 * must stay valid until the result is reported by gb_server_poll.  Rows may
 * hold at most 255 nonzeros.  Returns INVALIDINPUT for malformed input or a
 * request that could never fit the pool. */
GOOSEBERRY_API int gb_server_submit(gb_server_t * s, uint64_t id, dim_t n,
    const ind_t * rowptr, const dim_t * rowind, const double * rowval, const double * b,
    double * x_out, double tol_rel, size_t niter);

/* One scheduling step (see above).  Returns at once after queueing the
 * step's GPU work; *active / *queued (optional) receive the resident and
 * waiting request counts. */
GOOSEBERRY_API int gb_server_step(gb_server_t * s, size_t * active, size_t * queued);

/* Move up to `max` finished results into `out`; *count receives how many. */
GOOSEBERRY_API int gb_server_poll(gb_server_t * s, gb_server_result_t * out, size_t max,
    size_t * count);

/* Cancel request `id`.  A queued request is dropped at once; a resident one
 * is retired at the next gb_server_step (its slot and memory are freed and
 * x_out is left as it was).  Either way gb_server_poll then reports it with
 * status GB_CG_CANCELLED.  INVALIDINPUT if no queued or resident request has
 * that id (it was never submitted, or has already finished).  The reference
 * has no server, so no counterpart. */
GOOSEBERRY_API int gb_server_cancel(gb_server_t * s, uint64_t id);

/* Seconds since the server was created (the clock of the result stamps). */
GOOSEBERRY_API double gb_server_clock(const gb_server_t * s);

/* Where a server's time went. */
typedef struct gb_server_stats {
  size_t steps;             /* graph replays launched                        */
  double gpu_ms;            /* their device time (CUDA events)               */
  double wait_ms;           /* host time in gb_server_step waiting for the
                               previous replay to finish                     */
  double host_ms;           /* the rest of gb_server_step: retiring, admitting,
                               the tile list and slot table upload           */
  double submit_ms;         /* host time in gb_server_submit (copies, checks,
                               tile autotuning)                              */
  size_t tunings;           /* tile autotuner runs this server started       */
} gb_server_stats_t;
GOOSEBERRY_API int gb_server_stats(const gb_server_t * s, gb_server_stats_t * out);

/*
 * The tile autotuner.  The batched kernels walk a list of row tiles; a
 * request's rows are cut into tiles when it is submitted, from the request
 * alone, so its arithmetic (and result bits) do not depend on what else is
 * resident.  With tile_rows = 0 the size comes from a process-wide cache
 * keyed on the request's row-length class -- its longest row (rows of up to
 * 5, 7, 15, 63 or 255 entries), log2 of its row count and the server mode.
 * A key met for the first time is tuned on the spot: the request is
 * replicated into a batch that fills the GPU (in memory outside the pool),
 * and a few CG iterations of that batch are timed for each candidate size
 * (1024 to 16384 rows, no larger than the request); the fastest is cached.
 * gb_server_tuned_tile_rows reports the cached choice for a key (0: not
 * tuned yet).  No reference counterpart.
 */
GOOSEBERRY_API int gb_server_tuned_tile_rows(int mode, uint32_t n, uint32_t max_row_nnz,
    uint32_t * tile_rows);

#ifdef __cplusplus
}
#endif

#endif /* GOOSEBERRY_B200_H */
