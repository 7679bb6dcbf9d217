// gb_internal.h -- shared internals of libgooseberry_b200 (not installed).
//
// Layout of a device-resident CSR matrix and of its SpMV tile plan, error
// plumbing and launch helpers used by the .cu/.cpp translation units.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <vector>

#include "gooseberry_b200.h"

namespace gb {

// ---- errors -----------------------------------------------------------------

// Record a printf-style message as this thread's last error.
void set_error(const char * fmt, ...);
void clear_error();

#define GB_CUDA_TRY(expr)                                                      \
  do {                                                                         \
    cudaError_t gb_e_ = (expr);                                                \
    if (gb_e_ != cudaSuccess) {                                                \
      ::gb::set_error("%s failed: %s (%s:%d)", #expr,                          \
          cudaGetErrorString(gb_e_), __FILE__, __LINE__);                      \
      return GOOSEBERRY_ERROR_UNKNOWN;                                         \
    }                                                                          \
  } while (0)

#define GB_TRY(expr)                                                           \
  do {                                                                         \
    int gb_rc_ = (expr);                                                       \
    if (gb_rc_ != GOOSEBERRY_SUCCESS) return gb_rc_;                           \
  } while (0)

#define GB_CHECK_INPUT(cond, ...)                                              \
  do {                                                                         \
    if (!(cond)) {                                                             \
      ::gb::set_error(__VA_ARGS__);                                            \
      return GOOSEBERRY_ERROR_INVALIDINPUT;                                    \
    }                                                                          \
  } while (0)

// ---- SpMV tile plan ---------------------------------------------------------
//
// The rows are cut, in order, into tiles.  A normal tile is a run of whole
// rows holding at most `tile_items` rows + nonzeros; its products are staged
// in shared memory and reduced there, so no row crosses a normal tile.  A row
// too long for one tile (nnz >= tile_items) is a "long row": it is cut into
// consecutive chunk tiles of at most `chunk_nnz` nonzeros each; every chunk
// writes a partial sum into the plan's scratch and the last chunk to finish
// adds them up in chunk order (deterministic).

struct TileDesc {
  uint32_t row_begin;  // normal: first row; chunk: index into the long-row table
  uint32_t row_count;  // normal: rows in the tile (>= 1); chunk: 0
  uint32_t nnz_begin;  // first nonzero of the tile (absolute index)
  uint32_t nnz_count;  // nonzeros in the tile
};

struct LongRowDesc {
  uint32_t row;         // the row
  uint32_t first_tile;  // its chunks are tiles [first_tile, first_tile+nchunks)
  uint32_t nchunks;
  uint32_t pad;
};

// Device view of a plan, passed by value to kernels.
struct PlanView {
  const TileDesc * tiles;
  const LongRowDesc * longrows;
  double * chunk_partial;     // [ntiles] partial sums of chunk tiles
  unsigned int * long_count;  // [nlong] chunk-arrival counters (kept at 0)
  uint32_t ntiles;
  uint32_t nlong;
  uint32_t tile_items;
  uint32_t ncols;
  uint32_t nrows;
};

// Segmented plan (the SEG schedule, spmv_seg.cuh): one contiguous range of
// nonzeros per warp, balanced on rows + nonzeros, every range starting at a
// multiple of 4.  A row that starts before a warp's range and ends in it is
// the warp's head row; the row open at the range end continues (tail_last)
// or ends there.
struct SegRange {
  uint32_t nz_begin;    // first nonzero of the range (multiple of 4)
  uint32_t row_begin;   // first row whose start is >= nz_begin
  uint32_t head_row;    // row holding nz_begin when it starts earlier, else ~0
  uint32_t head_first;  // warp holding head_row's first nonzero
  uint32_t tail_last;   // warp holding the last nonzero of the row open at the range end,
                        // when that row continues past it, else ~0
  uint32_t span_count;  // warps with nonzeros of head_row, when head_row ends here
  uint32_t pad0, pad1;
};

struct Plan {
  uint32_t tile_items = 0;
  uint32_t chunk_nnz = 0;
  std::vector<TileDesc> tiles;
  std::vector<LongRowDesc> longrows;
  // row-length summary
  uint32_t max_row = 0, p50 = 0, p90 = 0, p99 = 0;
  double mean_row = 0.0;
  // segmented plan ([nwarps + 1] ranges; empty until built)
  std::vector<SegRange> seg;
  // device copies
  TileDesc * d_tiles = nullptr;
  LongRowDesc * d_longrows = nullptr;
  double * d_chunk_partial = nullptr;
  unsigned int * d_long_count = nullptr;
  SegRange * d_seg = nullptr;
  double * d_seg_rec = nullptr;  // [2 nwarps]: head records, then tail records
  unsigned int * d_seg_count = nullptr;
};

// Build the tile plan from a HOST copy of rowptr.  Returns INVALIDINPUT if
// rowptr decreases or does not span nnz.
int build_plan(uint32_t nrows, const uint32_t * rowptr, uint32_t nnz,
    uint32_t tile_items, Plan & plan);
// The segmented ranges for at most `max_warps` warps (HOST rowptr, already
// validated by build_plan).
void build_seg_plan(uint32_t nrows, const uint32_t * rowptr, uint32_t nnz,
    uint32_t max_warps, Plan & plan);
// Warps a segmented plan is built for on the current device.
uint32_t seg_max_warps(int sm_count);
int upload_plan(Plan & plan, cudaStream_t stream);
void free_plan(Plan & plan);

}  // namespace gb

// ---- the opaque handles -----------------------------------------------------

struct gb_csr {
  uint32_t nrows = 0, ncols = 0, nnz = 0;
  int device = 0;
  const uint32_t * rowptr = nullptr;  // device
  const uint32_t * rowind = nullptr;  // device
  const double * val64 = nullptr;     // device (may be null)
  const float * val32 = nullptr;      // device (may be null)
  // owned allocations (freed by gb_csr_destroy)
  void * own_rowptr = nullptr;
  void * own_rowind = nullptr;
  void * own_val64 = nullptr;
  void * own_val32 = nullptr;
  gb::Plan plan;
  int sched64 = GB_SCHED_AUTO;  // resolved schedule (never AUTO after create)
  int sched32 = GB_SCHED_AUTO;
  int sm_count = 0;
};

namespace gb {

inline PlanView plan_view(const gb_csr & a) {
  PlanView v;
  v.tiles = a.plan.d_tiles;
  v.longrows = a.plan.d_longrows;
  v.chunk_partial = a.plan.d_chunk_partial;
  v.long_count = a.plan.d_long_count;
  v.ntiles = static_cast<uint32_t>(a.plan.tiles.size());
  v.nlong = static_cast<uint32_t>(a.plan.longrows.size());
  v.tile_items = a.plan.tile_items;
  v.ncols = a.ncols;
  v.nrows = a.nrows;
  return v;
}

// Heuristic schedule from the row-length summary (used until autotuned).
int default_schedule(const Plan & plan);

// SpMV launchers (spmv.cu).  `stride` is the output element stride (1 for
// SpMV; bncols for the columns of a row-major SpMM result).
int launch_spmv_f64(const gb_csr & a, int sched, const double * x, double * y,
    uint32_t stride, cudaStream_t stream);
int launch_spmv_f32(const gb_csr & a, int sched, const float * x, float * y,
    uint32_t stride, cudaStream_t stream);
// C = A B for k >= 2 right-hand sides in one pass over A (spmm.cu); B
// column-major ncols x k, C row-major nrows x k.  Sets *done = false (and does
// nothing) when the matrix has rows too long for the fused kernel.
template <typename T>
int launch_spmm_fused(const gb_csr & a, uint32_t k, const T * vals, const T * b, T * c,
    cudaStream_t stream, bool * done);
// max(rowind) over nnz into *d_out (device), for validation.
int launch_max_index(const uint32_t * rowind, uint32_t nnz, unsigned int * d_out,
    cudaStream_t stream);
int launch_round_f32(const double * in, float * out, size_t n, cudaStream_t stream);

int sm_count_of_current_device(int * out);
// Whether `bytes` of working set fit in the current device's L2 (the CG
// kernels use L2-policy loads only then).
int l2_fits(size_t bytes, bool * out);
// Stream-ordered scratch from the library-owned memory pool.
int scratch_alloc(void ** p, size_t bytes, cudaStream_t s);
void scratch_free(void * p, cudaStream_t s);
// Object memory from the same pool: dev_alloc returns memory usable from any
// stream; dev_free may only be called once no work that uses the memory can
// still run (the destroy paths synchronise the device first).
int dev_alloc(void ** p, size_t bytes);
void dev_free(void * p);
// A zeroed pinned host slot of at most 128 bytes that kernels can read and
// write through *dev (cancel flags, status mirrors); free only once no work
// that uses it can still run.
int pinned_slot_alloc(size_t bytes, void ** host, void ** dev);
void pinned_slot_free(void * host);
// Raise a kernel's dynamic shared-memory limit on the current device to at
// least `bytes` (above the 48 KiB default).  Never lowers it: a kernel that is
// launched, or captured in graphs, at several sizes keeps the largest limit
// any of them needed.
int raise_smem_limit(const void * func, size_t bytes);
template <typename T>
int dev_alloc(T ** p, size_t bytes) {
  return dev_alloc(reinterpret_cast<void **>(p), bytes);
}

// Wrap device arrays allocated with dev_alloc into a matrix that owns them
// (gb_csr_destroy frees them).  On failure the arrays stay the caller's.
int csr_adopt(uint32_t nrows, uint32_t ncols, uint32_t nnz, uint32_t * rowptr,
    uint32_t * rowind, double * val64, float * val32, cudaStream_t stream, gb_csr ** out);

// Lossless compressed entries for the row schedule (codec.cu): columns as
// int16 distances from the row, values as 8-bit codes into a table of the
// distinct values or as exact floats.  Null members are not available.
// Per-row column patterns (ColPat8, spmv_tiles.cuh): a byte per row naming
// one of npat offset lists of kPatMax entries.
struct RowPatterns {
  uint8_t * code8 = nullptr;  // [nrows]
  int32_t * off = nullptr;    // [npat * kPatMax]
  uint32_t npat = 0;
};
// Built when every row has at most 7 entries and the matrix has at most 256
// distinct patterns (checked column by column); else `out` stays empty.
int build_row_patterns(const gb_csr & a, RowPatterns * out, cudaStream_t s);
void free_row_patterns(RowPatterns & p);

struct RowCodec {
  int16_t * col16 = nullptr;  // col - row
  uint8_t * code8 = nullptr;  // code of each value
  double * table = nullptr;   // [ntable] distinct values
  uint32_t ntable = 0;
  float * val32 = nullptr;    // (float)value, equal to the double
  int stage = 6;              // row entries held in the pipeline (5, 6 or 7)
  size_t entry_bytes() const {
    return (col16 ? 2 : 4) + (code8 ? 1 : (val32 ? 4 : 8));
  }
};
int build_row_codec(const gb_csr & a, RowCodec * c, cudaStream_t s);
void free_row_codec(RowCodec & c);
// The int16 column distances alone (*out stays null when some entry is
// farther than 32767 from the diagonal); free with dev_free.
int build_col16(const gb_csr & a, int16_t ** out, cudaStream_t s);
// Register stage of the row loop for this matrix's longest row (5, 6 or 7).
int row_stage_for(const gb_csr & a);

// Mixed-precision CG (cg_mixed.cu), owned by a gb_cg created with GB_CG_MIXED.
struct MixedCg;
int mixed_create(const gb_csr * a, bool plain_entries, MixedCg ** out);
size_t mixed_entry_bytes(const MixedCg * m);
size_t mixed_row_bytes(const MixedCg * m);
void mixed_destroy(MixedCg * m);
// `cancel` (host memory, may be null): a nonzero value stops the solve
// between graph replays with status GB_CG_CANCELLED.
int mixed_solve(MixedCg * m, const double * b, double * x, double tol, int tol_relative,
    size_t niter, double * history, size_t history_len, gb_cg_result_t * res,
    cudaStream_t stream, const int * cancel = nullptr);
int mixed_profile(MixedCg * m, const double * b, size_t iterations, double * ms,
    size_t ms_len, size_t * nkernels, cudaStream_t stream);

}  // namespace gb
