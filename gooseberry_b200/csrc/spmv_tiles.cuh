// spmv_tiles.cuh -- the tiled CSR SpMV kernel template (sm_100a).
//
// Computes y[i] = sum_{k in row i} val[k] * x[ind[k]] (reference
// src/blas.c:82-91) for every row of a CSR matrix.  Work is cut into the
// row-aligned tiles of a Plan (gb_internal.h).  One CTA handles one tile at a
// time, persistent over tiles in a fixed round-robin order:
//
//   1. stage: the tile's rowptr slice (as offsets relative to its first
//      nonzero) and the products val[k]*x[ind[k]] are written to shared
//      memory.  The rowind/rowval streams are read once, coalesced, with an
//      evict-first L2 policy; x is gathered through L2 with evict-last so it
//      stays resident while the matrix streams past.
//   2. reduce: the products are summed per row by the schedule SCHED:
//        THREAD  one thread per row (short, uniform rows),
//        GROUP<G> G lanes per row + shuffle tree (moderate rows),
//        MERGE   merge-path split of the tile's rows+nonzeros into equal
//                per-thread runs, with a block-wide segmented scan carrying
//                the partial sums of rows that cross threads (irregular rows).
//   3. each finished row is handed to the epilogue functor `Out`, which
//      stores y (plain SpMV) or fuses more work (the CG kernels).
//
// Chunk tiles of long rows are reduced with a block tree; each chunk leaves a
// partial in plan scratch and the last chunk to arrive (atomic ticket) sums
// the partials in chunk order.  All reduction orders are fixed by the plan,
// so results are bitwise reproducible run to run.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "gb_internal.h"

namespace gb {

enum : int {
  SCHED_THREAD = GB_SCHED_THREAD,
  SCHED_GROUP4 = GB_SCHED_GROUP4,
  SCHED_GROUP8 = GB_SCHED_GROUP8,
  SCHED_WARP = GB_SCHED_WARP,
  SCHED_MERGE = GB_SCHED_MERGE,
  SCHED_ROW = GB_SCHED_ROW,
  SCHED_WTILE = GB_SCHED_WTILE,
  SCHED_WMERGE = GB_SCHED_WMERGE
};

constexpr int kSpmvBlock = 256;
// Elements per thread whose loads are issued together, and the resident CTAs
// per SM the register budget is sized for (both tunable at build time).
#ifndef GB_SPMV_STAGE
#define GB_SPMV_STAGE 8
#endif
#ifndef GB_SPMV_MIN_BLOCKS
#define GB_SPMV_MIN_BLOCKS 3
#endif
constexpr int kStage = GB_SPMV_STAGE;
constexpr int kSpmvMinBlocks = GB_SPMV_MIN_BLOCKS;

// ---- cache-policy loads -------------------------------------------------------

__device__ __forceinline__ uint64_t policy_evict_first() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ uint64_t policy_evict_last() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
  return p;
}

// Each load exists twice: with an L2 eviction policy (a uint64_t from
// createpolicy: evict-first for a matrix stream, evict-last for gathered
// vectors) and plain (a NoHint tag).  The hinted form keeps an L2-sized
// working set resident across launches; on streams much larger than L2 and
// on random gathers it is slower than the plain form, so kernels take the
// policy as a type and the host picks per launch.
struct NoHint {};

#define GB_LD(NAME, T, REG, SUFFIX, HINTED, PLAIN)                                   \
  __device__ __forceinline__ T NAME(const T * p, uint64_t pol) {                   \
    T v;                                                                           \
    asm volatile(HINTED "." SUFFIX " %0, [%1], %2;" : "=" REG(v) : "l"(p), "l"(pol)); \
    return v;                                                                      \
  }                                                                                \
  __device__ __forceinline__ T NAME(const T * p, NoHint) {                         \
    T v;                                                                           \
    asm volatile(PLAIN "." SUFFIX " %0, [%1];" : "=" REG(v) : "l"(p));             \
    return v;                                                                      \
  }
// streamed once: no L1 allocation
GB_LD(ld_stream, uint32_t, "r", "u32", "ld.global.nc.L1::no_allocate.L2::cache_hint",
      "ld.global.nc.L1::no_allocate")
GB_LD(ld_stream, double, "d", "f64", "ld.global.nc.L1::no_allocate.L2::cache_hint",
      "ld.global.nc.L1::no_allocate")
GB_LD(ld_stream, float, "f", "f32", "ld.global.nc.L1::no_allocate.L2::cache_hint",
      "ld.global.nc.L1::no_allocate")
// read-only loads that DO allocate in L1 (for access patterns where several
// instructions of a warp touch the same sector, e.g. one row per lane)
GB_LD(ld_l1, uint32_t, "r", "u32", "ld.global.nc.L2::cache_hint", "ld.global.nc")
GB_LD(ld_l1, double, "d", "f64", "ld.global.nc.L2::cache_hint", "ld.global.nc")
GB_LD(ld_l1, float, "f", "f32", "ld.global.nc.L2::cache_hint", "ld.global.nc")
// gathered vector entries
GB_LD(ld_keep, double, "d", "f64", "ld.global.nc.L2::cache_hint", "ld.global.nc")
GB_LD(ld_keep, float, "f", "f32", "ld.global.nc.L2::cache_hint", "ld.global.nc")
#undef GB_LD

// The policy pair a kernel built with (HINT) or without L2 hints passes down.
template <bool HINT>
struct L2Pol;
template <>
struct L2Pol<true> {
  __device__ static uint64_t stream() { return policy_evict_first(); }
  __device__ static uint64_t keep() { return policy_evict_last(); }
};
template <>
struct L2Pol<false> {
  __device__ static NoHint stream() { return NoHint{}; }
  __device__ static NoHint keep() { return NoHint{}; }
};

// Round-to-nearest multiply and add that the compiler may not contract into
// a fused multiply-add (the reference's x86-64 build never fuses).
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }

// ---- shuffle helpers -----------------------------------------------------------

template <int G, typename T>
__device__ __forceinline__ T group_sum(T v) {
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

template <typename T>
__device__ __forceinline__ T block_sum(T v, T * red /* >= 32 entries */) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  v = group_sum<32>(v);
  __syncthreads();
  if (lane == 0) red[w] = v;
  __syncthreads();
  T s = T(0);
  if (threadIdx.x == 0) {
    const int nw = (blockDim.x + 31) >> 5;
    for (int i = 0; i < nw; ++i) s += red[i];  // fixed order
  }
  return s;  // valid in thread 0 only
}

// ---- the gather functors ------------------------------------------------------

// x[c] for a plain SpMV.
template <typename X>
struct GatherPlain {
  const X * x;
  template <class P>
  __device__ __forceinline__ X operator()(uint32_t c, P pol) const {
    return ld_keep(x + c, pol);
  }
};

// ---- the tile kernel ----------------------------------------------------------

// Shared-memory layout of the tile pipeline: two stages, each holding one
// tile's rowptr slice (tile_items + 1 entries), column indices and values
// (tile_items entries each), plus one product buffer.
template <typename V, typename Acc>
struct TileSmem {
  static __host__ __device__ size_t stage_bytes(uint32_t t) {
    const size_t offs = (sizeof(uint32_t) * (t + 1) + 15) & ~size_t(15);
    const size_t ind = (sizeof(uint32_t) * t + 15) & ~size_t(15);
    const size_t val = (sizeof(V) * t + 15) & ~size_t(15);
    return offs + ind + val;
  }
  static __host__ __device__ size_t bytes(uint32_t t) {
    return 2 * stage_bytes(t) + ((sizeof(Acc) * t + 15) & ~size_t(15));
  }
};

// cp.async (global -> shared, bypassing registers) with an L2 cache policy.
__device__ __forceinline__ void cp_async4(void * smem, const void * gmem, uint64_t pol) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.ca.shared.global.L2::cache_hint [%0], [%1], 4, %2;"
               :: "r"(s), "l"(gmem), "l"(pol) : "memory");
}
__device__ __forceinline__ void cp_async4(void * smem, const void * gmem, NoHint) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" :: "r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async8(void * smem, const void * gmem, uint64_t pol) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.ca.shared.global.L2::cache_hint [%0], [%1], 8, %2;"
               :: "r"(s), "l"(gmem), "l"(pol) : "memory");
}
__device__ __forceinline__ void cp_async8(void * smem, const void * gmem, NoHint) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" :: "r"(s), "l"(gmem) : "memory");
}
template <class P>
__device__ __forceinline__ void cp_async_v(void * smem, const double * g, P pol) {
  cp_async8(smem, g, pol);
}
template <class P>
__device__ __forceinline__ void cp_async_v(void * smem, const float * g, P pol) {
  cp_async4(smem, g, pol);
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" :: "n"(N) : "memory");
}

// Reduction of one staged tile.  `prod` holds the tile's products, `offs` the
// R+1 row offsets into prod.  Calls out.row(row, sum) once per row.
template <int SCHED, int BLOCK, typename Acc, class Out>
__device__ __forceinline__ void reduce_tile(const Acc * prod, const uint32_t * offs,
    uint32_t row0, int R, int N, Out & out, Acc * scan_v, uint32_t * scan_k) {
  const int tid = threadIdx.x;
  if (SCHED == SCHED_THREAD) {
    for (int r = tid; r < R; r += BLOCK) {
      Acc s = Acc(0);
      const uint32_t e = offs[r + 1];
      for (uint32_t k = offs[r]; k < e; ++k) s += prod[k];
      out.row(row0 + r, s);
    }
  } else if (SCHED == SCHED_GROUP4 || SCHED == SCHED_GROUP8 || SCHED == SCHED_WARP) {
    constexpr int G = SCHED == SCHED_GROUP4 ? 4 : (SCHED == SCHED_GROUP8 ? 8 : 32);
    constexpr int NG = BLOCK / G;
    const int g = tid / G, lane = tid % G;
    for (int base = 0; base < R; base += NG) {  // uniform trip count
      const int r = base + g;
      Acc s = Acc(0);
      if (r < R) {
        const uint32_t e = offs[r + 1];
        for (uint32_t k = offs[r] + lane; k < e; k += G) s += prod[k];
      }
      s = group_sum<G>(s);
      if (r < R && lane == 0) out.row(row0 + r, s);
    }
  } else {  // SCHED_MERGE
    const int items = R + N;
    const int per = (items + BLOCK - 1) / BLOCK;
    const int d0 = min(tid * per, items);
    const int d1 = min(d0 + per, items);
    // merge-path search on diagonal d0: smallest i with rowend(i) > d0-i-1
    int lo = max(0, d0 - N), hi = min(d0, R);
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (static_cast<int>(offs[mid + 1]) > d0 - mid - 1) hi = mid; else lo = mid + 1;
    }
    int i = lo, j = d0 - lo;
    const int i0 = i;
    Acc run = Acc(0), head = Acc(0);
    bool head_done = false;
    for (int d = d0; d < d1; ++d) {
      if (i < R && static_cast<int>(offs[i + 1]) <= j) {
        if (i == i0) { head = run; head_done = true; }
        else out.row(row0 + i, run);
        run = Acc(0);
        ++i;
      } else {
        run += prod[j];
        ++j;
      }
    }
    // segmented inclusive scan of (key = i, value = run) over threads
    const int lane = tid & 31, w = tid >> 5;
    uint32_t key = static_cast<uint32_t>(i);
    Acc v = run;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const Acc vu = __shfl_up_sync(0xffffffffu, v, o);
      const uint32_t ku = __shfl_up_sync(0xffffffffu, key, o);
      if (lane >= o && ku == key) v += vu;
    }
    if (lane == 31) { scan_v[w] = v; scan_k[w] = key; }
    __syncthreads();
    if (tid == 0) {
      for (int q = 1; q < BLOCK / 32; ++q)
        if (scan_k[q] == scan_k[q - 1]) scan_v[q] += scan_v[q - 1];
    }
    __syncthreads();
    if (w > 0 && key == scan_k[w - 1]) v += scan_v[w - 1];
    // carry-in = scanned value of thread tid-1 if it ended inside row i0
    Acc pv = __shfl_up_sync(0xffffffffu, v, 1);
    uint32_t pk = __shfl_up_sync(0xffffffffu, key, 1);
    if (lane == 0) {
      if (w > 0) { pv = scan_v[w - 1]; pk = scan_k[w - 1]; }
      else { pv = Acc(0); pk = 0xffffffffu; }
    }
    if (head_done) out.row(row0 + i0, (pk == static_cast<uint32_t>(i0) ? pv : Acc(0)) + head);
    __syncthreads();  // scan_v / scan_k reused by the next tile
  }
}

// Runs the tiles t_begin, t_begin + t_step, ... (< t_end) of a plan.
//
// Pipeline: while tile t is gathered and reduced, cp.async is already copying
// tile t + t_step's rowptr slice, indices and values into the other shared
// memory stage, so the matrix stream never waits behind the reduction.  Only
// the x gathers of the current tile are exposed latency; every thread issues
// kStage of them before consuming any.
//
// V: stored value type; Acc: product/accumulator type; Gather: x-access
// functor; Out: per-row epilogue with
//   row(row, Acc)                -- one finished row
//   long_row(lid, row, Acc)      -- a finished long row (called by one thread)
// `pol_matrix` is the L2 policy of the matrix stream (evict-first when the
// matrix cannot stay in L2, evict-normal/last when it can).
template <typename V, typename Acc, int SCHED, int BLOCK, class Gather, class Out, class PM,
    class PX>
__device__ __forceinline__ void spmv_tile_loop(const PlanView & plan, uint32_t t_begin,
    uint32_t t_end, uint32_t t_step, const uint32_t * __restrict__ rowptr,
    const uint32_t * __restrict__ rowind, const V * __restrict__ val,
    const Gather & gather, Out & out, PM pol_matrix, PX pol_x) {
  extern __shared__ __align__(16) unsigned char gb_smem[];
  __shared__ Acc scan_v[BLOCK / 32];
  __shared__ uint32_t scan_k[BLOCK / 32];
  __shared__ Acc red[32];

  const uint32_t T = plan.tile_items;
  const size_t sb = TileSmem<V, Acc>::stage_bytes(T);
  const size_t offs_b = (sizeof(uint32_t) * (T + 1) + 15) & ~size_t(15);
  const size_t ind_b = (sizeof(uint32_t) * T + 15) & ~size_t(15);
  Acc * prod = reinterpret_cast<Acc *>(gb_smem + 2 * sb);
  const uint32_t cmax = plan.ncols - 1;
  const int tid = threadIdx.x;

  auto stage_offs = [&](int s) { return reinterpret_cast<uint32_t *>(gb_smem + s * sb); };
  auto stage_ind = [&](int s) {
    return reinterpret_cast<uint32_t *>(gb_smem + s * sb + offs_b);
  };
  auto stage_val = [&](int s) { return reinterpret_cast<V *>(gb_smem + s * sb + offs_b + ind_b); };

  // queue the copies of tile t into stage s (chunk tiles stream from global)
  auto issue = [&](uint32_t t, int s) {
    const TileDesc d = plan.tiles[t];
    if (d.row_count != 0) {
      uint32_t * so = stage_offs(s);
      uint32_t * si = stage_ind(s);
      V * sv = stage_val(s);
      for (uint32_t r = tid; r <= d.row_count; r += BLOCK)
        cp_async4(so + r, rowptr + d.row_begin + r, pol_matrix);
      for (uint32_t k = tid; k < d.nnz_count; k += BLOCK) {
        cp_async4(si + k, rowind + d.nnz_begin + k, pol_matrix);
        cp_async_v(sv + k, val + d.nnz_begin + k, pol_matrix);
      }
    }
    cp_async_commit();
  };

  if (t_begin < t_end) issue(t_begin, 0);
  int s = 0;
  for (uint32_t t = t_begin; t < t_end; t += t_step) {
    const uint32_t tn = t + t_step;
    if (tn < t_end) issue(tn, s ^ 1); else cp_async_commit();
    cp_async_wait<1>();
    __syncthreads();
    const TileDesc d = plan.tiles[t];
    const uint32_t nb = d.nnz_begin;
    const int N = static_cast<int>(d.nnz_count);
    if (d.row_count == 0) {
      // ---- chunk of a long row: block tree sum, then last-arrival combine
      Acc sum = Acc(0);
      for (int base = 0; base < N; base += kStage * BLOCK) {
        uint32_t c[kStage];
        V v[kStage];
#pragma unroll
        for (int j = 0; j < kStage; ++j) {
          const int k = base + tid + j * BLOCK;
          if (k < N) {
            c[j] = ld_stream(rowind + nb + k, pol_matrix);
            v[j] = ld_stream(val + nb + k, pol_matrix);
          }
        }
#pragma unroll
        for (int j = 0; j < kStage; ++j) {
          const int k = base + tid + j * BLOCK;
          if (k < N) sum += static_cast<Acc>(v[j]) * gather(min(c[j], cmax), pol_x);
        }
      }
      sum = block_sum(sum, red);
      if (tid == 0) {
        plan.chunk_partial[t] = static_cast<double>(sum);
        __threadfence();
        const LongRowDesc L = plan.longrows[d.row_begin];
        const unsigned prev = atomicAdd(plan.long_count + d.row_begin, 1u);
        if (prev == L.nchunks - 1) {
          __threadfence();
          Acc tot = Acc(0);
          for (uint32_t q = 0; q < L.nchunks; ++q)
            tot += static_cast<Acc>(__ldcg(plan.chunk_partial + L.first_tile + q));
          plan.long_count[d.row_begin] = 0u;  // ready for the next launch
          out.long_row(d.row_begin, L.row, tot);
        }
      }
    } else {
      const int R = static_cast<int>(d.row_count);
      uint32_t * offs = stage_offs(s);
      const uint32_t * si = stage_ind(s);
      const V * sv = stage_val(s);
      for (int r = tid; r <= R; r += BLOCK) offs[r] -= nb;
      // products: kStage gathers in flight per thread
      for (int base = 0; base < N; base += kStage * BLOCK) {
        Acc xv[kStage];
#pragma unroll
        for (int j = 0; j < kStage; ++j) {
          const int k = base + tid + j * BLOCK;
          if (k < N) xv[j] = gather(min(si[k], cmax), pol_x);
        }
#pragma unroll
        for (int j = 0; j < kStage; ++j) {
          const int k = base + tid + j * BLOCK;
          if (k < N) prod[k] = static_cast<Acc>(sv[k]) * xv[j];
        }
      }
      __syncthreads();
      reduce_tile<SCHED, BLOCK, Acc>(prod, offs, d.row_begin, R, N, out, scan_v, scan_k);
    }
    __syncthreads();  // stage s and prod are free again
    s ^= 1;
  }
  cp_async_wait<0>();
}

// Row-parallel schedule: rows first, first + step, ... (< end), one thread per
// row, read straight from global memory (the L1 keeps the lines that
// neighbouring threads' rows share).  Each row is summed exactly like the
// reference's inner loop (src/blas.c:85-88): from 0, k ascending, the product
// rounded before the add (no fused multiply-add), so y is bit-identical to
// blas_spmult's.
//
// The loop is a three-stage register pipeline over a thread's rows: while the
// x values of row i are gathered, the indices/values (and the epilogue's
// per-row operands, Out::pre) of row i + step and the rowptr pair of row
// i + 2 step are already in flight, so a row costs about one memory round
// trip instead of three.  The first kRowStage entries of a row ride in the
// pipeline; longer rows finish their tail inline.
#ifndef GB_ROW_STAGE
#define GB_ROW_STAGE 6
#endif
#ifndef GB_ROW_MIN_BLOCKS
#define GB_ROW_MIN_BLOCKS 2
#endif
constexpr int kRowStage = GB_ROW_STAGE;
// resident CTAs per SM the register budget of a kernel is sized for
#ifndef GB_WMERGE_MIN_BLOCKS
#define GB_WMERGE_MIN_BLOCKS 3
#endif
template <int SCHED>
struct MinBlocks {
  static constexpr int value = SCHED == SCHED_ROW      ? GB_ROW_MIN_BLOCKS
                               : SCHED == SCHED_WMERGE ? GB_WMERGE_MIN_BLOCKS
                                                       : kSpmvMinBlocks;
};

// ---- entry codecs of the row schedule ------------------------------------------
//
// How a row-schedule kernel reads entry k of the matrix.  Besides the plain
// CSR arrays, two lossless encodings shrink the matrix stream (after the
// index and value compression of Kourtis, Goumas and Koziris, "Optimizing
// sparse matrix-vector multiplication using index and value compression",
// CF 2008): a column stored as its signed 16-bit distance from the row
// (when every entry lies within 32767 of the diagonal), and a value stored as
// an 8-bit code into a table of the matrix's distinct values (when it has at
// most 256).  A value stored as float when the float equals the double
// exactly is ValPlain<float> widened to double.  Decoding gives back the exact
// column and double, so results are bit-identical to the plain arrays.

__device__ __forceinline__ int32_t ld_l1_s16(const int16_t * p, uint64_t pol) {
  int32_t v;
  asm volatile("ld.global.nc.L2::cache_hint.s16 %0, [%1], %2;" : "=r"(v) : "l"(p), "l"(pol));
  return v;
}
__device__ __forceinline__ int32_t ld_l1_s16(const int16_t * p, NoHint) {
  int32_t v;
  asm volatile("ld.global.nc.s16 %0, [%1];" : "=r"(v) : "l"(p));
  return v;
}
__device__ __forceinline__ uint32_t ld_l1_u8(const uint8_t * p, uint64_t pol) {
  uint32_t v;
  asm volatile("ld.global.nc.L2::cache_hint.u8 %0, [%1], %2;" : "=r"(v) : "l"(p), "l"(pol));
  return v;
}
__device__ __forceinline__ uint32_t ld_l1_u8(const uint8_t * p, NoHint) {
  uint32_t v;
  asm volatile("ld.global.nc.u8 %0, [%1];" : "=r"(v) : "l"(p));
  return v;
}

struct ColU32 {  // the CSR column array
  const uint32_t * p;
  using Raw = uint32_t;
  static constexpr bool kInRange = false;  // clamp before gathering
  static constexpr bool kPerRow = false;
  template <class P>
  __device__ __forceinline__ Raw load(uint32_t k, P pol) const { return ld_l1(p + k, pol); }
  __device__ __forceinline__ uint32_t col(Raw r, uint32_t) const { return r; }
};

struct ColD16 {  // column - row, 16-bit
  const int16_t * p;
  using Raw = int32_t;
  static constexpr bool kInRange = true;  // built from validated columns
  static constexpr bool kPerRow = false;
  template <class P>
  __device__ __forceinline__ Raw load(uint32_t k, P pol) const { return ld_l1_s16(p + k, pol); }
  __device__ __forceinline__ uint32_t col(Raw r, uint32_t row) const {
    return row + static_cast<uint32_t>(r);
  }
};

// Columns from a per-row pattern code.  A row's pattern is the list of its
// columns' offsets from the diagonal; a matrix whose rows have at most
// kPatMax entries and form at most 256 distinct patterns (structured-grid
// stencils: 27 on a 3-D 7-point operator) stores one byte per row instead of
// a column per entry, and the kernel keeps the pattern table (offsets, row
// lengths still from rowptr) in shared memory.  The index compression of
// Kourtis, Goumas and Koziris (CF 2008), taken from entries to whole rows.
constexpr int kPatMax = 8;
struct ColPat8 {
  const uint8_t * code;  // [nrows] pattern of each row
  const int32_t * off;   // [256 * kPatMax] offsets (the kernel's shared copy)
  using Raw = int32_t;
  static constexpr bool kInRange = true;  // built from validated columns
  static constexpr bool kPerRow = true;
  template <class P>
  __device__ __forceinline__ uint32_t row_code(uint32_t i, P pol) const {
    return ld_l1_u8(code + i, pol);
  }
  __device__ __forceinline__ Raw offset(uint32_t c, int j) const { return off[c * kPatMax + j]; }
  __device__ __forceinline__ uint32_t col(Raw r, uint32_t row) const {
    return row + static_cast<uint32_t>(r);
  }
};

template <typename V>
struct ValPlain {  // values as stored (float widens exactly to double)
  const V * p;
  using Raw = V;
  template <class P>
  __device__ __forceinline__ Raw load(uint32_t k, P pol) const { return ld_l1(p + k, pol); }
  template <typename Acc>
  __device__ __forceinline__ Acc value(Raw r) const { return static_cast<Acc>(r); }
};

struct ValCode8 {  // 8-bit code into the distinct-value table (shared memory)
  const uint8_t * p;
  const double * table;
  using Raw = uint32_t;
  template <class P>
  __device__ __forceinline__ Raw load(uint32_t k, P pol) const { return ld_l1_u8(p + k, pol); }
  template <typename Acc>
  __device__ __forceinline__ Acc value(Raw r) const { return static_cast<Acc>(table[r]); }
};

template <class IC, class VC, int STAGE>
struct RowStageC {
  uint32_t b = 0, e = 0;
  uint32_t code = 0;  // per-row column accessors: the row's pattern
  typename IC::Raw c[STAGE];
  typename VC::Raw v[STAGE];
};

template <class IC, class VC, int STAGE, class P>
__device__ __forceinline__ void row_stage_load_c(RowStageC<IC, VC, STAGE> & s, uint32_t i,
    const IC & ic, const VC & vc, P pol) {
  if constexpr (IC::kPerRow) {  // the offsets are read from the table when gathering
    s.code = ic.row_code(i, pol);
#pragma unroll
    for (int j = 0; j < STAGE; ++j)
      if (s.b + j < s.e) s.v[j] = vc.load(s.b + j, pol);
  } else {
#pragma unroll
    for (int j = 0; j < STAGE; ++j) {
      if (s.b + j < s.e) {
        s.c[j] = ic.load(s.b + j, pol);
        s.v[j] = vc.load(s.b + j, pol);
      }
    }
  }
}

template <typename Acc, int STAGE, class IC, class VC, class Gather, class Out, class PM,
    class PX>
__device__ __forceinline__ void spmv_row_loop_c(uint32_t first, uint32_t end, uint32_t step,
    uint32_t ncols, const uint32_t * __restrict__ rowptr, const IC & ic, const VC & vc,
    const Gather & gather, Out & out, PM pol_matrix, PX pol_x) {
  const uint32_t cmax = ncols - 1;
  if (first >= end) return;
  // stage L: row `first`; stage P: rowptr pair of row first + step
  RowStageC<IC, VC, STAGE> cur;
  cur.b = __ldg(rowptr + first);
  cur.e = __ldg(rowptr + first + 1);
  typename Out::Pre cur_pre = out.pre(first);
  row_stage_load_c(cur, first, ic, vc, pol_matrix);
  uint32_t nb = 0, ne = 0;
  if (first + step < end) {
    nb = __ldg(rowptr + first + step);
    ne = __ldg(rowptr + first + step + 1);
  }
  for (uint32_t i = first; i < end; i += step) {
    // issue the next row's indices/values/operands and the rowptr two ahead
    RowStageC<IC, VC, STAGE> nxt;
    typename Out::Pre nxt_pre{};
    const uint32_t i1 = i + step, i2 = i + 2 * step;
    if (i1 < end) {
      nxt.b = nb;
      nxt.e = ne;
      nxt_pre = out.pre(i1);
      row_stage_load_c(nxt, i1, ic, vc, pol_matrix);
    }
    if (i2 < end) {
      nb = __ldg(rowptr + i2);
      ne = __ldg(rowptr + i2 + 1);
    }
    // gather and sum the current row (reference order)
    Acc xv[STAGE];
#pragma unroll
    for (int j = 0; j < STAGE; ++j) {
      if (cur.b + j < cur.e) {
        uint32_t c;
        if constexpr (IC::kPerRow) c = ic.col(ic.offset(cur.code, j), i);
        else c = ic.col(cur.c[j], i);
        xv[j] = gather(IC::kInRange ? c : min(c, cmax), pol_x);
      }
    }
    Acc sum = Acc(0);
#pragma unroll
    for (int j = 0; j < STAGE; ++j)
      if (cur.b + j < cur.e)
        sum = add_rn(sum, mul_rn(vc.template value<Acc>(cur.v[j]), xv[j]));
    if constexpr (!IC::kPerRow) {  // pattern rows fit the stage: no tail
      for (uint32_t k = cur.b + STAGE; k < cur.e; ++k)  // long-row tail
        sum = add_rn(sum, mul_rn(vc.template value<Acc>(vc.load(k, pol_matrix)),
                                 gather(IC::kInRange ? ic.col(ic.load(k, pol_matrix), i)
                                                     : min(ic.col(ic.load(k, pol_matrix), i),
                                                           cmax),
                                        pol_x)));
    }
    out.row_pre(i, sum, cur_pre);
    cur = nxt;
    cur_pre = nxt_pre;
  }
}

// The row loop over the plain CSR arrays: the same pipeline written for the
// two arrays directly (kept separate from spmv_row_loop_c, whose generic form
// costs the FP32 kernels registers and occupancy).
template <typename V, int STAGE>
struct RowStage {
  uint32_t b = 0, e = 0;
  uint32_t c[STAGE];
  V v[STAGE];
};

template <typename V, int STAGE, class P>
__device__ __forceinline__ void row_stage_load(RowStage<V, STAGE> & s, const uint32_t * rowind,
    const V * val, P pol) {
#pragma unroll
  for (int j = 0; j < STAGE; ++j) {
    if (s.b + j < s.e) {
      s.c[j] = ld_l1(rowind + s.b + j, pol);
      s.v[j] = ld_l1(val + s.b + j, pol);
    }
  }
}

template <typename V, typename Acc, int STAGE = kRowStage, class Gather, class Out, class PM,
    class PX>
__device__ __forceinline__ void spmv_row_loop(uint32_t first, uint32_t end, uint32_t step,
    uint32_t ncols, const uint32_t * __restrict__ rowptr,
    const uint32_t * __restrict__ rowind, const V * __restrict__ val, const Gather & gather,
    Out & out, PM pol_matrix, PX pol_x) {
  const uint32_t cmax = ncols - 1;
  if (first >= end) return;
  // stage L: row `first`; stage P: rowptr pair of row first + step
  RowStage<V, STAGE> cur;
  cur.b = __ldg(rowptr + first);
  cur.e = __ldg(rowptr + first + 1);
  typename Out::Pre cur_pre = out.pre(first);
  row_stage_load(cur, rowind, val, pol_matrix);
  uint32_t nb = 0, ne = 0;
  if (first + step < end) {
    nb = __ldg(rowptr + first + step);
    ne = __ldg(rowptr + first + step + 1);
  }
  for (uint32_t i = first; i < end; i += step) {
    // issue the next row's indices/values/operands and the rowptr two ahead
    RowStage<V, STAGE> nxt;
    typename Out::Pre nxt_pre{};
    const uint32_t i1 = i + step, i2 = i + 2 * step;
    if (i1 < end) {
      nxt.b = nb;
      nxt.e = ne;
      nxt_pre = out.pre(i1);
      row_stage_load(nxt, rowind, val, pol_matrix);
    }
    if (i2 < end) {
      nb = __ldg(rowptr + i2);
      ne = __ldg(rowptr + i2 + 1);
    }
    // gather and sum the current row (reference order)
    Acc xv[STAGE];
#pragma unroll
    for (int j = 0; j < STAGE; ++j)
      if (cur.b + j < cur.e) xv[j] = gather(min(cur.c[j], cmax), pol_x);
    Acc sum = Acc(0);
#pragma unroll
    for (int j = 0; j < STAGE; ++j)
      if (cur.b + j < cur.e) sum = add_rn(sum, mul_rn(static_cast<Acc>(cur.v[j]), xv[j]));
    for (uint32_t k = cur.b + STAGE; k < cur.e; ++k)  // long-row tail
      sum = add_rn(sum, mul_rn(static_cast<Acc>(ld_l1(val + k, pol_matrix)),
                               gather(min(ld_l1(rowind + k, pol_matrix), cmax), pol_x)));
    out.row_pre(i, sum, cur_pre);
    cur = nxt;
    cur_pre = nxt_pre;
  }
}

// ---- per-warp tiles -----------------------------------------------------------
//
// Each warp is an independent pipeline over its own small row-aligned tiles:
// while its lanes sum tile t, cp.async already streams tile t + step (rowptr
// slice, indices, values) into the warp's other shared-memory stage.  Only
// warp-level synchronisation is needed, so every warp of the SM keeps its own
// tile in flight (the CTA-wide tile loop above has one per CTA).  Per tile
// the products are formed nonzero-parallel (lane k, k + 32, ...; kStage x
// gathers in flight per lane whatever the row lengths, each product rounded
// on its own and written over its value in shared memory), then a lane sums
// whole rows of products, k ascending, exactly like the reference's
// unfused multiply-then-add loop (src/blas.c:85-88): the result is
// bit-identical to blas_spmult.

template <typename V>
struct WarpSmem {
  static __host__ __device__ size_t stage_bytes(uint32_t t) {
    return ((sizeof(uint32_t) * (t + 1) + 15) & ~size_t(15)) +
           ((sizeof(uint32_t) * t + 15) & ~size_t(15)) + ((sizeof(V) * t + 15) & ~size_t(15));
  }
  static __host__ __device__ size_t bytes(uint32_t t, int warps) {
    return static_cast<size_t>(warps) * 2 * stage_bytes(t);
  }
};

template <typename V, typename Acc, class Gather, class Out, class PM, class PX>
__device__ __forceinline__ void spmv_warp_loop(const PlanView & plan, uint32_t t_first,
    uint32_t t_end, uint32_t t_step, const uint32_t * __restrict__ rowptr,
    const uint32_t * __restrict__ rowind, const V * __restrict__ val, const Gather & gather,
    Out & out, PM pol_matrix, PX pol_x) {
  extern __shared__ __align__(16) unsigned char gb_smem[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t T = plan.tile_items;
  const size_t sb = WarpSmem<V>::stage_bytes(T);
  const size_t offs_b = (sizeof(uint32_t) * (T + 1) + 15) & ~size_t(15);
  const size_t ind_b = (sizeof(uint32_t) * T + 15) & ~size_t(15);
  unsigned char * mine = gb_smem + static_cast<size_t>(warp) * 2 * sb;
  const uint32_t cmax = plan.ncols - 1;

  auto offs_of = [&](int s) { return reinterpret_cast<uint32_t *>(mine + s * sb); };
  auto ind_of = [&](int s) { return reinterpret_cast<uint32_t *>(mine + s * sb + offs_b); };
  auto val_of = [&](int s) { return reinterpret_cast<V *>(mine + s * sb + offs_b + ind_b); };

  auto issue = [&](uint32_t t, int s) {
    const TileDesc d = plan.tiles[t];
    if (d.row_count != 0) {
      uint32_t * so = offs_of(s);
      uint32_t * si = ind_of(s);
      V * sv = val_of(s);
      for (uint32_t r = lane; r <= d.row_count; r += 32)
        cp_async4(so + r, rowptr + d.row_begin + r, pol_matrix);
      for (uint32_t k = lane; k < d.nnz_count; k += 32) {
        cp_async4(si + k, rowind + d.nnz_begin + k, pol_matrix);
        cp_async_v(sv + k, val + d.nnz_begin + k, pol_matrix);
      }
    }
    cp_async_commit();
  };

  if (t_first < t_end) issue(t_first, 0);
  int s = 0;
  for (uint32_t t = t_first; t < t_end; t += t_step) {
    const uint32_t tn = t + t_step;
    if (tn < t_end) issue(tn, s ^ 1); else cp_async_commit();
    cp_async_wait<1>();
    __syncwarp();
    const TileDesc d = plan.tiles[t];
    const uint32_t nb = d.nnz_begin;
    if (d.row_count == 0) {
      // chunk of a long row: the warp sums it, then last-arrival combine
      const int N = static_cast<int>(d.nnz_count);
      Acc sum = Acc(0);
      for (int base = 0; base < N; base += kStage * 32) {
        uint32_t c[kStage];
        V v[kStage];
#pragma unroll
        for (int j = 0; j < kStage; ++j) {
          const int k = base + lane + j * 32;
          if (k < N) {
            c[j] = ld_stream(rowind + nb + k, pol_matrix);
            v[j] = ld_stream(val + nb + k, pol_matrix);
          }
        }
#pragma unroll
        for (int j = 0; j < kStage; ++j) {
          const int k = base + lane + j * 32;
          if (k < N) sum += static_cast<Acc>(v[j]) * gather(min(c[j], cmax), pol_x);
        }
      }
      sum = group_sum<32>(sum);
      if (lane == 0) {
        plan.chunk_partial[t] = static_cast<double>(sum);
        __threadfence();
        const LongRowDesc L = plan.longrows[d.row_begin];
        const unsigned prev = atomicAdd(plan.long_count + d.row_begin, 1u);
        if (prev == L.nchunks - 1) {
          __threadfence();
          Acc tot = Acc(0);
          for (uint32_t q = 0; q < L.nchunks; ++q)
            tot += static_cast<Acc>(__ldcg(plan.chunk_partial + L.first_tile + q));
          plan.long_count[d.row_begin] = 0u;  // ready for the next launch
          out.long_row(d.row_begin, L.row, tot);
        }
      }
    } else {
      const uint32_t * so = offs_of(s);
      const uint32_t * si = ind_of(s);
      V * sv = val_of(s);
      // products, nonzero-parallel: every lane keeps kStage gathers in flight
      // whatever the row lengths; each product replaces its value in place
      const int N = static_cast<int>(d.nnz_count);
      for (int base = 0; base < N; base += kStage * 32) {
        Acc xv[kStage];
#pragma unroll
        for (int j = 0; j < kStage; ++j) {
          const int k = base + lane + j * 32;
          if (k < N) xv[j] = gather(min(si[k], cmax), pol_x);
        }
#pragma unroll
        for (int j = 0; j < kStage; ++j) {
          const int k = base + lane + j * 32;
          if (k < N) sv[k] = static_cast<V>(mul_rn(static_cast<Acc>(sv[k]), xv[j]));
        }
      }
      __syncwarp();
      // row sums, one row per lane, k ascending (the reference's order)
      for (uint32_t r = lane; r < d.row_count; r += 32) {
        const uint32_t i = d.row_begin + r;
        const typename Out::Pre pre = out.pre(i);
        const uint32_t b = so[r] - nb, e = so[r + 1] - nb;
        Acc sum = Acc(0);
        for (uint32_t k = b; k < e; ++k) sum = add_rn(sum, static_cast<Acc>(sv[k]));
        out.row_pre(i, sum, pre);
      }
    }
    __syncwarp();  // stage s is free again
    s ^= 1;
  }
  cp_async_wait<0>();
}

// ---- plain SpMV: direct register pipeline -------------------------------------
//
// For y = A x the tile's column indices and values are used only by the
// thread that gathers for them, so they need no shared-memory staging: each
// thread owns the items k = tid + j * BLOCK of a tile and loads their indices
// and values straight into registers (coalesced), one tile ahead.  Per tile:
// the x gathers of the current tile are issued first, then the next tile's
// index/value loads and the current tile's rowptr slice; the products go to
// shared memory only for the row reduction (the same reduce_tile as the staged
// loop, so rows are summed in the same order).  This keeps the L1 traffic to
// the gathers, the matrix stream and one product write + read per nonzero
// (the staged loop also writes and reads indices and values through shared
// memory), and it holds fewer registers, so more CTAs stay resident.
template <typename X>
struct IsPlainGather {
  static constexpr bool value = false;
};
template <typename X>
struct IsPlainGather<GatherPlain<X>> {
  static constexpr bool value = true;
};

// Plain y = A x on the row schedule: a 7-entry stage at three CTAs per SM
// (the 4096^2 Laplacian, 1.34 GB: 0.67 -> 0.94 of the copy peak against a
// 6-entry stage at two; the 160^3 operator 0.64 -> 0.76).  The CG kernels,
// whose epilogue and gathers carry more state, keep MinBlocks<SCHED_ROW>.
#ifndef GB_PLAIN_ROW_STAGE
#define GB_PLAIN_ROW_STAGE 7
#endif
#ifndef GB_PLAIN_ROW_MIN_BLOCKS
#define GB_PLAIN_ROW_MIN_BLOCKS 3
#endif
constexpr int kPlainRowStage = GB_PLAIN_ROW_STAGE;
template <int SCHED, class Gather>
struct TileMinBlocks {
  static constexpr int value = (SCHED == SCHED_ROW && IsPlainGather<Gather>::value)
                                   ? GB_PLAIN_ROW_MIN_BLOCKS
                                   : MinBlocks<SCHED>::value;
};

// Shared memory of the direct loop: rowptr slice (tile_items + 1) and products.
template <typename Acc>
struct DirectSmem {
  static __host__ __device__ size_t offs_bytes(uint32_t t) {
    return (sizeof(uint32_t) * (t + 1) + 15) & ~size_t(15);
  }
  static __host__ __device__ size_t bytes(uint32_t t) {
    return offs_bytes(t) + ((sizeof(Acc) * t + 15) & ~size_t(15));
  }
};

#ifndef GB_DIRECT_KT
#define GB_DIRECT_KT 4
#endif
#ifndef GB_DIRECT_MIN_BLOCKS
#define GB_DIRECT_MIN_BLOCKS 6
#endif
#ifndef GB_DIRECT_BLOCK
#define GB_DIRECT_BLOCK 128
#endif
constexpr int kDirectKt = GB_DIRECT_KT;  // items per thread per tile (tile <= kDirectKt * BLOCK)
constexpr int kDirectMinBlocks = GB_DIRECT_MIN_BLOCKS;
constexpr int kDirectBlock = GB_DIRECT_BLOCK;  // threads per CTA of the direct loop

template <typename V, typename Acc, int SCHED, int BLOCK, class Out, class PM, class PX>
__device__ __forceinline__ void spmv_direct_loop(const PlanView & plan, uint32_t t_begin,
    uint32_t t_end, uint32_t t_step, const uint32_t * __restrict__ rowptr,
    const uint32_t * __restrict__ rowind, const V * __restrict__ val,
    const Acc * __restrict__ x, Out & out, PM pol_matrix, PX pol_x) {
  extern __shared__ __align__(16) unsigned char gb_smem[];
  __shared__ Acc scan_v[BLOCK / 32];
  __shared__ uint32_t scan_k[BLOCK / 32];
  __shared__ Acc red[32];
  constexpr int KT = kDirectKt;
  const uint32_t T = plan.tile_items;
  uint32_t * offs = reinterpret_cast<uint32_t *>(gb_smem);
  Acc * prod = reinterpret_cast<Acc *>(gb_smem + DirectSmem<Acc>::offs_bytes(T));
  const uint32_t cmax = plan.ncols - 1;
  const int tid = threadIdx.x;

  // per-tile register state: indices (loaded two tiles ahead), values and
  // rowptr slice (one tile ahead), gathered x (issued one tile ahead)
  uint32_t c[KT];
  V v[KT];
  Acc xv[KT];
  uint32_t o[KT + 1];
  auto load_ind = [&](const TileDesc & d) {
    if (d.row_count == 0) return;  // long-row chunks stream when they run
#pragma unroll
    for (int j = 0; j < KT; ++j) {
      const uint32_t k = tid + j * BLOCK;
      if (k < d.nnz_count) c[j] = ld_stream(rowind + d.nnz_begin + k, pol_matrix);
    }
  };
  auto load_rest = [&](const TileDesc & d) {  // values and rowptr slice
    if (d.row_count == 0) return;
#pragma unroll
    for (int j = 0; j < KT; ++j) {
      const uint32_t k = tid + j * BLOCK;
      if (k < d.nnz_count) v[j] = ld_stream(val + d.nnz_begin + k, pol_matrix);
    }
#pragma unroll
    for (int j = 0; j <= KT; ++j) {
      const uint32_t r = tid + j * BLOCK;
      if (r <= d.row_count) o[j] = __ldg(rowptr + d.row_begin + r);
    }
  };
  auto gather_all = [&](const TileDesc & d) {
    if (d.row_count == 0) return;
#pragma unroll
    for (int j = 0; j < KT; ++j) {
      const uint32_t k = tid + j * BLOCK;
      if (k < d.nnz_count) xv[j] = ld_keep(x + min(c[j], cmax), pol_x);
    }
  };
  auto tile_at = [&](uint32_t t) { return t < t_end ? plan.tiles[t] : TileDesc{0, 1, 0, 0}; };

  if (t_begin >= t_end) return;
  TileDesc d_cur = plan.tiles[t_begin];
  TileDesc d_nxt = tile_at(t_begin + t_step);
  TileDesc d_nn = tile_at(t_begin + 2 * t_step);
  load_ind(d_cur);
  load_rest(d_cur);
  gather_all(d_cur);
  load_ind(d_nxt);
  for (uint32_t t = t_begin; t < t_end; t += t_step) {
    const bool has_next = t + t_step < t_end;
    const uint32_t nb = d_cur.nnz_begin;
    const int N = static_cast<int>(d_cur.nnz_count);
    if (d_cur.row_count == 0) {
      // ---- chunk of a long row (up to kChunkTiles tiles of nonzeros): stream
      // indices and values, KT gathers in flight per thread
      Acc sum = Acc(0);
      for (int base = 0; base < N; base += KT * BLOCK) {
        uint32_t cc[KT];
        V vv[KT];
#pragma unroll
        for (int j = 0; j < KT; ++j) {
          const int k = base + tid + j * BLOCK;
          if (k < N) {
            cc[j] = ld_stream(rowind + nb + k, pol_matrix);
            vv[j] = ld_stream(val + nb + k, pol_matrix);
          }
        }
        Acc xx[KT];
#pragma unroll
        for (int j = 0; j < KT; ++j) {
          const int k = base + tid + j * BLOCK;
          if (k < N) xx[j] = ld_keep(x + min(cc[j], cmax), pol_x);
        }
#pragma unroll
        for (int j = 0; j < KT; ++j) {
          const int k = base + tid + j * BLOCK;
          if (k < N) sum += static_cast<Acc>(vv[j]) * xx[j];
        }
      }
      // start the next tile (its indices are in c) before this chunk's reduction
      if (has_next) {
        load_rest(d_nxt);
        gather_all(d_nxt);
        load_ind(d_nn);
      }
      const TileDesc d_n3 = tile_at(t + 3 * t_step);
      sum = block_sum(sum, red);
      if (tid == 0) {
        plan.chunk_partial[t] = static_cast<double>(sum);
        __threadfence();
        const LongRowDesc L = plan.longrows[d_cur.row_begin];
        const unsigned prev = atomicAdd(plan.long_count + d_cur.row_begin, 1u);
        if (prev == L.nchunks - 1) {
          __threadfence();
          Acc tot = Acc(0);
          for (uint32_t q = 0; q < L.nchunks; ++q)
            tot += static_cast<Acc>(__ldcg(plan.chunk_partial + L.first_tile + q));
          plan.long_count[d_cur.row_begin] = 0u;  // ready for the next launch
          out.long_row(d_cur.row_begin, L.row, tot);
        }
      }
      __syncthreads();
      d_cur = d_nxt;
      d_nxt = d_nn;
      d_nn = d_n3;
      continue;
    }
    // ---- row tile: products and rowptr slice into shared memory
    const int R = static_cast<int>(d_cur.row_count);
#pragma unroll
    for (int j = 0; j < KT; ++j) {
      const int k = tid + j * BLOCK;
      if (k < N) prod[k] = static_cast<Acc>(v[j]) * xv[j];
    }
#pragma unroll
    for (int j = 0; j <= KT; ++j) {
      const int r = tid + j * BLOCK;
      if (r <= R) offs[r] = o[j] - nb;
    }
    __syncthreads();
    // the next tile's gathers and loads are in flight during this reduction
    if (has_next) {
      gather_all(d_nxt);
      load_rest(d_nxt);
      load_ind(d_nn);
    }
    const TileDesc d_n3 = tile_at(t + 3 * t_step);
    reduce_tile<SCHED, BLOCK, Acc>(prod, offs, d_cur.row_begin, R, N, out, scan_v, scan_k);
    __syncthreads();  // offs / prod are free again
    d_cur = d_nxt;
    d_nxt = d_nn;
    d_nn = d_n3;
  }
}

// ---- per-warp merge tiles ------------------------------------------------------
//
// Per-warp tiles of at most 32 * kWmKt items (rows + nonzeros), no CTA-wide
// barrier anywhere: every warp is its own pipeline.  Lanes own the items
// lane + 32 j of a tile; their column indices are loaded two tiles ahead,
// values and the rowptr slice one tile ahead, and the x gathers of tile t + 1
// are issued before tile t is reduced, so gathers stay in flight while the
// warp reduces.  The products and the rowptr slice go to the warp's own
// shared memory; the reduction walks the merge path of (row ends, nonzeros):
// each lane takes an equal share of it whatever the row lengths, sums its run
// of products sequentially, and a segmented shuffle scan carries the partial
// sums of rows that span lanes.  A row's sum is thus a short left-to-right
// sum per lane plus a tree over at most 32 lanes (within the condition-scaled
// tolerance of the reference's sequential sum, not bit-identical).  Long rows
// are chunks as in the other schedules.
#ifndef GB_WMERGE_KT
#define GB_WMERGE_KT 4
#endif
constexpr int kWmKt = GB_WMERGE_KT;  // items per lane per tile: tile_items <= 32 * kWmKt

template <typename Acc>
struct WMergeSmem {
  static __host__ __device__ size_t offs_bytes(uint32_t t) {
    return (sizeof(uint32_t) * (t + 1) + 15) & ~size_t(15);
  }
  static __host__ __device__ size_t warp_bytes(uint32_t t) {
    return offs_bytes(t) + ((sizeof(Acc) * t + 15) & ~size_t(15));
  }
  static __host__ __device__ size_t bytes(uint32_t t, int warps) {
    return static_cast<size_t>(warps) * warp_bytes(t);
  }
};

template <typename V, typename Acc, class Gather, class Out, class PM, class PX>
__device__ __forceinline__ void spmv_wmerge_loop(const PlanView & plan, uint32_t t_first,
    uint32_t t_end, uint32_t t_step, const uint32_t * __restrict__ rowptr,
    const uint32_t * __restrict__ rowind, const V * __restrict__ val, const Gather & gather,
    Out & out, PM pol_matrix, PX pol_x) {
  extern __shared__ __align__(16) unsigned char gb_smem[];
  constexpr int KT = kWmKt;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t T = plan.tile_items;
  unsigned char * mine = gb_smem + static_cast<size_t>(warp) * WMergeSmem<Acc>::warp_bytes(T);
  uint32_t * offs = reinterpret_cast<uint32_t *>(mine);
  Acc * prod = reinterpret_cast<Acc *>(mine + WMergeSmem<Acc>::offs_bytes(T));
  const uint32_t cmax = plan.ncols - 1;

  uint32_t c[KT];
  V v[KT];
  Acc xv[KT];
  uint32_t o[KT + 1];
  auto load_ind = [&](const TileDesc & d) {
    if (d.row_count == 0) return;  // long-row chunks stream when they run
#pragma unroll
    for (int j = 0; j < KT; ++j) {
      const uint32_t k = lane + j * 32;
      if (k < d.nnz_count) c[j] = ld_stream(rowind + d.nnz_begin + k, pol_matrix);
    }
  };
  auto load_rest = [&](const TileDesc & d) {  // values and rowptr slice
    if (d.row_count == 0) return;
#pragma unroll
    for (int j = 0; j < KT; ++j) {
      const uint32_t k = lane + j * 32;
      if (k < d.nnz_count) v[j] = ld_stream(val + d.nnz_begin + k, pol_matrix);
    }
#pragma unroll
    for (int j = 0; j <= KT; ++j) {
      const uint32_t r = lane + j * 32;
      if (r <= d.row_count) o[j] = __ldg(rowptr + d.row_begin + r);
    }
  };
  auto gather_all = [&](const TileDesc & d) {
    if (d.row_count == 0) return;
#pragma unroll
    for (int j = 0; j < KT; ++j) {
      const uint32_t k = lane + j * 32;
      if (k < d.nnz_count) xv[j] = gather(min(c[j], cmax), pol_x);
    }
  };
  auto tile_at = [&](uint32_t t) { return t < t_end ? plan.tiles[t] : TileDesc{0, 1, 0, 0}; };

  if (t_first >= t_end) return;
  TileDesc d_cur = plan.tiles[t_first];
  TileDesc d_nxt = tile_at(t_first + t_step);
  TileDesc d_nn = tile_at(t_first + 2 * t_step);
  load_ind(d_cur);
  load_rest(d_cur);
  gather_all(d_cur);
  load_ind(d_nxt);
  for (uint32_t t = t_first; t < t_end; t += t_step) {
    const bool has_next = t + t_step < t_end;
    const uint32_t nb = d_cur.nnz_begin;
    const int N = static_cast<int>(d_cur.nnz_count);
    if (d_cur.row_count == 0) {
      // ---- chunk of a long row: the warp streams it, KT gathers per lane
      Acc sum = Acc(0);
      for (int base = 0; base < N; base += KT * 32) {
        uint32_t cc[KT];
        V vv[KT];
#pragma unroll
        for (int j = 0; j < KT; ++j) {
          const int k = base + lane + j * 32;
          if (k < N) {
            cc[j] = ld_stream(rowind + nb + k, pol_matrix);
            vv[j] = ld_stream(val + nb + k, pol_matrix);
          }
        }
        Acc xx[KT];
#pragma unroll
        for (int j = 0; j < KT; ++j) {
          const int k = base + lane + j * 32;
          if (k < N) xx[j] = gather(min(cc[j], cmax), pol_x);
        }
#pragma unroll
        for (int j = 0; j < KT; ++j) {
          const int k = base + lane + j * 32;
          if (k < N) sum += static_cast<Acc>(vv[j]) * xx[j];
        }
      }
      if (has_next) {
        load_rest(d_nxt);
        gather_all(d_nxt);
        load_ind(d_nn);
      }
      const TileDesc d_n3 = tile_at(t + 3 * t_step);
      sum = group_sum<32>(sum);
      if (lane == 0) {
        plan.chunk_partial[t] = static_cast<double>(sum);
        __threadfence();
        const LongRowDesc L = plan.longrows[d_cur.row_begin];
        const unsigned prev = atomicAdd(plan.long_count + d_cur.row_begin, 1u);
        if (prev == L.nchunks - 1) {
          __threadfence();
          Acc tot = Acc(0);
          for (uint32_t q = 0; q < L.nchunks; ++q)
            tot += static_cast<Acc>(__ldcg(plan.chunk_partial + L.first_tile + q));
          plan.long_count[d_cur.row_begin] = 0u;  // ready for the next launch
          out.long_row(d_cur.row_begin, L.row, tot);
        }
      }
      __syncwarp();
      d_cur = d_nxt;
      d_nxt = d_nn;
      d_nn = d_n3;
      continue;
    }
    // ---- row tile: products and rowptr slice into the warp's shared memory
    const int R = static_cast<int>(d_cur.row_count);
    const uint32_t row0 = d_cur.row_begin;
#pragma unroll
    for (int j = 0; j < KT; ++j) {
      const int k = lane + j * 32;
      if (k < N) prod[k] = static_cast<Acc>(v[j]) * xv[j];
    }
#pragma unroll
    for (int j = 0; j <= KT; ++j) {
      const int r = lane + j * 32;
      if (r <= R) offs[r] = o[j] - nb;
    }
    __syncwarp();
    // the next tile's gathers and loads are in flight during this reduction
    if (has_next) {
      gather_all(d_nxt);
      load_rest(d_nxt);
      load_ind(d_nn);
    }
    const TileDesc d_n3 = tile_at(t + 3 * t_step);
    // merge path over (R row ends, N products): lane share [m0, m1)
    const int items = R + N;
    const int per = (items + 31) >> 5;
    const int m0 = min(lane * per, items);
    const int m1 = min(m0 + per, items);
    int lo = max(0, m0 - N), hi = min(m0, R);
    while (lo < hi) {  // smallest i with offs[i + 1] > m0 - i - 1
      const int mid = (lo + hi) >> 1;
      if (static_cast<int>(offs[mid + 1]) > m0 - mid - 1) hi = mid; else lo = mid + 1;
    }
    int i = lo, j = m0 - lo;
    const int i0 = i;
    Acc run = Acc(0), head = Acc(0);
    bool head_done = false;
    for (int m = m0; m < m1; ++m) {
      if (i < R && static_cast<int>(offs[i + 1]) <= j) {
        if (i == i0) { head = run; head_done = true; }
        else out.row(row0 + i, run);
        run = Acc(0);
        ++i;
      } else {
        run += prod[j];
        ++j;
      }
    }
    // segmented inclusive scan of (row, partial) over the lanes
    uint32_t key = static_cast<uint32_t>(i);
    Acc sc = run;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const Acc vu = __shfl_up_sync(0xffffffffu, sc, off);
      const uint32_t ku = __shfl_up_sync(0xffffffffu, key, off);
      if (lane >= off && ku == key) sc += vu;
    }
    Acc pv = __shfl_up_sync(0xffffffffu, sc, 1);
    const uint32_t pk = __shfl_up_sync(0xffffffffu, key, 1);
    if (head_done)
      out.row(row0 + i0, (lane > 0 && pk == static_cast<uint32_t>(i0) ? pv : Acc(0)) + head);
    __syncwarp();  // offs / prod are free again
    d_cur = d_nxt;
    d_nxt = d_nn;
    d_nn = d_n3;
  }
}

// Dynamic shared memory a schedule needs per CTA.
template <typename V, typename Acc>
__host__ __device__ inline size_t spmv_smem_bytes(int sched, uint32_t tile_items, int block) {
  if (sched == SCHED_ROW) return 0;
  if (sched == SCHED_WTILE) return WarpSmem<V>::bytes(tile_items, block / 32);
  if (sched == SCHED_WMERGE) return WMergeSmem<Acc>::bytes(tile_items, block / 32);
  return TileSmem<V, Acc>::bytes(tile_items);
}

// Work units a schedule distributes over CTAs (for the grid size).
inline uint32_t spmv_work_units(int sched, uint32_t nrows, uint32_t ntiles, int block) {
  if (sched == SCHED_ROW) return (nrows + block - 1) / block;
  if (sched == SCHED_WTILE || sched == SCHED_WMERGE)
    return (ntiles + block / 32 - 1) / (block / 32);
  return ntiles;
}

// Round-robin driver: CTA b runs tiles b, b + gridDim.x, ... (for the row
// schedule rows in a grid-stride loop, for per-warp tiles warp w of CTA b
// runs tiles b * warps + w, ...); then out.finish() once per thread.  HINT
// selects the L2-policy loads (L2Pol).
template <typename V, typename Acc, int SCHED, int BLOCK, class Gather, class Out,
    bool DIRECT = false, bool HINT = false>
__device__ __forceinline__ void spmv_tiles_body(const PlanView plan,
    const uint32_t * __restrict__ rowptr, const uint32_t * __restrict__ rowind,
    const V * __restrict__ val, const Gather gather, Out & out) {
  const auto pm = L2Pol<HINT>::stream();
  const auto px = L2Pol<HINT>::keep();
  if constexpr (SCHED == SCHED_ROW) {
    constexpr int STAGE = IsPlainGather<Gather>::value ? kPlainRowStage : kRowStage;
    spmv_row_loop<V, Acc, STAGE>(blockIdx.x * BLOCK + threadIdx.x, plan.nrows,
        gridDim.x * BLOCK, plan.ncols, rowptr, rowind, val, gather, out, pm, px);
  } else if constexpr (SCHED == SCHED_WTILE) {
    constexpr int W = BLOCK / 32;
    spmv_warp_loop<V, Acc>(plan, blockIdx.x * W + (threadIdx.x >> 5), plan.ntiles,
        gridDim.x * W, rowptr, rowind, val, gather, out, pm, px);
  } else if constexpr (SCHED == SCHED_WMERGE) {
    constexpr int W = BLOCK / 32;
    spmv_wmerge_loop<V, Acc>(plan, blockIdx.x * W + (threadIdx.x >> 5), plan.ntiles,
        gridDim.x * W, rowptr, rowind, val, gather, out, pm, px);
  } else if constexpr (DIRECT && IsPlainGather<Gather>::value) {
    spmv_direct_loop<V, Acc, SCHED, BLOCK>(plan, blockIdx.x, plan.ntiles, gridDim.x, rowptr,
        rowind, val, gather.x, out, pm, px);
  } else {
    spmv_tile_loop<V, Acc, SCHED, BLOCK>(plan, blockIdx.x, plan.ntiles, gridDim.x, rowptr,
        rowind, val, gather, out, pm, px);
  }
  out.finish();
}

}  // namespace gb
