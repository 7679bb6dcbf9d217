// spmv_seg.cuh -- the segmented SpMV schedule (GB_SCHED_SEG, sm_100a).
//
// Computes y[i] = sum_{k in row i} val[k] * x[ind[k]] (reference
// src/blas.c:82-91) for every row, with no CTA barrier and no row-aligned
// tiles.  The nonzeros are cut into one contiguous range per warp, balanced
// on rows + nonzeros (a merge-path split, rounded to multiples of 4 so every
// range starts on a 16-byte boundary of rowind and rowval).  A warp walks its
// range in windows of 32 * K nonzeros; lane l owns the K consecutive
// positions w0 + K l ... of a window:
//
//   * indices and values arrive with 128-bit loads (uint4 / double2 / float4),
//     indices two windows ahead, values one window ahead, and the x gathers of
//     window i + 1 are in flight while window i is reduced;
//   * the rows that start in a window are enumerated from rowptr, 32 at a
//     time (coalesced), and each marks its first position in a per-warp
//     shared-memory window with its row id (empty rows are written as 0);
//   * every lane sums its K products left to right, cutting at the marks;
//     rows that run across lanes are joined by a segmented inclusive scan over
//     the warp's lanes (shuffles), and across windows by a warp-uniform carry.
//
// Row lengths do not matter: a 3-nonzero row and a 200,000-nonzero row cost
// the same per nonzero.  A row that crosses warp ranges leaves one partial
// per warp (a "tail" record in the warps where it starts or runs through, a
// "head" record in the warp where it ends); each such warp takes a ticket on
// the end warp's counter and the last to arrive adds the partials in warp
// order (deterministic, like the tile plan's long-row chunks).  A row's sum is
// a left-to-right sum per lane joined by a shuffle tree: within the
// condition-scaled tolerance of the reference's sequential sum, not
// bit-identical to it.
#pragma once

#include "spmv_tiles.cuh"

namespace gb {

constexpr uint32_t kSegNone = 0xffffffffu;

#ifndef GB_SEG_BLOCK
#define GB_SEG_BLOCK 256
#endif
// Three CTAs of 256 threads per SM (85 registers): the FP64 form spills at
// four (64 registers) and ran the 8M-row power-law SpMV in 0.82 ms against
// 0.66 ms at three; the FP32 form is as fast at three as at four.
#ifndef GB_SEG_MIN_BLOCKS
#define GB_SEG_MIN_BLOCKS 3
#endif
#ifndef GB_SEG_K
#define GB_SEG_K 4
#endif
constexpr int kSegBlock = GB_SEG_BLOCK;
constexpr int kSegMinBlocks = GB_SEG_MIN_BLOCKS;
constexpr int kSegWarps = kSegBlock / 32;

// Device view of a segmented plan (SegPlan, gb_internal.h).
struct SegView {
  const SegRange * ranges;  // [nwarps + 1]; ranges[nwarps].nz_begin == nnz
  double * head_rec;        // [nwarps] partial of the row a warp finishes
  double * tail_rec;        // [nwarps] partial of the row a warp leaves open
  unsigned int * count;     // [nwarps] tickets, indexed by the finishing warp
  uint32_t nwarps, nrows, ncols, nnz;
};

// ---- 128-bit streaming loads --------------------------------------------------

// (An evict-first L2 policy on these loads, to keep x resident against the
// matrix stream, made the 8M-row power-law SpMV slower: 0.65 -> 0.81 ms; so
// did letting them allocate in L1: 0.65 -> 0.73 ms.)
__device__ __forceinline__ void ld_stream4(const uint32_t * p, uint32_t * o) {
  asm volatile("ld.global.nc.L1::no_allocate.v4.u32 {%0, %1, %2, %3}, [%4];"
               : "=r"(o[0]), "=r"(o[1]), "=r"(o[2]), "=r"(o[3])
               : "l"(p));
}
__device__ __forceinline__ void ld_stream4(const double * p, double * o) {
  asm volatile("ld.global.nc.L1::no_allocate.v2.f64 {%0, %1}, [%2];"
               : "=d"(o[0]), "=d"(o[1])
               : "l"(p));
  asm volatile("ld.global.nc.L1::no_allocate.v2.f64 {%0, %1}, [%2];"
               : "=d"(o[2]), "=d"(o[3])
               : "l"(p + 2));
}
__device__ __forceinline__ void ld_stream4(const float * p, float * o) {
  asm volatile("ld.global.nc.L1::no_allocate.v4.f32 {%0, %1, %2, %3}, [%4];"
               : "=f"(o[0]), "=f"(o[1]), "=f"(o[2]), "=f"(o[3])
               : "l"(p));
}

// K consecutive entries from position q (a multiple of 4) of a stream, the
// ones at or past `lim` read as zero.  Whole groups of four take one 16-byte
// load; only a range's last, partial group is read element by element.
template <int K, typename T>
__device__ __forceinline__ void seg_load(const T * __restrict__ a, uint32_t q, uint32_t lim,
    T * o) {
#pragma unroll
  for (int g = 0; g < K / 4; ++g) {
    const uint32_t p = q + 4 * g;
    if (p + 4 <= lim) {
      ld_stream4(a + p, o + 4 * g);
    } else {
#pragma unroll
      for (int j = 0; j < 4; ++j)
        o[4 * g + j] = p + j < lim ? ld_stream(a + p + j, NoHint{}) : T(0);
    }
  }
}

__device__ __forceinline__ uint32_t lanemask_lt() {
  uint32_t m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// rowptr[r] for r <= nrows, else "past everything".
__device__ __forceinline__ uint32_t seg_rowptr(const uint32_t * __restrict__ rowptr,
    uint32_t r, uint32_t nrows) {
  return r <= nrows ? __ldg(rowptr + r) : 0xffffffffu;
}

// Marks the rows that start in positions [a, b) of the matrix: flags[start -
// w0] = row for a non-empty row, y = 0 for an empty one.  `cursor` is the
// first row whose start is >= a and `rp` holds rowptr[cursor + lane]; returns
// the first row whose start is >= b and leaves rp = rowptr[that + lane].
template <class Out>
__device__ __forceinline__ uint32_t seg_enumerate(uint32_t w0, uint32_t b, uint32_t cursor,
    uint32_t & rp, const uint32_t * __restrict__ rowptr, uint32_t nrows, uint32_t * flags,
    Out & out, int lane) {
  for (;;) {
    const uint32_t r = cursor + lane;
    const bool in = r < nrows && rp < b;
    const unsigned m = __ballot_sync(0xffffffffu, in);  // a prefix of the lanes
    uint32_t nx = __shfl_down_sync(0xffffffffu, rp, 1);
    if (in) {
      if (lane == 31) nx = __ldg(rowptr + r + 1);
      if (nx > rp) flags[rp - w0] = r;
      else out.row(r, 0);
    }
    const int cnt = __popc(m);
    cursor += cnt;
    rp = cnt == 0 ? rp : seg_rowptr(rowptr, cursor + lane, nrows);
    if (cnt < 32) return cursor;
  }
}

// Adds a partial of a row that crosses warp ranges; the last of the row's
// warps to arrive writes the row.  Called by one lane.
template <typename Acc, class Out>
__device__ __forceinline__ void seg_ticket(const SegView & sv, uint32_t wb, uint32_t row,
    Out & out) {
  __threadfence();
  const SegRange E = sv.ranges[wb];
  const unsigned prev = atomicAdd(sv.count + wb, 1u);
  if (prev + 1 != E.span_count) return;
  __threadfence();
  Acc s = Acc(0);
  uint32_t nb = sv.ranges[E.head_first].nz_begin;
  for (uint32_t u = E.head_first; u < wb; ++u) {
    const uint32_t ne = sv.ranges[u + 1].nz_begin;
    if (ne > nb) s += static_cast<Acc>(__ldcg(sv.tail_rec + u));
    nb = ne;
  }
  s += static_cast<Acc>(__ldcg(sv.head_rec + wb));
  sv.count[wb] = 0u;  // ready for the next launch
  out.row(row, s);
}

template <typename V, typename Acc, int K, class Out>
__device__ __forceinline__ void spmv_seg_body(const SegView sv,
    const uint32_t * __restrict__ rowptr, const uint32_t * __restrict__ rowind,
    const V * __restrict__ val, const Acc * __restrict__ x, Out & out) {
  constexpr uint32_t WIN = 32 * K;
  __shared__ __align__(16) uint32_t seg_flags[kSegWarps][WIN];
  const int lane = threadIdx.x & 31;
  const uint32_t w = blockIdx.x * kSegWarps + (threadIdx.x >> 5);
  if (w >= sv.nwarps) return;
  uint32_t * flags = seg_flags[threadIdx.x >> 5];
  const SegRange R = sv.ranges[w];
  const uint32_t nz0 = R.nz_begin, nz1 = sv.ranges[w + 1].nz_begin;
  const uint32_t nrows = sv.nrows, cmax = sv.ncols - 1;

  uint32_t cursor = R.row_begin;
  uint32_t rp = seg_rowptr(rowptr, cursor + lane, nrows);
  if (nz1 > nz0) {
    const uint32_t nwin = (nz1 - nz0 + WIN - 1) / WIN;
#pragma unroll
    for (int j = 0; j < K; ++j) flags[K * lane + j] = kSegNone;

    // window registers: indices two windows ahead, gathers one, values loaded
    // once the window before is reduced
    uint32_t c_nx[K];
    V v_cur[K];
    Acc x_cur[K], x_nx[K];
    const uint32_t q0 = nz0 + K * lane;
    {
      uint32_t c0[K];
      seg_load<K>(rowind, q0, nz1, c0);
      seg_load<K>(val, q0, nz1, v_cur);
#pragma unroll
      for (int j = 0; j < K; ++j) x_cur[j] = q0 + j < nz1 ? __ldg(x + min(c0[j], cmax)) : Acc(0);
    }
    if (nwin > 1) seg_load<K>(rowind, q0 + WIN, nz1, c_nx);
    __syncwarp();
    cursor = seg_enumerate(nz0, min(nz0 + WIN, nz1), cursor, rp, rowptr, nrows, flags, out,
        lane);

    // the row open at the window start, and its partial sum so far
    uint32_t cur_row = R.head_row;
    Acc carry = Acc(0);
    for (uint32_t i = 0; i < nwin; ++i) {
      const uint32_t w0 = nz0 + i * WIN;
      const uint32_t q = w0 + K * lane;
      if (i + 1 < nwin) {  // gathers of window i + 1
#pragma unroll
        for (int j = 0; j < K; ++j)
          x_nx[j] = q + WIN + j < nz1 ? __ldg(x + min(c_nx[j], cmax)) : Acc(0);
      }
      if (i + 2 < nwin) seg_load<K>(rowind, q + 2 * WIN, nz1, c_nx);
      __syncwarp();  // window i's marks are written

      // ---- reduce window i
      uint32_t f[K];
#pragma unroll
      for (int j = 0; j < K; j += 4) {
        const uint4 t = *reinterpret_cast<const uint4 *>(flags + K * lane + j);
        f[j] = t.x;
        f[j + 1] = t.y;
        f[j + 2] = t.z;
        f[j + 3] = t.w;
        *reinterpret_cast<uint4 *>(flags + K * lane + j) =
            make_uint4(kSegNone, kSegNone, kSegNone, kSegNone);
      }
      Acc acc = Acc(0), head = Acc(0);
      bool has = false;
      uint32_t prow = 0;
#pragma unroll
      for (int j = 0; j < K; ++j) {
        if (f[j] != kSegNone) {
          if (has) out.row(prow, acc);  // a row that starts and ends in this lane
          else head = acc;
          has = true;
          prow = f[j];
          acc = Acc(0);
        }
        acc = fma(static_cast<Acc>(v_cur[j]), x_cur[j], acc);
      }
      // segmented inclusive scan of the lanes' open tails
      const unsigned hm = __ballot_sync(0xffffffffu, has);
      const unsigned le = hm & (lanemask_lt() | (1u << lane));
      const int seg0 = le ? 31 - __clz(le) : -1;  // nearest marked lane <= this one
      Acc sv_acc = acc;
#pragma unroll
      for (int off = 1; off < 32; off <<= 1) {
        const Acc up = __shfl_up_sync(0xffffffffu, sv_acc, off);
        if (lane - off >= seg0 && lane >= off) sv_acc = up + sv_acc;
      }
      if (seg0 < 0) sv_acc = carry + sv_acc;
      Acc cin = __shfl_up_sync(0xffffffffu, sv_acc, 1);
      if (lane == 0) cin = carry;
      const unsigned lt = hm & lanemask_lt();
      const int src = lt ? 31 - __clz(lt) : 0;
      const uint32_t prev_row = __shfl_sync(0xffffffffu, prow, src);
      if (has) {  // the row open at this lane's start ends before its first mark
        const uint32_t ro = lt ? prev_row : cur_row;
        if (ro != kSegNone) {
          const Acc v = cin + head;
          if (ro == R.head_row) {  // started in an earlier warp's range
            sv.head_rec[w] = static_cast<double>(v);
            seg_ticket<Acc>(sv, w, ro, out);
          } else {
            out.row(ro, v);
          }
        }
      }
      carry = __shfl_sync(0xffffffffu, sv_acc, 31);
      if (hm) cur_row = __shfl_sync(0xffffffffu, prow, 31 - __clz(hm));

      if (i + 1 < nwin) {  // values of window i + 1
        seg_load<K>(val, q + WIN, nz1, v_cur);
#pragma unroll
        for (int j = 0; j < K; ++j) x_cur[j] = x_nx[j];
        __syncwarp();  // every lane has read and cleared its marks
        cursor = seg_enumerate(w0 + WIN, min(w0 + 2 * WIN, nz1), cursor, rp, rowptr, nrows,
            flags, out, lane);
      }
    }
    // the row open at the range end
    if (lane == 0 && cur_row != kSegNone) {
      if (R.tail_last == kSegNone) {  // it ends here
        if (cur_row == R.head_row) {
          sv.head_rec[w] = static_cast<double>(carry);
          seg_ticket<Acc>(sv, w, cur_row, out);
        } else {
          out.row(cur_row, carry);
        }
      } else {
        sv.tail_rec[w] = static_cast<double>(carry);
        seg_ticket<Acc>(sv, R.tail_last, cur_row, out);
      }
    }
  }
  // rows after the last nonzero are empty
  if (w + 1 == sv.nwarps)
    for (uint32_t r = cursor + lane; r < nrows; r += 32) out.row(r, 0);
}

}  // namespace gb
