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
  SCHED_MERGE = GB_SCHED_MERGE
};

constexpr int kSpmvBlock = 256;

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

__device__ __forceinline__ uint32_t ld_stream(const uint32_t * p, uint64_t pol) {
  uint32_t v;
  asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.u32 %0, [%1], %2;"
               : "=r"(v) : "l"(p), "l"(pol));
  return v;
}
__device__ __forceinline__ double ld_stream(const double * p, uint64_t pol) {
  double v;
  asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.f64 %0, [%1], %2;"
               : "=d"(v) : "l"(p), "l"(pol));
  return v;
}
__device__ __forceinline__ float ld_stream(const float * p, uint64_t pol) {
  float v;
  asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.f32 %0, [%1], %2;"
               : "=f"(v) : "l"(p), "l"(pol));
  return v;
}
__device__ __forceinline__ double ld_keep(const double * p, uint64_t pol) {
  double v;
  asm volatile("ld.global.nc.L2::cache_hint.f64 %0, [%1], %2;"
               : "=d"(v) : "l"(p), "l"(pol));
  return v;
}
__device__ __forceinline__ float ld_keep(const float * p, uint64_t pol) {
  float v;
  asm volatile("ld.global.nc.L2::cache_hint.f32 %0, [%1], %2;"
               : "=f"(v) : "l"(p), "l"(pol));
  return v;
}

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
  __device__ __forceinline__ X operator()(uint32_t c, uint64_t pol) const {
    return ld_keep(x + c, pol);
  }
};

// ---- the tile kernel ----------------------------------------------------------

template <typename Acc>
struct TileSmem {
  // products (tile_items entries) followed by row offsets (tile_items + 1)
  static __host__ __device__ size_t bytes(uint32_t tile_items) {
    return sizeof(Acc) * tile_items + sizeof(uint32_t) * (tile_items + 1) + 16;
  }
};

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

// The persistent tile kernel.  V: stored value type; Acc: product/accumulator
// type; Gather: x-access functor; Out: per-row epilogue with
//   row(row, Acc)                -- one finished row
//   long_row(lid, row, Acc)      -- a finished long row (single thread)
//   finish()                     -- once per thread after the last tile
template <typename V, typename Acc, int SCHED, int BLOCK, class Gather, class Out>
__device__ __forceinline__ void spmv_tiles_body(const PlanView plan,
    const uint32_t * __restrict__ rowptr, const uint32_t * __restrict__ rowind,
    const V * __restrict__ val, const Gather gather, Out & out) {
  extern __shared__ __align__(16) unsigned char gb_smem[];
  __shared__ Acc scan_v[BLOCK / 32];
  __shared__ uint32_t scan_k[BLOCK / 32];
  __shared__ Acc red[32];
  __shared__ bool last_chunk;

  Acc * prod = reinterpret_cast<Acc *>(gb_smem);
  uint32_t * offs = reinterpret_cast<uint32_t *>(prod + plan.tile_items);
  const uint64_t pol_stream = policy_evict_first();
  const uint64_t pol_keep = policy_evict_last();
  const uint32_t cmax = plan.ncols - 1;
  const int tid = threadIdx.x;

  for (uint32_t t = blockIdx.x; t < plan.ntiles; t += gridDim.x) {
    const TileDesc d = plan.tiles[t];
    const uint32_t nb = d.nnz_begin;
    const int N = static_cast<int>(d.nnz_count);
    if (d.row_count == 0) {
      // ---- chunk of a long row: block tree sum, then last-arrival combine
      Acc s = Acc(0);
      for (int k = tid; k < N; k += BLOCK) {
        const uint32_t c = min(ld_stream(rowind + nb + k, pol_stream), cmax);
        s += static_cast<Acc>(ld_stream(val + nb + k, pol_stream)) * gather(c, pol_keep);
      }
      s = block_sum(s, red);
      if (tid == 0) {
        plan.chunk_partial[t] = static_cast<double>(s);
        __threadfence();
        const LongRowDesc L = plan.longrows[d.row_begin];
        const unsigned prev = atomicAdd(plan.long_count + d.row_begin, 1u);
        last_chunk = (prev == L.nchunks - 1);
        if (last_chunk) {
          __threadfence();
          Acc tot = Acc(0);
          for (uint32_t q = 0; q < L.nchunks; ++q)
            tot += static_cast<Acc>(__ldcg(plan.chunk_partial + L.first_tile + q));
          plan.long_count[d.row_begin] = 0u;  // ready for the next launch
          out.long_row(d.row_begin, L.row, tot);
        }
      }
      __syncthreads();
      continue;
    }
    const int R = static_cast<int>(d.row_count);
    // ---- stage row offsets and products
    for (int r = tid; r <= R; r += BLOCK) offs[r] = rowptr[d.row_begin + r] - nb;
    const uint32_t * ip = rowind + nb;
    const V * vp = val + nb;
    int k = tid;
    for (; k + 3 * BLOCK < N; k += 4 * BLOCK) {
      const uint32_t c0 = min(ld_stream(ip + k, pol_stream), cmax);
      const uint32_t c1 = min(ld_stream(ip + k + BLOCK, pol_stream), cmax);
      const uint32_t c2 = min(ld_stream(ip + k + 2 * BLOCK, pol_stream), cmax);
      const uint32_t c3 = min(ld_stream(ip + k + 3 * BLOCK, pol_stream), cmax);
      const V v0 = ld_stream(vp + k, pol_stream);
      const V v1 = ld_stream(vp + k + BLOCK, pol_stream);
      const V v2 = ld_stream(vp + k + 2 * BLOCK, pol_stream);
      const V v3 = ld_stream(vp + k + 3 * BLOCK, pol_stream);
      const Acc x0 = gather(c0, pol_keep);
      const Acc x1 = gather(c1, pol_keep);
      const Acc x2 = gather(c2, pol_keep);
      const Acc x3 = gather(c3, pol_keep);
      prod[k] = static_cast<Acc>(v0) * x0;
      prod[k + BLOCK] = static_cast<Acc>(v1) * x1;
      prod[k + 2 * BLOCK] = static_cast<Acc>(v2) * x2;
      prod[k + 3 * BLOCK] = static_cast<Acc>(v3) * x3;
    }
    for (; k < N; k += BLOCK) {
      const uint32_t c = min(ld_stream(ip + k, pol_stream), cmax);
      prod[k] = static_cast<Acc>(ld_stream(vp + k, pol_stream)) * gather(c, pol_keep);
    }
    __syncthreads();
    reduce_tile<SCHED, BLOCK, Acc>(prod, offs, d.row_begin, R, N, out, scan_v, scan_k);
    __syncthreads();
  }
  out.finish();
}

}  // namespace gb
