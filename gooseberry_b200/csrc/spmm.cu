// spmm.cu -- C = A B for several right-hand sides in one launch (the
// reference's __sparse_mult_dense_block with bncols > 1, src/blas.c:67-92).
//
// B is column-major (B[j * ncols + c], the reference's layout), C row-major
// (C[i * k + j]).  One thread per row (grid-stride): the row's first
// kSpmmStage (or, when every row fits, 5) indices and values are loaded once
// into registers, then for each column j (two columns at a time on 5-entry
// rows) all of the row's gathers from those columns of B are issued before any
// is used, and C[i * k + j] is written.  Each element is summed k ascending
// with unfused multiply and add, exactly like the reference's inner loop, so C
// is bit-identical to blas_spmult's.  Against one SpMV per column, A's indices
// and values leave memory once instead of k times and the product is one
// launch; few registers per thread keep many rows in flight.  Matrices with
// rows too long for one thread keep the per-column SpMV.
#include <algorithm>

#include "gb_internal.h"
#include "spmv_tiles.cuh"

namespace gb {
namespace {

constexpr int kSpmmBlock = 256;
constexpr int kSpmmStage = 8;  // a row's entries held in registers (longer rows: tail loop)
// Rows of at most 5 entries (2D stencils) take a 5-entry stage, two columns of
// B at a time (both columns' gathers in flight together) and three CTAs per
// SM (80 registers, no spills): on the 1024^2 Laplacian with k = 8, 82.9 ->
// 66.1 us.  (The 5-entry stage one column at a time: 104.9 us; pairs at the
// default occupancy: 76.8 us.)  Longer rows keep the 8-entry stage, one column
// at a time.
#ifndef GB_SPMM_PAIRS
#define GB_SPMM_PAIRS 1
#endif
#ifndef GB_SPMM_MIN_BLOCKS
#define GB_SPMM_MIN_BLOCKS 3
#endif

template <typename T, int STAGE>
__global__ void __launch_bounds__(kSpmmBlock, STAGE <= 5 ? GB_SPMM_MIN_BLOCKS : 4) spmm_rows_kernel(uint32_t nrows, uint32_t ncols,
    uint32_t k, const uint32_t * __restrict__ rowptr, const uint32_t * __restrict__ rowind,
    const T * __restrict__ val, const T * __restrict__ b, T * __restrict__ c) {
  const uint32_t cmax = ncols - 1;
  for (uint32_t i = blockIdx.x * kSpmmBlock + threadIdx.x; i < nrows;
       i += gridDim.x * kSpmmBlock) {
    const uint32_t rb = __ldg(rowptr + i), re = __ldg(rowptr + i + 1);
    uint32_t col[STAGE];
    T w[STAGE];
#pragma unroll
    for (int s = 0; s < STAGE; ++s)
      if (rb + s < re) {
        col[s] = min(__ldg(rowind + rb + s), cmax);
        w[s] = __ldg(val + rb + s);
      }
    T * crow = c + static_cast<size_t>(i) * k;
    uint32_t j = 0;
    // two columns at a time: both columns' gathers are in flight together
    if constexpr (STAGE <= 5 && GB_SPMM_PAIRS) for (; j + 2 <= k; j += 2) {
      const T * bj = b + static_cast<size_t>(j) * ncols;
      const T * bj1 = bj + ncols;
      T x[STAGE], x1[STAGE];
#pragma unroll
      for (int s = 0; s < STAGE; ++s)
        if (rb + s < re) {
          x[s] = __ldg(bj + col[s]);
          x1[s] = __ldg(bj1 + col[s]);
        }
      T acc = T(0), acc1 = T(0);
#pragma unroll
      for (int s = 0; s < STAGE; ++s)
        if (rb + s < re) {
          acc = add_rn(acc, mul_rn(w[s], x[s]));
          acc1 = add_rn(acc1, mul_rn(w[s], x1[s]));
        }
      for (uint32_t t = rb + STAGE; t < re; ++t) {  // long-row tail
        const uint32_t ct = min(__ldg(rowind + t), cmax);
        const T wt = __ldg(val + t);
        acc = add_rn(acc, mul_rn(wt, __ldg(bj + ct)));
        acc1 = add_rn(acc1, mul_rn(wt, __ldg(bj1 + ct)));
      }
      crow[j] = acc;
      crow[j + 1] = acc1;
    }
    for (; j < k; ++j) {
      const T * bj = b + static_cast<size_t>(j) * ncols;
      T x[STAGE];
#pragma unroll
      for (int s = 0; s < STAGE; ++s)
        if (rb + s < re) x[s] = __ldg(bj + col[s]);
      T acc = T(0);
#pragma unroll
      for (int s = 0; s < STAGE; ++s)
        if (rb + s < re) acc = add_rn(acc, mul_rn(w[s], x[s]));
      for (uint32_t t = rb + STAGE; t < re; ++t)  // long-row tail
        acc = add_rn(acc, mul_rn(__ldg(val + t), __ldg(bj + min(__ldg(rowind + t), cmax))));
      crow[j] = acc;
    }
  }
}

}  // namespace

// Longest row the fused kernel takes: a thread walks its rows alone.
constexpr uint32_t kSpmmMaxRow = 256;

template <typename T>
int launch_spmm_fused(const gb_csr & a, uint32_t k, const T * vals, const T * b, T * c,
    cudaStream_t stream, bool * done) {
  *done = false;
  if (a.plan.max_row > kSpmmMaxRow || k < 2) return GOOSEBERRY_SUCCESS;
  *done = true;
  if (a.nrows == 0) return GOOSEBERRY_SUCCESS;
  int sms = 148;
  GB_TRY(sm_count_of_current_device(&sms));
  const uint32_t grid = std::max<uint32_t>(1, std::min<uint32_t>(
      (a.nrows + kSpmmBlock - 1) / kSpmmBlock, static_cast<uint32_t>(sms) * 8));
  auto kern = a.plan.max_row <= 5 ? spmm_rows_kernel<T, 5> : spmm_rows_kernel<T, kSpmmStage>;
  kern<<<grid, kSpmmBlock, 0, stream>>>(a.nrows, std::max<uint32_t>(a.ncols, 1), k, a.rowptr,
      a.rowind, vals, b, c);
  GB_CUDA_TRY(cudaGetLastError());
  return GOOSEBERRY_SUCCESS;
}

template int launch_spmm_fused<double>(const gb_csr &, uint32_t, const double *, const double *,
    double *, cudaStream_t, bool *);
template int launch_spmm_fused<float>(const gb_csr &, uint32_t, const float *, const float *,
    float *, cudaStream_t, bool *);

}  // namespace gb
