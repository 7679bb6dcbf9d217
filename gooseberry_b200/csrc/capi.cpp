// capi.cpp -- the drop-in gooseberry.h entry points (host pointers).
//
// Each call mirrors the reference's synchronous host API: inputs are copied
// to the GPU, the kernels run there and the result is copied back before the
// call returns.  Reference entry points: gooseberry_scale / _add_scalar /
// _spmult (src/gooseberry.c:35-67) and the internal cgd (src/cgd.c:40-129).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include "gb_internal.h"

namespace gb {
int launch_scale_f64(size_t n, double * v, double s, cudaStream_t st);
int launch_scale_f32(size_t n, float * v, float s, cudaStream_t st);
int launch_add_scalar_f64(size_t n, double * v, double s, cudaStream_t st);
int launch_add_scalar_f32(size_t n, float * v, float s, cudaStream_t st);
}  // namespace gb

namespace {

// One library stream per device for the synchronous drop-in calls.
cudaStream_t dropin_stream(int * rc) {
  static std::mutex mu;
  static std::vector<cudaStream_t> streams;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    gb::set_error("no CUDA device: %s", cudaGetErrorString(cudaGetLastError()));
    *rc = GOOSEBERRY_ERROR_UNKNOWN;
    return nullptr;
  }
  std::lock_guard<std::mutex> lock(mu);
  if (streams.size() <= static_cast<size_t>(dev)) streams.resize(dev + 1, nullptr);
  if (!streams[dev]) {
    cudaError_t e = cudaStreamCreateWithFlags(&streams[dev], cudaStreamNonBlocking);
    if (e != cudaSuccess) {
      gb::set_error("cudaStreamCreate failed: %s", cudaGetErrorString(e));
      *rc = GOOSEBERRY_ERROR_UNKNOWN;
      return nullptr;
    }
  }
  *rc = GOOSEBERRY_SUCCESS;
  return streams[dev];
}

// Device buffer (library pool) freed at scope exit, after the device is idle.
struct DevBuf {
  void * p = nullptr;
  ~DevBuf() {
    if (p) {
      cudaDeviceSynchronize();
      gb::dev_free(p);
    }
  }
};

template <typename T>
int vec_op(ind_t n, T * val, T s, bool add) {
  if (n == 0) return GOOSEBERRY_SUCCESS;
  GB_CHECK_INPUT(val != nullptr, "val is NULL");
  int rc = GOOSEBERRY_SUCCESS;
  cudaStream_t st = dropin_stream(&rc);
  GB_TRY(rc);
  DevBuf d;
  GB_TRY(gb::dev_alloc(&d.p, n * sizeof(T)));
  GB_CUDA_TRY(cudaMemcpyAsync(d.p, val, n * sizeof(T), cudaMemcpyHostToDevice, st));
  if (sizeof(T) == 8) {
    rc = add ? gb::launch_add_scalar_f64(n, static_cast<double *>(d.p), s, st)
             : gb::launch_scale_f64(n, static_cast<double *>(d.p), s, st);
  } else {
    rc = add ? gb::launch_add_scalar_f32(n, static_cast<float *>(d.p), static_cast<float>(s), st)
             : gb::launch_scale_f32(n, static_cast<float *>(d.p), static_cast<float>(s), st);
  }
  GB_TRY(rc);
  GB_CUDA_TRY(cudaMemcpyAsync(val, d.p, n * sizeof(T), cudaMemcpyDeviceToHost, st));
  GB_CUDA_TRY(cudaStreamSynchronize(st));
  return GOOSEBERRY_SUCCESS;
}

struct CsrGuard {
  gb_csr_t * a = nullptr;
  ~CsrGuard() {
    if (a) gb_csr_destroy(a);
  }
};

template <typename T>
int spmult_impl(dim_t anrows, dim_t ancols, dim_t bncols, const ind_t * rowptr,
    const dim_t * rowind, const T * rowval, const T * bcolval, T * crowval,
    const dim_t * blocks, dim_t nblocks) {
  if (anrows == 0 || bncols == 0) return GOOSEBERRY_SUCCESS;
  GB_CHECK_INPUT(rowptr && crowval, "NULL array");
  const uint32_t nnz = rowptr[anrows];
  GB_CHECK_INPUT(nnz == 0 || (rowind && rowval && bcolval), "NULL array");
  if (blocks) {
    for (dim_t c = 0; c < nblocks; ++c)
      GB_CHECK_INPUT(blocks[c] <= anrows && blocks[c + 1] <= anrows,
          "block %u = [%u, %u) exceeds %u rows", c, blocks[c], blocks[c + 1], anrows);
    if (nblocks == 0) return GOOSEBERRY_SUCCESS;  // no rows computed
  }
  int rc = GOOSEBERRY_SUCCESS;
  cudaStream_t st = dropin_stream(&rc);
  GB_TRY(rc);
  const bool f64 = sizeof(T) == 8;
  CsrGuard g;
  GB_TRY(gb_csr_create(anrows, ancols, nnz, rowptr, rowind,
      f64 ? reinterpret_cast<const double *>(rowval) : nullptr,
      f64 ? nullptr : reinterpret_cast<const float *>(rowval),
      f64 ? GB_CSR_VALUES_F64 : GB_CSR_VALUES_F32, st, &g.a));
  DevBuf db, dc;
  const size_t bsz = static_cast<size_t>(ancols) * bncols;
  const size_t csz = static_cast<size_t>(anrows) * bncols;
  GB_TRY(gb::dev_alloc(&db.p, std::max<size_t>(bsz, 1) * sizeof(T)));
  GB_TRY(gb::dev_alloc(&dc.p, csz * sizeof(T)));
  if (bsz) GB_CUDA_TRY(cudaMemcpyAsync(db.p, bcolval, bsz * sizeof(T), cudaMemcpyHostToDevice, st));
  bool fused = false;
  GB_TRY(gb::launch_spmm_fused<T>(*g.a, bncols,
      f64 ? reinterpret_cast<const T *>(g.a->val64) : reinterpret_cast<const T *>(g.a->val32),
      static_cast<const T *>(db.p), static_cast<T *>(dc.p), st, &fused));
  for (dim_t j = 0; j < bncols && !fused; ++j) {
    if (f64) {
      GB_TRY(gb::launch_spmv_f64(*g.a, g.a->sched64,
          static_cast<const double *>(db.p) + static_cast<size_t>(j) * ancols,
          static_cast<double *>(dc.p) + j, bncols, st));
    } else {
      GB_TRY(gb::launch_spmv_f32(*g.a, g.a->sched32,
          static_cast<const float *>(db.p) + static_cast<size_t>(j) * ancols,
          static_cast<float *>(dc.p) + j, bncols, st));
    }
  }
  if (!blocks) {
    GB_CUDA_TRY(cudaMemcpyAsync(crowval, dc.p, csz * sizeof(T), cudaMemcpyDeviceToHost, st));
  } else {
    // only the rows inside the blocks are written back (blas.c:576-595)
    for (dim_t c = 0; c < nblocks; ++c) {
      const dim_t s = blocks[c], e = blocks[c + 1];
      if (e <= s) continue;
      const size_t off = static_cast<size_t>(s) * bncols;
      const size_t cnt = static_cast<size_t>(e - s) * bncols;
      GB_CUDA_TRY(cudaMemcpyAsync(crowval + off, static_cast<T *>(dc.p) + off,
          cnt * sizeof(T), cudaMemcpyDeviceToHost, st));
    }
  }
  GB_CUDA_TRY(cudaStreamSynchronize(st));
  return GOOSEBERRY_SUCCESS;
}

int cgd_f64(dim_t n, const ind_t * rowptr, const dim_t * rowind, const double * rowval,
    const double * b, double * x, double error, size_t niter, size_t * iterations,
    double * rnorm, double * history, size_t history_len) {
  GB_CHECK_INPUT(rowptr && b && x, "NULL array");
  GB_CHECK_INPUT(n > 0, "CG needs a non-empty matrix");
  const uint32_t nnz = rowptr[n];
  GB_CHECK_INPUT(nnz == 0 || (rowind && rowval), "NULL array");
  int rc = GOOSEBERRY_SUCCESS;
  cudaStream_t st = dropin_stream(&rc);
  GB_TRY(rc);
  CsrGuard g;
  GB_TRY(gb_csr_create(n, n, nnz, rowptr, rowind, rowval, nullptr, GB_CSR_VALUES_F64, st,
      &g.a));
  gb_cg_t * s = nullptr;
  GB_TRY(gb_cg_create(g.a, GB_CG_F64, &s));
  DevBuf db, dx;
  rc = GOOSEBERRY_SUCCESS;
  gb_cg_result_t res{};
  rc = gb::dev_alloc(&db.p, n * sizeof(double));
  if (rc == GOOSEBERRY_SUCCESS) rc = gb::dev_alloc(&dx.p, n * sizeof(double));
  if (rc == GOOSEBERRY_SUCCESS &&
      cudaMemcpyAsync(db.p, b, n * sizeof(double), cudaMemcpyHostToDevice, st) != cudaSuccess) {
    gb::set_error("CG buffers: %s", cudaGetErrorString(cudaGetLastError()));
    rc = GOOSEBERRY_ERROR_UNKNOWN;
  }
  if (rc == GOOSEBERRY_SUCCESS)
    rc = gb_cg_solve(s, static_cast<const double *>(db.p), static_cast<double *>(dx.p), error,
        0, niter, history, history_len, &res, st);
  if (rc == GOOSEBERRY_SUCCESS) {
    cudaError_t e = cudaMemcpyAsync(x, dx.p, n * sizeof(double), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
      gb::set_error("CG download: %s", cudaGetErrorString(e));
      rc = GOOSEBERRY_ERROR_UNKNOWN;
    }
  }
  gb_cg_destroy(s);
  GB_TRY(rc);
  if (iterations) *iterations = res.iterations;
  if (rnorm) *rnorm = res.rnorm;
  return GOOSEBERRY_SUCCESS;
}

}  // namespace

extern "C" {

int gooseberry_scale(ind_t n, float * val, float s) { return vec_op<float>(n, val, s, false); }
int gooseberry_scale_f64(ind_t n, double * val, double s) {
  return vec_op<double>(n, val, s, false);
}
int gooseberry_add_scalar(ind_t n, float * val, float s) { return vec_op<float>(n, val, s, true); }
int gooseberry_add_scalar_f64(ind_t n, double * val, double s) {
  return vec_op<double>(n, val, s, true);
}

int gooseberry_spmult(dim_t anrows, dim_t ancols, dim_t bncols, const ind_t * arowptr,
    const dim_t * arowind, const float * arowval, const float * bcolval, float * crowval,
    const dim_t * blocks, dim_t nblocks) {
  return spmult_impl<float>(anrows, ancols, bncols, arowptr, arowind, arowval, bcolval,
      crowval, blocks, nblocks);
}

int gooseberry_spmult_f64(dim_t anrows, dim_t ancols, dim_t bncols, const ind_t * arowptr,
    const dim_t * arowind, const double * arowval, const double * bcolval, double * crowval,
    const dim_t * blocks, dim_t nblocks) {
  return spmult_impl<double>(anrows, ancols, bncols, arowptr, arowind, arowval, bcolval,
      crowval, blocks, nblocks);
}

int gooseberry_cgd_f64(dim_t n, const ind_t * rowptr, const dim_t * rowind,
    const double * rowval, const double * b, double * x, double error, size_t niter,
    size_t * iterations, double * rnorm, double * history, size_t history_len) {
  return cgd_f64(n, rowptr, rowind, rowval, b, x, error, niter, iterations, rnorm, history,
      history_len);
}

// Float ABI: the solve runs in double on the device (never less accurate than
// the reference's float build) and x is rounded back to float.
int gooseberry_cgd(dim_t n, const ind_t * rowptr, const dim_t * rowind, const float * rowval,
    const float * b, float * x, float error, size_t niter, size_t * iterations,
    double * rnorm, double * history, size_t history_len) {
  GB_CHECK_INPUT(rowptr && b && x, "NULL array");
  GB_CHECK_INPUT(n > 0, "CG needs a non-empty matrix");
  const uint32_t nnz = rowptr[n];
  GB_CHECK_INPUT(nnz == 0 || (rowind && rowval), "NULL array");
  std::vector<double> v(rowval, rowval + nnz), bb(b, b + n), xx(n);
  GB_TRY(cgd_f64(n, rowptr, rowind, v.data(), bb.data(), xx.data(), error, niter, iterations,
      rnorm, history, history_len));
  for (dim_t i = 0; i < n; ++i) x[i] = static_cast<float>(xx[i]);
  return GOOSEBERRY_SUCCESS;
}

}  // extern "C"
