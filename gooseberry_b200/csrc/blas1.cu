// blas1.cu -- BLAS-1 on device vectors: dot, sparse . dense dot, scale,
// add_scalar, add, sub (reference src/blas.c:244-336, 397-451).
//
// All are HBM-streaming grid-stride kernels with grids a multiple of the SM
// count.  The CG solver does not call them: it fuses the same vector work into
// its own kernels (cg.cu).  The dot product reduces per-CTA partials in a fixed
// order, so it is bitwise reproducible for a given n on a given GPU (the
// reference's OpenMP reduction order varies with the thread count,
// src/blas.c:423-427).
#include <algorithm>
#include <map>
#include <mutex>
#include <vector>

#include "gb_internal.h"
#include "spmv_tiles.cuh"

namespace gb {

namespace {

constexpr int kBlock = 256;

// [begin, end) of CTA `b` out of `g` over n elements, split in 2-element units
__device__ __forceinline__ void chunk_of(size_t n, unsigned b, unsigned g, size_t & s,
    size_t & e) {
  const size_t units = (n + 1) / 2;
  const size_t q = units / g, r = units % g;
  const size_t us = b * q + min(static_cast<size_t>(b), r);
  const size_t ue = us + q + (b < r ? 1 : 0);
  s = min(us * 2, n);
  e = min(ue * 2, n);
}

template <typename T>
__global__ void __launch_bounds__(kBlock) dot_partial_kernel(size_t n,
    const T * __restrict__ a, const T * __restrict__ b, double * __restrict__ partial) {
  __shared__ double red[32];
  size_t s, e;
  chunk_of(n, blockIdx.x, gridDim.x, s, e);
  double acc = 0.0;
  for (size_t i = s + threadIdx.x; i < e; i += kBlock)
    acc += static_cast<double>(a[i]) * static_cast<double>(b[i]);
  acc = block_sum(acc, red);
  if (threadIdx.x == 0) partial[blockIdx.x] = acc;
}

__global__ void __launch_bounds__(kBlock) dot_final_kernel(unsigned g,
    const double * __restrict__ partial, double * __restrict__ out) {
  __shared__ double red[32];
  double acc = 0.0;
  for (unsigned i = threadIdx.x; i < g; i += kBlock) acc += partial[i];
  acc = block_sum(acc, red);
  if (threadIdx.x == 0) *out = acc;
}

// Sparse . dense: each CTA owns a fixed contiguous chunk of the nonzeros;
// its threads stream indices and values (evict-first) and keep kSpdotK
// gathers of x in flight each, accumulating in double.  This is the streaming
// and gather work of a CSR SpMV without its row reductions, so its time on a
// matrix's own (rowind, rowval, x) is a floor for that SpMV on this GPU.
constexpr int kSpdotK = 8;

template <typename T>
__global__ void __launch_bounds__(kBlock) spdot_partial_kernel(size_t nnz,
    const uint32_t * __restrict__ ind, const T * __restrict__ val, const T * __restrict__ x,
    size_t nx, double * __restrict__ partial) {
  __shared__ double red[32];
  size_t s, e;
  chunk_of(nnz, blockIdx.x, gridDim.x, s, e);
  const NoHint pol_m, pol_x;  // plain loads: faster than L2-policy loads on this pattern
  const uint32_t cmax = static_cast<uint32_t>(nx - 1);
  double acc = 0.0;
  for (size_t base = s + threadIdx.x; base < e; base += static_cast<size_t>(kSpdotK) * kBlock) {
    uint32_t c[kSpdotK];
    T v[kSpdotK];
#pragma unroll
    for (int j = 0; j < kSpdotK; ++j) {
      const size_t i = base + static_cast<size_t>(j) * kBlock;
      if (i < e) {
        c[j] = ld_stream(ind + i, pol_m);
        v[j] = ld_stream(val + i, pol_m);
      }
    }
    T xv[kSpdotK];
#pragma unroll
    for (int j = 0; j < kSpdotK; ++j) {
      const size_t i = base + static_cast<size_t>(j) * kBlock;
      if (i < e) xv[j] = ld_keep(x + min(c[j], cmax), pol_x);
    }
#pragma unroll
    for (int j = 0; j < kSpdotK; ++j) {
      const size_t i = base + static_cast<size_t>(j) * kBlock;
      if (i < e) acc += static_cast<double>(v[j]) * static_cast<double>(xv[j]);
    }
  }
  acc = block_sum(acc, red);
  if (threadIdx.x == 0) partial[blockIdx.x] = acc;
}

template <typename T>
__global__ void __launch_bounds__(kBlock) scale_kernel(size_t n, T * __restrict__ v, T s) {
  for (size_t i = blockIdx.x * static_cast<size_t>(kBlock) + threadIdx.x; i < n;
       i += static_cast<size_t>(gridDim.x) * kBlock)
    v[i] *= s;
}

template <typename T>
__global__ void __launch_bounds__(kBlock) add_scalar_kernel(size_t n, T * __restrict__ v, T s) {
  for (size_t i = blockIdx.x * static_cast<size_t>(kBlock) + threadIdx.x; i < n;
       i += static_cast<size_t>(gridDim.x) * kBlock)
    v[i] += s;
}

// c = a + sign*b; c may alias a or b (each element read before written)
template <typename T>
__global__ void __launch_bounds__(kBlock) axpby_kernel(size_t n, const T * a, const T * b,
    T * c, int subtract) {
  for (size_t i = blockIdx.x * static_cast<size_t>(kBlock) + threadIdx.x; i < n;
       i += static_cast<size_t>(gridDim.x) * kBlock) {
    const T av = a[i], bv = b[i];
    c[i] = subtract ? av - bv : av + bv;
  }
}

unsigned grid_for(size_t n, int per_sm) {
  int sms = 148;
  sm_count_of_current_device(&sms);
  const size_t want = (n + kBlock * 4 - 1) / (kBlock * 4);
  return static_cast<unsigned>(std::max<size_t>(1, std::min<size_t>(want,
      static_cast<size_t>(sms) * per_sm)));
}

template <typename T>
int dot_impl(size_t n, const T * a, const T * b, double * result, cudaStream_t s) {
  GB_CHECK_INPUT(result != nullptr, "result is NULL");
  GB_CHECK_INPUT(n == 0 || (a && b), "NULL vector");
  const unsigned g = grid_for(n, 4);
  double * partial = nullptr;
  GB_TRY(scratch_alloc(reinterpret_cast<void **>(&partial), g * sizeof(double), s));
  dot_partial_kernel<T><<<g, kBlock, 0, s>>>(n, a, b, partial);
  dot_final_kernel<<<1, kBlock, 0, s>>>(g, partial, result);
  cudaError_t e = cudaGetLastError();
  scratch_free(partial, s);
  GB_CUDA_TRY(e);
  return GOOSEBERRY_SUCCESS;
}

template <typename T>
int spdot_impl(size_t nnz, const uint32_t * ind, const T * val, const T * x, size_t nx,
    double * result, cudaStream_t s) {
  GB_CHECK_INPUT(result != nullptr, "result is NULL");
  GB_CHECK_INPUT(nnz == 0 || (ind && val && x && nx > 0), "NULL vector or empty x");
  const unsigned g = grid_for(nnz, 4);
  double * partial = nullptr;
  GB_TRY(scratch_alloc(reinterpret_cast<void **>(&partial), g * sizeof(double), s));
  spdot_partial_kernel<T><<<g, kBlock, 0, s>>>(nnz, ind, val, x, nx, partial);
  dot_final_kernel<<<1, kBlock, 0, s>>>(g, partial, result);
  cudaError_t e = cudaGetLastError();
  scratch_free(partial, s);
  GB_CUDA_TRY(e);
  return GOOSEBERRY_SUCCESS;
}

}  // namespace

int launch_scale_f64(size_t n, double * v, double s, cudaStream_t st) {
  if (n == 0) return GOOSEBERRY_SUCCESS;
  scale_kernel<double><<<grid_for(n, 8), kBlock, 0, st>>>(n, v, s);
  GB_CUDA_TRY(cudaGetLastError());
  return GOOSEBERRY_SUCCESS;
}
int launch_scale_f32(size_t n, float * v, float s, cudaStream_t st) {
  if (n == 0) return GOOSEBERRY_SUCCESS;
  scale_kernel<float><<<grid_for(n, 8), kBlock, 0, st>>>(n, v, s);
  GB_CUDA_TRY(cudaGetLastError());
  return GOOSEBERRY_SUCCESS;
}
int launch_add_scalar_f64(size_t n, double * v, double s, cudaStream_t st) {
  if (n == 0) return GOOSEBERRY_SUCCESS;
  add_scalar_kernel<double><<<grid_for(n, 8), kBlock, 0, st>>>(n, v, s);
  GB_CUDA_TRY(cudaGetLastError());
  return GOOSEBERRY_SUCCESS;
}
int launch_add_scalar_f32(size_t n, float * v, float s, cudaStream_t st) {
  if (n == 0) return GOOSEBERRY_SUCCESS;
  add_scalar_kernel<float><<<grid_for(n, 8), kBlock, 0, st>>>(n, v, s);
  GB_CUDA_TRY(cudaGetLastError());
  return GOOSEBERRY_SUCCESS;
}

// ---- allocation-free dot product --------------------------------------------
//
// Same two-kernel reduction as dot_impl, but each CTA owns a fixed chunk of
// kNoAllocChunk elements and writes its partial sum into a file-scope device
// array instead of memory obtained from the allocator.  Host code must not
// pass `g_dot_scratch` itself to a kernel: in host code that name is only a
// host-side stand-in for the symbol, so the device address is looked up with
// cudaGetSymbolAddress once per device and cached.

namespace {

constexpr size_t kNoAllocChunk = 16384;       // elements per CTA
constexpr unsigned kNoAllocMaxChunks = 8192;  // partial sums the array holds
static_assert(GB_DOT_NOALLOC_MAX_N == kNoAllocChunk * kNoAllocMaxChunks,
    "header limit and array size disagree");

static __device__ __align__(256) double g_dot_scratch[kNoAllocMaxChunks];

std::mutex g_dot_scratch_mu;
// Device address of the array per CUDA context, keyed by the context's unique
// id: a cudaDeviceReset (or any teardown of a primary context) reloads the
// module in a new context with a new id, so a stale address is never reused.
std::map<unsigned long long, double *> g_dot_scratch_ptr;

__global__ void __launch_bounds__(kBlock) dot_chunk_kernel(size_t n,
    const double * __restrict__ a, const double * __restrict__ b,
    double * __restrict__ partial) {
  __shared__ double red[32];
  const size_t s = static_cast<size_t>(blockIdx.x) * kNoAllocChunk;
  const size_t e = min(n, s + kNoAllocChunk);
  double acc = 0.0;
  for (size_t i = s + threadIdx.x; i < e; i += kBlock) acc += a[i] * b[i];
  acc = block_sum(acc, red);
  if (threadIdx.x == 0) partial[blockIdx.x] = acc;
}

// Unique id of the calling thread's current CUDA context (driver entry
// points cuCtxGetCurrent / cuCtxGetId, resolved once through the runtime so
// the library needs no link to the driver library).  False when unavailable.
bool current_context_id(unsigned long long * id) {
  using GetCurrent = int (*)(void **);
  using GetId = int (*)(void *, unsigned long long *);
  static GetCurrent get_current = nullptr;
  static GetId get_id = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void * f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f, 12000, cudaEnableDefault, &q) ==
            cudaSuccess && q == cudaDriverEntryPointSuccess)
      get_current = reinterpret_cast<GetCurrent>(f);
    if (cudaGetDriverEntryPointByVersion("cuCtxGetId", &f, 12000, cudaEnableDefault, &q) ==
            cudaSuccess && q == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<GetId>(f);
  });
  void * ctx = nullptr;
  return get_current && get_id && get_current(&ctx) == 0 && ctx && get_id(ctx, id) == 0;
}

// Device address of g_dot_scratch in the current context: looked up once per
// context (the first call on a device, with that device current), or on
// every call if the context id cannot be read.
int dot_scratch_address(double ** out) {
  int dev = 0;
  GB_CUDA_TRY(cudaGetDevice(&dev));
  unsigned long long ctx = 0;
  bool keyed = current_context_id(&ctx);
  if (!keyed) {  // no context bound to this thread yet: bind the primary one
    GB_CUDA_TRY(cudaFree(nullptr));
    keyed = current_context_id(&ctx);
  }
  std::lock_guard<std::mutex> lock(g_dot_scratch_mu);
  if (keyed) {
    auto it = g_dot_scratch_ptr.find(ctx);
    if (it != g_dot_scratch_ptr.end()) {
      *out = it->second;
      return GOOSEBERRY_SUCCESS;
    }
  }
  void * p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_dot_scratch);
  if (e != cudaSuccess || p == nullptr) {
    set_error("cudaGetSymbolAddress of the dot scratch array failed on device %d: %s", dev,
        cudaGetErrorString(e));
    return GOOSEBERRY_ERROR_UNKNOWN;
  }
  if (keyed) g_dot_scratch_ptr[ctx] = static_cast<double *>(p);
  *out = static_cast<double *>(p);
  return GOOSEBERRY_SUCCESS;
}

}  // namespace

}  // namespace gb

extern "C" {

int gb_dot_f64_noalloc(size_t n, const double * a, const double * b, double * result,
    gb_stream_t stream) {
  GB_CHECK_INPUT(result != nullptr, "result is NULL");
  GB_CHECK_INPUT(n == 0 || (a && b), "NULL vector");
  GB_CHECK_INPUT(n <= GB_DOT_NOALLOC_MAX_N,
      "n = %zu exceeds the %zu elements the allocation-free dot product can reduce "
      "(its fixed scratch holds %u partial sums of %zu elements each)",
      n, static_cast<size_t>(GB_DOT_NOALLOC_MAX_N), gb::kNoAllocMaxChunks,
      gb::kNoAllocChunk);
  double * scratch = nullptr;
  GB_TRY(gb::dot_scratch_address(&scratch));
  const unsigned chunks = static_cast<unsigned>(
      std::max<size_t>(1, (n + gb::kNoAllocChunk - 1) / gb::kNoAllocChunk));
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  gb::dot_chunk_kernel<<<chunks, gb::kBlock, 0, s>>>(n, a, b, scratch);
  gb::dot_final_kernel<<<1, gb::kBlock, 0, s>>>(chunks, scratch, result);
  GB_CUDA_TRY(cudaGetLastError());
  return GOOSEBERRY_SUCCESS;
}

int gb_dot_f64(size_t n, const double * a, const double * b, double * result,
    gb_stream_t stream) {
  return gb::dot_impl<double>(n, a, b, result, static_cast<cudaStream_t>(stream));
}

int gb_dot_f32(size_t n, const float * a, const float * b, double * result,
    gb_stream_t stream) {
  return gb::dot_impl<float>(n, a, b, result, static_cast<cudaStream_t>(stream));
}

int gb_spdot_f64(size_t nnz, const dim_t * ind, const double * val, const double * x,
    size_t nx, double * result, gb_stream_t stream) {
  return gb::spdot_impl<double>(nnz, ind, val, x, nx, result,
      static_cast<cudaStream_t>(stream));
}

int gb_spdot_f32(size_t nnz, const dim_t * ind, const float * val, const float * x,
    size_t nx, double * result, gb_stream_t stream) {
  return gb::spdot_impl<float>(nnz, ind, val, x, nx, result, static_cast<cudaStream_t>(stream));
}

int gb_scale_f64(size_t n, double * v, double s, gb_stream_t stream) {
  GB_CHECK_INPUT(n == 0 || v, "NULL vector");
  return gb::launch_scale_f64(n, v, s, static_cast<cudaStream_t>(stream));
}

int gb_scale_f32(size_t n, float * v, float s, gb_stream_t stream) {
  GB_CHECK_INPUT(n == 0 || v, "NULL vector");
  return gb::launch_scale_f32(n, v, s, static_cast<cudaStream_t>(stream));
}

int gb_add_scalar_f64(size_t n, double * v, double s, gb_stream_t stream) {
  GB_CHECK_INPUT(n == 0 || v, "NULL vector");
  return gb::launch_add_scalar_f64(n, v, s, static_cast<cudaStream_t>(stream));
}

int gb_add_scalar_f32(size_t n, float * v, float s, gb_stream_t stream) {
  GB_CHECK_INPUT(n == 0 || v, "NULL vector");
  return gb::launch_add_scalar_f32(n, v, s, static_cast<cudaStream_t>(stream));
}

int gb_add_f64(size_t n, const double * a, const double * b, double * c,
    gb_stream_t stream) {
  GB_CHECK_INPUT(n == 0 || (a && b && c), "NULL vector");
  if (n == 0) return GOOSEBERRY_SUCCESS;
  gb::axpby_kernel<double><<<gb::grid_for(n, 8), gb::kBlock, 0,
      static_cast<cudaStream_t>(stream)>>>(n, a, b, c, 0);
  GB_CUDA_TRY(cudaGetLastError());
  return GOOSEBERRY_SUCCESS;
}

int gb_sub_f64(size_t n, const double * a, const double * b, double * c,
    gb_stream_t stream) {
  GB_CHECK_INPUT(n == 0 || (a && b && c), "NULL vector");
  if (n == 0) return GOOSEBERRY_SUCCESS;
  gb::axpby_kernel<double><<<gb::grid_for(n, 8), gb::kBlock, 0,
      static_cast<cudaStream_t>(stream)>>>(n, a, b, c, 1);
  GB_CUDA_TRY(cudaGetLastError());
  return GOOSEBERRY_SUCCESS;
}

}  // extern "C"
