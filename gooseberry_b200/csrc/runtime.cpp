// runtime.cpp -- error state, device queries and the stream-ordered scratch
// pool of libgooseberry_b200.
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <mutex>
#include <string>
#include <vector>

#include "gb_internal.h"

namespace gb {

namespace {
thread_local std::string g_last_error;
}

void set_error(const char * fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  std::vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
}

void clear_error() { g_last_error.clear(); }

int sm_count_of_current_device(int * out) {
  int dev = 0;
  GB_CUDA_TRY(cudaGetDevice(&dev));
  GB_CUDA_TRY(cudaDeviceGetAttribute(out, cudaDevAttrMultiProcessorCount, dev));
  return GOOSEBERRY_SUCCESS;
}

// Whether `bytes` of working set fit in the current device's L2.
int l2_fits(size_t bytes, bool * out) {
  int dev = 0, l2 = 0;
  GB_CUDA_TRY(cudaGetDevice(&dev));
  GB_CUDA_TRY(cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, dev));
  *out = bytes <= static_cast<size_t>(l2);
  return GOOSEBERRY_SUCCESS;
}

namespace {
std::mutex g_pool_mu;
std::vector<cudaMemPool_t> g_pools;  // per device, created on first use
}  // namespace

// Small per-call scratch (reduction partials, histories) comes from a memory
// pool the library owns: it keeps its memory between calls (release threshold
// = all), so a stream-ordered allocation costs no driver mapping after the
// first one, and the device's default pool and its settings stay untouched.
int scratch_alloc(void ** p, size_t bytes, cudaStream_t s) {
  int dev = 0;
  GB_CUDA_TRY(cudaGetDevice(&dev));
  cudaMemPool_t pool = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_pool_mu);
    if (g_pools.size() <= static_cast<size_t>(dev)) g_pools.resize(dev + 1, nullptr);
    if (!g_pools[dev]) {
      cudaMemPoolProps props = {};
      props.allocType = cudaMemAllocationTypePinned;
      props.handleTypes = cudaMemHandleTypeNone;
      props.location.type = cudaMemLocationTypeDevice;
      props.location.id = dev;
      cudaMemPool_t np = nullptr;
      GB_CUDA_TRY(cudaMemPoolCreate(&np, &props));
      uint64_t keep = UINT64_MAX;
      GB_CUDA_TRY(cudaMemPoolSetAttribute(np, cudaMemPoolAttrReleaseThreshold, &keep));
      g_pools[dev] = np;
    }
    pool = g_pools[dev];
  }
  GB_CUDA_TRY(cudaMallocFromPoolAsync(p, bytes, pool, s));
  return GOOSEBERRY_SUCCESS;
}

void scratch_free(void * p, cudaStream_t s) {
  if (p) cudaFreeAsync(p, s);
}

}  // namespace gb

extern "C" const char * gb_last_error(void) { return gb::g_last_error.c_str(); }
