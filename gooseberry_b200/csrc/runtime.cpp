// runtime.cpp -- error state, device queries and the stream-ordered scratch
// pool of libgooseberry_b200.
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <map>
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
struct DevicePool {
  cudaMemPool_t pool = nullptr;
  cudaStream_t alloc_stream = nullptr;  // orders the pool's own allocations and frees
};
std::mutex g_pool_mu;
std::vector<DevicePool> g_pools;  // per device, created on first use
// Memory the pool keeps for reuse after frees; beyond this it returns memory
// to the device at synchronisation points.
constexpr uint64_t kPoolKeepBytes = 4ull << 30;

int pool_of_current_device(DevicePool * out) {
  int dev = 0;
  GB_CUDA_TRY(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lock(g_pool_mu);
  if (g_pools.size() <= static_cast<size_t>(dev)) g_pools.resize(dev + 1);
  DevicePool & d = g_pools[dev];
  if (!d.pool) {
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.handleTypes = cudaMemHandleTypeNone;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t np = nullptr;
    GB_CUDA_TRY(cudaMemPoolCreate(&np, &props));
    uint64_t keep = kPoolKeepBytes;
    GB_CUDA_TRY(cudaMemPoolSetAttribute(np, cudaMemPoolAttrReleaseThreshold, &keep));
    GB_CUDA_TRY(cudaStreamCreateWithFlags(&d.alloc_stream, cudaStreamNonBlocking));
    d.pool = np;
  }
  *out = d;
  return GOOSEBERRY_SUCCESS;
}
}  // namespace

// Device memory of the library's objects and per-call scratch comes from a
// memory pool the library owns: after the first use an allocation costs no
// driver mapping and a free no device-wide synchronisation, and the device's
// default pool and its settings stay untouched.
int scratch_alloc(void ** p, size_t bytes, cudaStream_t s) {
  DevicePool d;
  GB_TRY(pool_of_current_device(&d));
  GB_CUDA_TRY(cudaMallocFromPoolAsync(p, bytes, d.pool, s));
  return GOOSEBERRY_SUCCESS;
}

void scratch_free(void * p, cudaStream_t s) {
  if (p) cudaFreeAsync(p, s);
}

int dev_alloc(void ** p, size_t bytes) {
  DevicePool d;
  GB_TRY(pool_of_current_device(&d));
  GB_CUDA_TRY(cudaMallocFromPoolAsync(p, bytes ? bytes : 1, d.pool, d.alloc_stream));
  GB_CUDA_TRY(cudaStreamSynchronize(d.alloc_stream));  // usable from any stream now
  return GOOSEBERRY_SUCCESS;
}

void dev_free(void * p) {
  if (!p) return;
  DevicePool d;
  if (pool_of_current_device(&d) != GOOSEBERRY_SUCCESS) return;
  cudaFreeAsync(p, d.alloc_stream);
}

namespace {
std::mutex g_smem_mu;
std::map<std::pair<const void *, int>, size_t> g_smem_limit;
}  // namespace

int raise_smem_limit(const void * func, size_t bytes) {
  if (bytes <= 48 * 1024) return GOOSEBERRY_SUCCESS;
  int dev = 0;
  GB_CUDA_TRY(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lock(g_smem_mu);
  size_t & lim = g_smem_limit[std::make_pair(func, dev)];
  if (bytes > lim) {
    GB_CUDA_TRY(cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize,
        static_cast<int>(bytes)));
    lim = bytes;
  }
  return GOOSEBERRY_SUCCESS;
}

namespace {
// Small pinned, device-mapped host slots, carved from blocks that are kept for
// the life of the process: a mapped host allocation costs milliseconds (and
// its free a device-wide synchronisation), far more than the solve-setup work
// it serves.
constexpr size_t kSlotBytes = 128;
constexpr size_t kSlotBlockBytes = 64 * 1024;
std::mutex g_slot_mu;
std::vector<void *> g_slot_free;
}  // namespace

int pinned_slot_alloc(size_t bytes, void ** host, void ** dev) {
  *host = nullptr;
  if (dev) *dev = nullptr;
  GB_CHECK_INPUT(bytes <= kSlotBytes, "pinned slot of %zu bytes (at most %zu)", bytes,
      kSlotBytes);
  void * h = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_slot_mu);
    if (g_slot_free.empty()) {
      void * block = nullptr;
      GB_CUDA_TRY(cudaHostAlloc(&block, kSlotBlockBytes,
          cudaHostAllocMapped | cudaHostAllocPortable));
      for (size_t o = kSlotBlockBytes; o >= kSlotBytes; o -= kSlotBytes)
        g_slot_free.push_back(static_cast<char *>(block) + o - kSlotBytes);
    }
    h = g_slot_free.back();
    g_slot_free.pop_back();
  }
  std::memset(h, 0, kSlotBytes);
  if (dev) {
    const cudaError_t e = cudaHostGetDevicePointer(dev, h, 0);
    if (e != cudaSuccess) {
      pinned_slot_free(h);
      set_error("cudaHostGetDevicePointer failed: %s", cudaGetErrorString(e));
      return GOOSEBERRY_ERROR_UNKNOWN;
    }
  }
  *host = h;
  return GOOSEBERRY_SUCCESS;
}

void pinned_slot_free(void * host) {
  if (!host) return;
  std::lock_guard<std::mutex> lock(g_slot_mu);
  g_slot_free.push_back(host);
}

}  // namespace gb

extern "C" const char * gb_last_error(void) { return gb::g_last_error.c_str(); }
