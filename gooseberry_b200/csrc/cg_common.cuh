// cg_common.cuh -- launch and reduction helpers shared by the CG solvers
// (cg.cu: plain FP64; cg_mixed.cu: FP32 inner iterations with FP64
// residual refinement).
#pragma once

#include <cuda_runtime.h>

#include "gb_internal.h"
#include "spmv_tiles.cuh"

namespace gb {
namespace {

constexpr int kVecBlock = 256;

// Programmatic dependent launch: a kernel lets the next one in the stream be
// scheduled as soon as its own CTAs start retiring, and waits for the
// previous kernel's completion (and memory) before touching any data.
__device__ __forceinline__ void pdl_wait_and_release() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

template <typename... KArgs, typename... Args>
cudaError_t launch_k(void (*k)(KArgs...), unsigned grid, unsigned block, size_t smem,
    cudaStream_t s, bool pdl, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(block);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = pdl ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, k, static_cast<KArgs>(args)...);
}

// Returns true in thread 0 of the last CTA to arrive (ticket pattern).
__device__ __forceinline__ bool arrive_last(unsigned int * ticket, bool * flag) {
  __syncthreads();  // every thread's writes of this CTA precede thread 0's fence
  if (threadIdx.x == 0) {
    __threadfence();
    const unsigned prev = atomicAdd(ticket, 1u);
    *flag = (prev == gridDim.x - 1);
  }
  __syncthreads();
  return *flag;
}

// Sum of partial[0..n) in a fixed order (for a given n and CTA size), by one
// CTA; result valid in thread 0.  Thread t adds entries t, t + blockDim.x,
// ... (all loads of a batch issued before the adds), then the warp tree and
// the per-warp sums in warp order.
__device__ __forceinline__ double ordered_sum(const double * partial, unsigned n,
    double * red) {
  constexpr int U = 8;
  double acc = 0.0;
  for (unsigned base = 0; base < n; base += U * blockDim.x) {
    double v[U];
#pragma unroll
    for (int j = 0; j < U; ++j) {
      const unsigned i = base + j * blockDim.x + threadIdx.x;
      v[j] = i < n ? __ldcg(partial + i) : 0.0;
    }
#pragma unroll
    for (int j = 0; j < U; ++j) acc += v[j];
  }
  return block_sum(acc, red);
}

// ordered_sum with `side()` called by every thread right after its first
// batch of partial loads is issued: loads made there are in flight together
// with the partials (one round trip instead of two).  Same sum, same order.
template <class F>
__device__ __forceinline__ double ordered_sum_with(const double * partial, unsigned n,
    double * red, F && side) {
  constexpr int U = 8;
  double acc = 0.0;
  bool called = false;
  for (unsigned base = 0; base < n; base += U * blockDim.x) {
    double v[U];
#pragma unroll
    for (int j = 0; j < U; ++j) {
      const unsigned i = base + j * blockDim.x + threadIdx.x;
      v[j] = i < n ? __ldcg(partial + i) : 0.0;
    }
    if (!called) {
      side();
      called = true;
    }
#pragma unroll
    for (int j = 0; j < U; ++j) acc += v[j];
  }
  if (!called) side();
  return block_sum(acc, red);
}

}  // namespace
}  // namespace gb
