// permute.cu -- bandwidth-reducing (Cuthill-McKee) order and sparse
// permutation of a CSR matrix on the device.
//
// Reference: src/permute.c:45-104 (__cuthillmckee_block), :288-337
// (permute_cuthillmckee), :120-205 (permute_sparse); callers
// src/gooseberry_bin.c:986-993 (`permute -p bandwidth`) and :1655-1676
// (`blas -b`, per row block).
//
// Cuthill-McKee, as the reference runs it per diagonal block [start, end):
// the in-block degree of a vertex counts its row's columns inside the block;
// each component starts at the remaining vertex of least degree; breadth-first
// from it, every ordered vertex appends its remaining in-block neighbours in
// ascending degree.  Equal degrees are taken smaller vertex id first (the
// reference's queue is domlib's dlpq, which is not vendored; its tie order is
// not known).
//
// Level-synchronous form used here.  A vertex of level L+1 is appended by the
// first vertex of level L (in order) that has it as a neighbour, so level
// L+1 is the set of unvisited neighbours of level L ordered by (position of
// that first parent, degree, id).  Each level is one pass over the frontier's
// rows: an atomicMin of the parent's position into claim[k] leaves every new
// vertex with its first parent, the first claimant appends it to a candidate
// list, and a sort of (parent offset, rank) keys -- rank being the vertex's
// place in the global (degree, id) order -- puts the level in order.  Vertices
// ordered earlier hold claims below the frontier's first position, so a later
// atomicMin never changes them.  The next component's start is the first
// unvisited entry of the (degree, id) order, found by a scan that only moves
// forward.
//
// Small levels (the long thin BFS of a mesh) run inside one persistent CTA,
// which loops over levels and components with the frontier, its row offsets
// and the level's keys in shared memory and sorts the keys there.  A level
// whose frontier or candidate list outgrows that CTA is handed to device-wide
// kernels (edge-balanced expansion, radix sort), after which the CTA resumes.
//
// With row blocks, edges leaving a block are ignored; components then never
// cross blocks, so ordering all blocks in one run and stably partitioning the
// result by block gives every block the order it gets on its own.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <cstddef>
#include <cstring>
#include <vector>

#include "gb_internal.h"

namespace gb {
namespace {

constexpr uint32_t kUnvisited = 0xffffffffu;
constexpr int kCmThreads = 1024;
constexpr uint32_t kCmSmallFrontier = 4096;  // frontier vertices the CTA expands
constexpr uint32_t kCmSmallEdges = 32768;    // frontier entries the CTA expands
constexpr uint32_t kCmSmallLevel = 4096;     // candidates the CTA sorts
constexpr int kCmUnroll = 4;                 // frontier entries in flight per thread
constexpr int kCmExpandThreads = 256;
constexpr uint32_t kCmLaneEdges = 8;         // entries per lane per warp chunk

enum : uint32_t { kCmDone = 0, kCmExpand = 1, kCmSort = 2 };

struct CmState {
  uint32_t a, b;   // current level: perm[a, b)
  uint32_t next;   // scan position in order[] for the next component start
  uint32_t count;  // candidates of the last expansion, in cand[0, count)
  uint32_t mode;   // kCmDone / kCmExpand / kCmSort
  uint32_t pad[3];
};

struct CmGraph {
  const uint32_t * rowptr;
  const uint32_t * rowind;
  const uint32_t * bidx;    // block of each vertex; null: one block [0, n)
  const uint32_t * blocks;  // nblocks+1 boundaries (device)
  uint32_t n;
};

struct CmSmem {
  uint32_t off[kCmSmallFrontier + 1];  // frontier row offsets (exclusive scan)
  uint32_t rs[kCmSmallFrontier];       // row start of each frontier vertex
  uint32_t lo[kCmSmallFrontier];       // block range of each frontier vertex
  uint32_t hi[kCmSmallFrontier];
  unsigned long long key[kCmSmallLevel];
  uint32_t warp_sum[kCmThreads / 32];
  uint32_t count, found, maxb;
};

// Children one parent may have for the bucket ordering of a small level
// (larger families take the bitonic sort).
constexpr uint32_t kCmBucketMax = 32;
constexpr int kCmHeld = kCmSmallLevel / kCmThreads;  // candidates per thread

__device__ __forceinline__ void cm_block_range(const CmGraph & g, uint32_t v, uint32_t & lo,
    uint32_t & hi) {
  if (g.bidx) {
    const uint32_t b = __ldg(g.bidx + v);
    lo = __ldg(g.blocks + b);
    hi = __ldg(g.blocks + b + 1);
  } else {
    lo = 0;
    hi = g.n;
  }
}

// Block of each vertex (blocks cover [0, n) in order).
__global__ void cm_bidx_kernel(const uint32_t * blocks, uint32_t nblocks, uint32_t n,
    uint32_t * bidx) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
    uint32_t lo = 0, hi = nblocks;  // largest b with blocks[b] <= v (skips empty blocks)
    while (hi - lo > 1) {
      const uint32_t mid = (lo + hi) / 2;
      if (__ldg(blocks + mid) <= v) lo = mid; else hi = mid;
    }
    bidx[v] = lo;
  }
}

// In-block degree (src/permute.c:66-77), one warp per row; iota for the sort.
__global__ void cm_degree_kernel(CmGraph g, uint32_t * deg, uint32_t * iota) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t warps = gridDim.x * (blockDim.x / 32);
  for (uint32_t v = (blockIdx.x * blockDim.x + threadIdx.x) / 32; v < g.n; v += warps) {
    uint32_t lo, hi;
    cm_block_range(g, v, lo, hi);
    const uint32_t s = __ldg(g.rowptr + v), e = __ldg(g.rowptr + v + 1);
    uint32_t d = 0;
    for (uint32_t j = s + lane; j < e; j += 32) {
      const uint32_t k = __ldg(g.rowind + j);
      d += (k >= lo && k < hi) ? 1u : 0u;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) d += __shfl_xor_sync(0xffffffffu, d, o);
    if (lane == 0) {
      deg[v] = d;
      iota[v] = v;
    }
  }
}

__global__ void cm_rank_kernel(const uint32_t * order, uint32_t n, uint32_t * rank) {
  for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x)
    rank[order[r]] = r;
}

// Exclusive scan of one value per thread over the CTA; returns the prefix and
// sets *total.  Ends with the CTA synchronised.
__device__ uint32_t cm_block_scan(uint32_t v, uint32_t * warp_sum, uint32_t * total) {
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x / 32;
  uint32_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= static_cast<uint32_t>(o)) x += y;
  }
  if (lane == 31) warp_sum[warp] = x;
  __syncthreads();
  if (warp == 0) {
    uint32_t w = warp_sum[lane];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= static_cast<uint32_t>(o)) w += y;
    }
    warp_sum[lane] = w;  // inclusive
  }
  __syncthreads();
  const uint32_t before = warp ? warp_sum[warp - 1] : 0u;
  *total = warp_sum[kCmThreads / 32 - 1];
  const uint32_t r = before + x - v;
  __syncthreads();
  return r;
}

// The persistent single-CTA driver: runs levels and components while they fit
// its shared memory, then records why it stopped.  claim[] is read through L2
// (__ldcg) because the atomics that write it bypass L1.
__global__ void __launch_bounds__(kCmThreads, 1)
cm_small_kernel(CmGraph g, const uint32_t * __restrict__ order,
    const uint32_t * __restrict__ rank, uint32_t * claim, uint32_t * perm, uint32_t * cand,
    CmState * st, uint32_t nbits) {
  extern __shared__ __align__(16) unsigned char cm_smem_raw[];
  CmSmem & sm = *reinterpret_cast<CmSmem *>(cm_smem_raw);
  const uint32_t tid = threadIdx.x;
  const uint32_t n = g.n;
  const unsigned long long mask = (1ull << nbits) - 1ull;
  uint32_t a = st->a, b = st->b, next = st->next, count = 0, mode = kCmDone;

  for (;;) {
    if (a == b) {
      if (b >= n) {
        mode = kCmDone;
        break;
      }
      // first unvisited vertex of the (degree, id) order: the new component's
      // start (src/permute.c:83-84)
      uint32_t found = kUnvisited;
      for (uint32_t base = next; base < n; base += kCmThreads) {
        const uint32_t r = base + tid;
        const bool f = r < n && __ldcg(claim + __ldg(order + r)) == kUnvisited;
        if (tid == 0) sm.found = kUnvisited;
        if (__syncthreads_or(f)) {
          if (f) atomicMin(&sm.found, r);
          __syncthreads();
          found = sm.found;
          break;
        }
      }
      if (found == kUnvisited) {  // nothing left (cannot happen while b < n)
        mode = kCmDone;
        break;
      }
      const uint32_t s = __ldg(order + found);
      next = found + 1;
      if (tid == 0) {
        claim[s] = b;
        perm[b] = s;
      }
      b += 1;
      __syncthreads();
    }

    // stage the frontier perm[a, b): row starts, lengths, block ranges
    const uint32_t L = b - a;
    if (L > kCmSmallFrontier) {
      mode = kCmExpand;
      break;
    }
    uint32_t len[4], sum = 0;
    bool big = false;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const uint32_t i = tid * 4 + q;
      len[q] = 0;
      if (i < L) {
        const uint32_t v = __ldcg(perm + a + i);
        const uint32_t rs = __ldg(g.rowptr + v);
        len[q] = __ldg(g.rowptr + v + 1) - rs;
        sm.rs[i] = rs;
        uint32_t lo, hi;
        cm_block_range(g, v, lo, hi);
        sm.lo[i] = lo;
        sm.hi[i] = hi;
        big |= len[q] > kCmSmallEdges;
      }
      sum += len[q];
    }
    if (__syncthreads_or(big)) {
      mode = kCmExpand;
      break;
    }
    uint32_t total;
    uint32_t off = cm_block_scan(sum, sm.warp_sum, &total);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const uint32_t i = tid * 4 + q;
      if (i < L) sm.off[i] = off;
      off += len[q];
    }
    if (tid == 0) {
      sm.off[L] = total;
      sm.count = 0;
    }
    if (total > kCmSmallEdges) {  // uniform: total is the same in every thread
      mode = kCmExpand;
      break;
    }
    __syncthreads();

    // expand: one thread per frontier entry, kCmUnroll entries in flight per
    // thread (their loads and atomics are issued before any result is used)
    for (uint32_t e0 = tid; e0 < total; e0 += kCmUnroll * kCmThreads) {
      uint32_t k[kCmUnroll], p[kCmUnroll];
      bool in[kCmUnroll];
#pragma unroll
      for (int u = 0; u < kCmUnroll; ++u) {
        const uint32_t e = e0 + u * kCmThreads;
        in[u] = false;
        k[u] = 0;
        p[u] = 0;
        if (e < total) {
          uint32_t lo = 0, hi = L;  // largest i with off[i] <= e
          while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) / 2;
            if (sm.off[mid] <= e) lo = mid; else hi = mid;
          }
          k[u] = __ldg(g.rowind + sm.rs[lo] + (e - sm.off[lo]));
          p[u] = lo;
          in[u] = true;
        }
      }
      uint32_t old[kCmUnroll];
#pragma unroll
      for (int u = 0; u < kCmUnroll; ++u) {
        in[u] = in[u] && k[u] >= sm.lo[p[u]] && k[u] < sm.hi[p[u]];
        old[u] = in[u] ? atomicMin(claim + k[u], a + p[u]) : 0u;
      }
#pragma unroll
      for (int u = 0; u < kCmUnroll; ++u) {
        if (in[u] && old[u] == kUnvisited) {
          const uint32_t slot = atomicAdd(&sm.count, 1u);
          cand[slot] = k[u];
        }
      }
    }
    __syncthreads();
    count = sm.count;
    if (count > kCmSmallLevel) {
      mode = kCmSort;
      break;
    }
    if (count == 0) {  // component finished
      a = b;
      continue;
    }

    // order the level by (first parent, degree, id) in shared memory.
    // Usually each parent has a few children: bucket the candidates by parent
    // (counts, scan, scatter), then sort each bucket by rank in one thread.
    uint32_t hk[kCmHeld], hp[kCmHeld], hpos[kCmHeld];
#pragma unroll
    for (int q = 0; q < kCmHeld; ++q) {
      const uint32_t i = tid * kCmHeld + q;
      if (i < L) sm.rs[i] = 0;  // bucket counts (the row starts are spent)
    }
    if (tid == 0) sm.maxb = 0;
    __syncthreads();
#pragma unroll
    for (int q = 0; q < kCmHeld; ++q) {
      const uint32_t i = tid + q * kCmThreads;
      if (i < count) {
        hk[q] = __ldcg(cand + i);
        hp[q] = __ldcg(claim + hk[q]) - a;
        hpos[q] = atomicAdd(&sm.rs[hp[q]], 1u);
        atomicMax(&sm.maxb, hpos[q] + 1);
      }
    }
    __syncthreads();
    if (sm.maxb <= kCmBucketMax) {
      uint32_t cnt[kCmHeld], csum = 0;
#pragma unroll
      for (int q = 0; q < kCmHeld; ++q) {
        const uint32_t i = tid * kCmHeld + q;
        cnt[q] = i < L ? sm.rs[i] : 0u;
        csum += cnt[q];
      }
      uint32_t tot;
      uint32_t o = cm_block_scan(csum, sm.warp_sum, &tot);
#pragma unroll
      for (int q = 0; q < kCmHeld; ++q) {
        const uint32_t i = tid * kCmHeld + q;
        if (i < L) sm.lo[i] = o;  // bucket starts (the block ranges are spent)
        o += cnt[q];
      }
      __syncthreads();
      uint32_t * slot_rank = reinterpret_cast<uint32_t *>(sm.key);
#pragma unroll
      for (int q = 0; q < kCmHeld; ++q) {
        const uint32_t i = tid + q * kCmThreads;
        if (i < count) slot_rank[sm.lo[hp[q]] + hpos[q]] = __ldg(rank + hk[q]);
      }
      __syncthreads();
#pragma unroll
      for (int q = 0; q < kCmHeld; ++q) {  // insertion sort of each bucket
        const uint32_t i = tid * kCmHeld + q;
        if (i < L) {
          const uint32_t s0 = sm.lo[i], c = sm.rs[i];
          for (uint32_t x = 1; x < c; ++x) {
            const uint32_t v = slot_rank[s0 + x];
            uint32_t y = x;
            while (y > 0 && slot_rank[s0 + y - 1] > v) {
              slot_rank[s0 + y] = slot_rank[s0 + y - 1];
              --y;
            }
            slot_rank[s0 + y] = v;
          }
        }
      }
      __syncthreads();
      for (uint32_t i = tid; i < count; i += kCmThreads)
        perm[b + i] = __ldg(order + slot_rank[i]);
      a = b;
      b += count;
      __syncthreads();
      continue;
    }
    uint32_t P = 1;
    while (P < count) P <<= 1;
    for (uint32_t i = tid; i < P; i += kCmThreads) {
      unsigned long long key = ~0ull;
      if (i < count) {
        const uint32_t k = __ldcg(cand + i);
        key = (static_cast<unsigned long long>(__ldcg(claim + k) - a) << nbits) | __ldg(rank + k);
      }
      sm.key[i] = key;
    }
    __syncthreads();
    for (uint32_t kk = 2; kk <= P; kk <<= 1) {
      for (uint32_t j = kk >> 1; j > 0; j >>= 1) {
        for (uint32_t i = tid; i < P; i += kCmThreads) {
          const uint32_t ixj = i ^ j;
          if (ixj > i) {
            const unsigned long long x = sm.key[i], y = sm.key[ixj];
            if ((x > y) == ((i & kk) == 0)) {
              sm.key[i] = y;
              sm.key[ixj] = x;
            }
          }
        }
        __syncthreads();
      }
    }
    for (uint32_t i = tid; i < count; i += kCmThreads)
      perm[b + i] = __ldg(order + static_cast<uint32_t>(sm.key[i] & mask));
    a = b;
    b += count;
    __syncthreads();
  }
  if (tid == 0) {
    st->a = a;
    st->b = b;
    st->next = next;
    st->count = count;
    st->mode = mode;
  }
}

// Row lengths of a large frontier (the scan turns them into offsets).
__global__ void cm_front_len_kernel(const uint32_t * rowptr, const uint32_t * perm, uint32_t a,
    uint32_t L, uint32_t * len) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i <= L; i += gridDim.x * blockDim.x) {
    uint32_t l = 0;
    if (i < L) {
      const uint32_t v = perm[a + i];
      l = __ldg(rowptr + v + 1) - __ldg(rowptr + v);
    }
    len[i] = l;
  }
}

// Edge-balanced expansion of a large frontier: each warp takes chunks of
// 32 * kCmLaneEdges consecutive frontier entries; lanes walk the row offsets
// forward.  New vertices go to cand[] through one atomic per warp and step.
__global__ void __launch_bounds__(kCmExpandThreads)
cm_expand_kernel(CmGraph g, const uint32_t * __restrict__ perm, uint32_t a, uint32_t L,
    const uint32_t * __restrict__ off, uint32_t * claim, uint32_t * cand, uint32_t * count) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t warps = gridDim.x * (blockDim.x / 32);
  const uint32_t total = __ldg(off + L);
  constexpr uint32_t kChunk = 32 * kCmLaneEdges;
  const uint32_t nchunks = (total + kChunk - 1) / kChunk;
  for (uint32_t c = (blockIdx.x * blockDim.x + threadIdx.x) / 32; c < nchunks; c += warps) {
    const uint32_t e0 = c * kChunk;
    uint32_t lo = 0, hi = L;  // largest i with off[i] <= e0
    while (hi - lo > 1) {
      const uint32_t mid = (lo + hi) / 2;
      if (__ldg(off + mid) <= e0) lo = mid; else hi = mid;
    }
    uint32_t idx = lo, cur = kUnvisited, rs = 0, base = 0, blo = 0, bhi = 0;
#pragma unroll 1
    for (uint32_t j = 0; j < kCmLaneEdges; ++j) {
      const uint32_t e = e0 + j * 32 + lane;
      uint32_t k = 0;
      bool take = false;
      if (e < total) {
        while (__ldg(off + idx + 1) <= e) ++idx;
        if (idx != cur) {
          cur = idx;
          const uint32_t v = __ldg(perm + a + idx);
          rs = __ldg(g.rowptr + v);
          base = __ldg(off + idx);
          cm_block_range(g, v, blo, bhi);
        }
        k = __ldg(g.rowind + rs + (e - base));
        if (k >= blo && k < bhi) take = atomicMin(claim + k, a + idx) == kUnvisited;
      }
      const uint32_t m = __ballot_sync(0xffffffffu, take);
      if (m) {
        const uint32_t leader = __ffs(m) - 1;
        uint32_t slot = 0;
        if (lane == leader) slot = atomicAdd(count, static_cast<uint32_t>(__popc(m)));
        slot = __shfl_sync(0xffffffffu, slot, leader);
        if (take) cand[slot + __popc(m & ((1u << lane) - 1u))] = k;
      }
    }
  }
}

__global__ void cm_key_kernel(const uint32_t * cand, uint32_t count, const uint32_t * claim,
    const uint32_t * rank, uint32_t a, uint32_t nbits, unsigned long long * keys) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
    const uint32_t k = cand[i];
    keys[i] = (static_cast<unsigned long long>(claim[k] - a) << nbits) | rank[k];
  }
}

__global__ void cm_decode_kernel(const unsigned long long * keys, uint32_t count,
    const uint32_t * order, uint32_t nbits, uint32_t * out) {
  const unsigned long long mask = (1ull << nbits) - 1ull;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x)
    out[i] = order[static_cast<uint32_t>(keys[i] & mask)];
}

__global__ void cm_block_key_kernel(const uint32_t * perm, const uint32_t * bidx, uint32_t n,
    uint32_t * keys) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    keys[i] = bidx[perm[i]];
}

uint32_t host_bits(uint64_t x) {  // bits to hold 0..x
  uint32_t b = 0;
  while (x) {
    ++b;
    x >>= 1;
  }
  return b;
}

// Scratch from the library pool, released in one place.
struct ScratchSet {
  cudaStream_t s;
  std::vector<void *> p;
  explicit ScratchSet(cudaStream_t st) : s(st) {}
  template <typename T>
  int get(T ** out, size_t count) {
    void * q = nullptr;
    GB_TRY(scratch_alloc(&q, std::max<size_t>(count, 1) * sizeof(T), s));
    p.push_back(q);
    *out = static_cast<T *>(q);
    return GOOSEBERRY_SUCCESS;
  }
  ~ScratchSet() {
    for (void * q : p) scratch_free(q, s);
  }
};

int grid_for(size_t items, int threads) {
  int sms = 148;
  sm_count_of_current_device(&sms);
  const size_t want = (items + threads - 1) / threads;
  return static_cast<int>(std::max<size_t>(1, std::min<size_t>(want, static_cast<size_t>(sms) * 8)));
}

}  // namespace

// Cuthill-McKee order of the n x n device CSR (rowptr, rowind) into the
// device array perm (perm[new] = old).  blocks: host array of nblocks+1
// boundaries covering [0, n), or null for one block.  max_row bounds the
// degree.  Synchronises `stream` once per large level.
int check_blocks(uint32_t n, const uint32_t * blocks, uint32_t nblocks) {
  if (!blocks) return GOOSEBERRY_SUCCESS;
  GB_CHECK_INPUT(blocks[0] == 0 && blocks[nblocks] == n,
      "row blocks must cover [0, %u): got [%u, %u)", n, blocks[0], blocks[nblocks]);
  for (uint32_t c = 0; c < nblocks; ++c)
    GB_CHECK_INPUT(blocks[c] <= blocks[c + 1], "row block %u has a negative size", c);
  return GOOSEBERRY_SUCCESS;
}

int cuthillmckee_device(uint32_t n, const uint32_t * rowptr, const uint32_t * rowind,
    uint32_t max_row, const uint32_t * blocks, uint32_t nblocks, uint32_t * perm,
    cudaStream_t stream) {
  if (n == 0) return GOOSEBERRY_SUCCESS;
  GB_TRY(check_blocks(n, blocks, nblocks));
  ScratchSet sc(stream);
  uint32_t *deg, *iota, *order, *rank, *claim, *cand, *len, *off;
  unsigned long long *keys, *keys_alt;
  CmState * st;
  GB_TRY(sc.get(&deg, n));
  GB_TRY(sc.get(&iota, n));
  GB_TRY(sc.get(&order, n));
  GB_TRY(sc.get(&rank, n));
  GB_TRY(sc.get(&claim, n));
  GB_TRY(sc.get(&cand, n));
  GB_TRY(sc.get(&len, static_cast<size_t>(n) + 1));
  GB_TRY(sc.get(&off, static_cast<size_t>(n) + 1));
  GB_TRY(sc.get(&keys, n));
  GB_TRY(sc.get(&keys_alt, n));
  GB_TRY(sc.get(&st, 1));
  uint32_t * count =
      reinterpret_cast<uint32_t *>(reinterpret_cast<char *>(st) + offsetof(CmState, pad));

  CmGraph g{rowptr, rowind, nullptr, nullptr, n};
  uint32_t *d_blocks = nullptr, *bidx = nullptr;
  if (blocks) {
    GB_TRY(sc.get(&d_blocks, static_cast<size_t>(nblocks) + 1));
    GB_TRY(sc.get(&bidx, n));
    GB_CUDA_TRY(cudaMemcpyAsync(d_blocks, blocks, (static_cast<size_t>(nblocks) + 1) * 4,
        cudaMemcpyHostToDevice, stream));
    cm_bidx_kernel<<<grid_for(n, 256), 256, 0, stream>>>(d_blocks, nblocks, n, bidx);
    GB_CUDA_TRY(cudaGetLastError());
    g.bidx = bidx;
    g.blocks = d_blocks;
  }

  // CUB temporary storage: the largest of the sorts and the scan
  const uint32_t nbits = std::max<uint32_t>(1, host_bits(n - 1));
  size_t tmp_bytes = 0, t = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, t, deg, deg, iota, order, n, 0, 32, stream);
  tmp_bytes = std::max(tmp_bytes, t);
  cub::DeviceRadixSort::SortKeys(nullptr, t, keys, keys_alt, n, 0, 64, stream);
  tmp_bytes = std::max(tmp_bytes, t);
  cub::DeviceScan::ExclusiveSum(nullptr, t, len, off, n + 1, stream);
  tmp_bytes = std::max(tmp_bytes, t);
  void * tmp = nullptr;
  GB_TRY(sc.get(reinterpret_cast<unsigned char **>(&tmp), tmp_bytes));

  // degrees and the (degree, id) order
  cm_degree_kernel<<<grid_for(static_cast<size_t>(n) * 32, 256), 256, 0, stream>>>(g, deg, iota);
  GB_CUDA_TRY(cudaGetLastError());
  uint32_t * deg_sorted = cand;  // free until the first level
  GB_CUDA_TRY(cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, deg, deg_sorted, iota, order, n, 0,
      static_cast<int>(std::max<uint32_t>(1, host_bits(max_row))), stream));
  cm_rank_kernel<<<grid_for(n, 256), 256, 0, stream>>>(order, n, rank);
  GB_CUDA_TRY(cudaGetLastError());
  GB_CUDA_TRY(cudaMemsetAsync(claim, 0xff, static_cast<size_t>(n) * 4, stream));

  CmState h{};
  GB_CUDA_TRY(cudaMemcpyAsync(st, &h, sizeof(h), cudaMemcpyHostToDevice, stream));
  const size_t smem = sizeof(CmSmem);
  GB_CUDA_TRY(cudaFuncSetAttribute(cm_small_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
      static_cast<int>(smem)));
  const int egrid = grid_for(static_cast<size_t>(n) * 4, kCmExpandThreads);
  for (;;) {
    cm_small_kernel<<<1, kCmThreads, smem, stream>>>(g, order, rank, claim, perm, cand, st, nbits);
    GB_CUDA_TRY(cudaGetLastError());
    GB_CUDA_TRY(cudaMemcpyAsync(&h, st, sizeof(h), cudaMemcpyDeviceToHost, stream));
    GB_CUDA_TRY(cudaStreamSynchronize(stream));
    if (h.mode == kCmDone) break;
    const uint32_t L = h.b - h.a;
    if (h.mode == kCmExpand) {
      cm_front_len_kernel<<<grid_for(static_cast<size_t>(L) + 1, 256), 256, 0, stream>>>(
          rowptr, perm, h.a, L, len);
      GB_CUDA_TRY(cudaGetLastError());
      GB_CUDA_TRY(cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, len, off, L + 1, stream));
      GB_CUDA_TRY(cudaMemsetAsync(count, 0, 4, stream));
      cm_expand_kernel<<<egrid, kCmExpandThreads, 0, stream>>>(g, perm, h.a, L, off, claim,
          cand, count);
      GB_CUDA_TRY(cudaGetLastError());
      GB_CUDA_TRY(cudaMemcpyAsync(&h.count, count, 4, cudaMemcpyDeviceToHost, stream));
      GB_CUDA_TRY(cudaStreamSynchronize(stream));
    }
    if (h.count > 0) {
      const uint32_t kbits = nbits + host_bits(L - 1);
      cm_key_kernel<<<grid_for(h.count, 256), 256, 0, stream>>>(cand, h.count, claim, rank, h.a,
          nbits, keys);
      GB_CUDA_TRY(cudaGetLastError());
      GB_CUDA_TRY(cub::DeviceRadixSort::SortKeys(tmp, tmp_bytes, keys, keys_alt, h.count, 0,
          static_cast<int>(kbits), stream));
      cm_decode_kernel<<<grid_for(h.count, 256), 256, 0, stream>>>(keys_alt, h.count, order, nbits,
          perm + h.b);
      GB_CUDA_TRY(cudaGetLastError());
    }
    h.a = h.b;
    h.b += h.count;
    h.count = 0;
    h.mode = kCmDone;
    GB_CUDA_TRY(cudaMemcpyAsync(st, &h, sizeof(h), cudaMemcpyHostToDevice, stream));
  }
  if (h.b != n) {
    set_error("internal error: ordered %u of %u vertices", h.b, n);
    return GOOSEBERRY_ERROR_UNKNOWN;
  }

  if (blocks && nblocks > 1) {
    // stable partition by block: each block keeps its vertices' relative order
    uint32_t *bkey, *bkey_out;
    GB_TRY(sc.get(&bkey, n));
    GB_TRY(sc.get(&bkey_out, n));
    size_t t2 = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, t2, bkey, bkey_out, perm, cand, n, 0, 32, stream);
    unsigned char * tmp2 = nullptr;
    GB_TRY(sc.get(&tmp2, t2));
    cm_block_key_kernel<<<grid_for(n, 256), 256, 0, stream>>>(perm, bidx, n, bkey);
    GB_CUDA_TRY(cudaGetLastError());
    GB_CUDA_TRY(cub::DeviceRadixSort::SortPairs(tmp2, t2, bkey, bkey_out, perm, cand, n, 0,
        static_cast<int>(std::max<uint32_t>(1, host_bits(nblocks - 1))), stream));
    GB_CUDA_TRY(cudaMemcpyAsync(perm, cand, static_cast<size_t>(n) * 4, cudaMemcpyDeviceToDevice,
        stream));
  }
  GB_CUDA_TRY(cudaStreamSynchronize(stream));
  return GOOSEBERRY_SUCCESS;
}

namespace {

// ---- sparse permutation (src/permute.c:120-205) ------------------------------

__global__ void pm_check_kernel(const uint32_t * perm, uint32_t n, uint32_t * seen,
    uint32_t * bad) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint32_t v = perm[i];
    if (v >= n || atomicExch(seen + v, 1u) != 0u) atomicExch(bad, 1u);
  }
}

__global__ void pm_len_kernel(const uint32_t * rowptr, const uint32_t * rowperm, uint32_t n,
    uint32_t * len) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i <= n; i += gridDim.x * blockDim.x) {
    uint32_t l = 0;
    if (i < n) {
      const uint32_t v = rowperm ? rowperm[i] : i;
      l = rowptr[v + 1] - rowptr[v];
    }
    len[i] = l;
  }
}

__global__ void pm_rename_kernel(const uint32_t * colperm, uint32_t ncols, uint32_t * rename) {
  for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < ncols; j += gridDim.x * blockDim.x)
    rename[colperm[j]] = j;
}

// One warp per new row: copy old row rowperm[i] with its entries in order.
__global__ void pm_copy_kernel(const uint32_t * __restrict__ rowptr,
    const uint32_t * __restrict__ rowind, const double * __restrict__ val64,
    const float * __restrict__ val32, const uint32_t * __restrict__ rowperm,
    const uint32_t * __restrict__ rename, const uint32_t * __restrict__ prowptr, uint32_t n,
    uint32_t * __restrict__ prowind, double * __restrict__ pval64, float * __restrict__ pval32) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t warps = gridDim.x * (blockDim.x / 32);
  for (uint32_t i = (blockIdx.x * blockDim.x + threadIdx.x) / 32; i < n; i += warps) {
    const uint32_t v = rowperm ? __ldg(rowperm + i) : i;
    const uint32_t s = __ldg(rowptr + v), e = __ldg(rowptr + v + 1), d = __ldg(prowptr + i);
    for (uint32_t j = s + lane; j < e; j += 32) {
      const uint32_t c = __ldg(rowind + j);
      prowind[d + (j - s)] = rename ? __ldg(rename + c) : c;
      if (pval64) pval64[d + (j - s)] = __ldg(val64 + j);
      if (pval32) pval32[d + (j - s)] = __ldg(val32 + j);
    }
  }
}

// Dense row-major nrows x ncols: out[i][j] = in[rowperm[i]][colperm[j]], or
// out[rowperm[i]][colperm[j]] = in[i][j] when reverse (null: identity).
template <typename T>
__global__ void pm_dense_kernel(uint32_t nrows, uint32_t ncols, const T * __restrict__ in,
    T * __restrict__ out, const uint32_t * __restrict__ rowperm,
    const uint32_t * __restrict__ colperm, int reverse) {
  const size_t total = static_cast<size_t>(nrows) * ncols;
  for (size_t q = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; q < total;
       q += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const uint32_t i = static_cast<uint32_t>(q / ncols), j = static_cast<uint32_t>(q % ncols);
    const size_t v = rowperm ? rowperm[i] : i;
    const size_t u = colperm ? colperm[j] : j;
    if (reverse) out[v * ncols + u] = in[q];
    else out[q] = in[v * ncols + u];
  }
}

__global__ void pm_vector_kernel(const double * x, const uint32_t * perm, uint32_t n, int reverse,
    double * y) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    if (reverse) y[perm[i]] = x[i];
    else y[i] = x[perm[i]];
  }
}

int check_perm(const uint32_t * perm, uint32_t n, const char * what, ScratchSet & sc,
    cudaStream_t stream) {
  if (!perm || n == 0) return GOOSEBERRY_SUCCESS;
  uint32_t * seen;
  GB_TRY(sc.get(&seen, static_cast<size_t>(n) + 1));
  GB_CUDA_TRY(cudaMemsetAsync(seen, 0, (static_cast<size_t>(n) + 1) * 4, stream));
  pm_check_kernel<<<grid_for(n, 256), 256, 0, stream>>>(perm, n, seen, seen + n);
  GB_CUDA_TRY(cudaGetLastError());
  uint32_t bad = 0;
  GB_CUDA_TRY(cudaMemcpyAsync(&bad, seen + n, 4, cudaMemcpyDeviceToHost, stream));
  GB_CUDA_TRY(cudaStreamSynchronize(stream));
  GB_CHECK_INPUT(bad == 0, "%s is not a permutation of 0..%u", what, n - 1);
  return GOOSEBERRY_SUCCESS;
}

}  // namespace

// Permute the device CSR (rowptr, rowind, val64 / val32 -- either may be
// null) into the preallocated outputs: new row i is old row rowperm[i], old
// column colperm[j] becomes column j.  Null permutations mean identity.  The
// permutations are checked; columns must be < ncols (the caller's matrix is
// validated).
int permute_sparse_device(uint32_t nrows, uint32_t ncols, const uint32_t * rowptr,
    const uint32_t * rowind, const double * val64, const float * val32,
    const uint32_t * rowperm, const uint32_t * colperm, uint32_t * prowptr, uint32_t * prowind,
    double * pval64, float * pval32, cudaStream_t stream) {
  ScratchSet sc(stream);
  GB_TRY(check_perm(rowperm, nrows, "rowperm", sc, stream));
  GB_TRY(check_perm(colperm, ncols, "colperm", sc, stream));
  uint32_t *len, *rename = nullptr;
  GB_TRY(sc.get(&len, static_cast<size_t>(nrows) + 1));
  pm_len_kernel<<<grid_for(static_cast<size_t>(nrows) + 1, 256), 256, 0, stream>>>(rowptr,
      rowperm, nrows, len);
  GB_CUDA_TRY(cudaGetLastError());
  size_t t = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, t, len, prowptr, nrows + 1, stream);
  unsigned char * tmp;
  GB_TRY(sc.get(&tmp, t));
  GB_CUDA_TRY(cub::DeviceScan::ExclusiveSum(tmp, t, len, prowptr, nrows + 1, stream));
  if (colperm) {
    GB_TRY(sc.get(&rename, ncols));
    pm_rename_kernel<<<grid_for(ncols, 256), 256, 0, stream>>>(colperm, ncols, rename);
    GB_CUDA_TRY(cudaGetLastError());
  }
  if (nrows) {
    pm_copy_kernel<<<grid_for(static_cast<size_t>(nrows) * 32, 256), 256, 0, stream>>>(rowptr,
        rowind, val64, val32, rowperm, rename, prowptr, nrows, prowind, pval64, pval32);
    GB_CUDA_TRY(cudaGetLastError());
  }
  GB_CUDA_TRY(cudaStreamSynchronize(stream));
  return GOOSEBERRY_SUCCESS;
}

}  // namespace gb

// ---- C ABI ------------------------------------------------------------------

namespace {

// Host rowptr check shared by the host-array entry points.
int check_rowptr(uint32_t n, const uint32_t * rowptr, uint32_t * max_row) {
  GB_CHECK_INPUT(rowptr != nullptr, "rowptr is NULL");
  GB_CHECK_INPUT(rowptr[0] == 0, "rowptr[0] must be 0");
  uint32_t m = 0;
  for (uint32_t i = 0; i < n; ++i) {
    GB_CHECK_INPUT(rowptr[i + 1] >= rowptr[i], "rowptr decreases at row %u", i);
    m = std::max(m, rowptr[i + 1] - rowptr[i]);
  }
  if (max_row) *max_row = m;
  return GOOSEBERRY_SUCCESS;
}

template <typename T>
int upload(gb::ScratchSet & sc, T ** d, const T * h, size_t count, cudaStream_t s) {
  GB_TRY(sc.get(d, count));
  if (count && h)
    GB_CUDA_TRY(cudaMemcpyAsync(*d, h, count * sizeof(T), cudaMemcpyHostToDevice, s));
  return GOOSEBERRY_SUCCESS;
}

// A permutation of 0..n-1 (checked on the host: the caller's arrays).
int check_perm_host(const uint32_t * perm, uint32_t n, const char * what) {
  if (!perm) return GOOSEBERRY_SUCCESS;
  std::vector<unsigned char> seen(n, 0);
  for (uint32_t i = 0; i < n; ++i) {
    GB_CHECK_INPUT(perm[i] < n && !seen[perm[i]], "%s is not a permutation of 0..%u", what,
        n - 1);
    seen[perm[i]] = 1;
  }
  return GOOSEBERRY_SUCCESS;
}

template <typename T>
int permute_dense_host(dim_t nrows, dim_t ncols, T * rowval, const dim_t * rowperm,
    const dim_t * colperm, int reverse) {
  if (!rowperm && !colperm) return GOOSEBERRY_SUCCESS;
  const size_t total = static_cast<size_t>(nrows) * ncols;
  if (total == 0) return GOOSEBERRY_SUCCESS;
  GB_CHECK_INPUT(rowval != nullptr, "rowval is NULL");
  GB_TRY(check_perm_host(rowperm, nrows, "rowperm"));
  GB_TRY(check_perm_host(colperm, ncols, "colperm"));
  cudaStream_t s = nullptr;
  gb::ScratchSet sc(s);
  T *in, *out;
  uint32_t *rpm = nullptr, *cpm = nullptr;
  GB_TRY(upload(sc, &in, rowval, total, s));
  GB_TRY(sc.get(&out, total));
  if (rowperm) GB_TRY(upload(sc, &rpm, rowperm, nrows, s));
  if (colperm) GB_TRY(upload(sc, &cpm, colperm, ncols, s));
  gb::pm_dense_kernel<T><<<gb::grid_for(total, 256), 256, 0, s>>>(nrows, ncols, in, out, rpm, cpm,
      reverse);
  GB_CUDA_TRY(cudaGetLastError());
  GB_CUDA_TRY(cudaMemcpyAsync(rowval, out, total * sizeof(T), cudaMemcpyDeviceToHost, s));
  GB_CUDA_TRY(cudaStreamSynchronize(s));
  return GOOSEBERRY_SUCCESS;
}

template <typename T>
int permute_sparse_host(dim_t nrows, dim_t ncols, ind_t * rowptr, dim_t * rowind, T * rowval,
    const dim_t * rowperm, const dim_t * colperm) {
  if (!rowperm && !colperm) return GOOSEBERRY_SUCCESS;
  GB_TRY(check_rowptr(nrows, rowptr, nullptr));
  const uint32_t nnz = rowptr[nrows];
  GB_CHECK_INPUT(nnz == 0 || (rowind && rowval), "NULL array");
  if (colperm) {
    for (uint32_t j = 0; j < nnz; ++j)
      GB_CHECK_INPUT(rowind[j] < ncols, "column index %u out of range for %u columns",
          rowind[j], ncols);
  }
  cudaStream_t s = nullptr;
  gb::ScratchSet sc(s);
  uint32_t *rp, *ri, *rpm = nullptr, *cpm = nullptr, *prp, *pri;
  T *rv, *prv;
  GB_TRY(upload(sc, &rp, rowptr, static_cast<size_t>(nrows) + 1, s));
  GB_TRY(upload(sc, &ri, rowind, nnz, s));
  GB_TRY(upload(sc, &rv, rowval, nnz, s));
  if (rowperm) GB_TRY(upload(sc, &rpm, rowperm, nrows, s));
  if (colperm) GB_TRY(upload(sc, &cpm, colperm, ncols, s));
  GB_TRY(sc.get(&prp, static_cast<size_t>(nrows) + 1));
  GB_TRY(sc.get(&pri, nnz));
  GB_TRY(sc.get(&prv, nnz));
  constexpr bool kF64 = sizeof(T) == 8;
  GB_TRY(gb::permute_sparse_device(nrows, ncols, rp, ri,
      kF64 ? reinterpret_cast<const double *>(rv) : nullptr,
      kF64 ? nullptr : reinterpret_cast<const float *>(rv), rpm, cpm, prp, pri,
      kF64 ? reinterpret_cast<double *>(prv) : nullptr,
      kF64 ? nullptr : reinterpret_cast<float *>(prv), s));
  GB_CUDA_TRY(cudaMemcpyAsync(rowptr, prp, (static_cast<size_t>(nrows) + 1) * 4,
      cudaMemcpyDeviceToHost, s));
  if (nnz) {
    GB_CUDA_TRY(cudaMemcpyAsync(rowind, pri, static_cast<size_t>(nnz) * 4, cudaMemcpyDeviceToHost, s));
    GB_CUDA_TRY(cudaMemcpyAsync(rowval, prv, static_cast<size_t>(nnz) * sizeof(T),
        cudaMemcpyDeviceToHost, s));
  }
  GB_CUDA_TRY(cudaStreamSynchronize(s));
  return GOOSEBERRY_SUCCESS;
}

}  // namespace

extern "C" {

int gooseberry_permute_cuthillmckee(dim_t nrows, dim_t ncols, const ind_t * rowptr,
    const dim_t * rowind, const void * rowval, const dim_t * blocks, dim_t nblocks,
    dim_t * perm) {
  (void)rowval;  // the order depends on the structure only
  gb::clear_error();
  GB_CHECK_INPUT(nrows == ncols,
      "Cuthill-McKee requires a structurally symmetric matrix: Given %ux%u", nrows, ncols);
  if (blocks && nblocks == 0) return GOOSEBERRY_SUCCESS;  // no block: nothing ordered
  if (nrows == 0) return GOOSEBERRY_SUCCESS;
  GB_CHECK_INPUT(perm != nullptr, "perm is NULL");
  uint32_t max_row = 0;
  GB_TRY(check_rowptr(nrows, rowptr, &max_row));
  GB_TRY(gb::check_blocks(nrows, blocks, nblocks));
  const uint32_t nnz = rowptr[nrows];
  GB_CHECK_INPUT(nnz == 0 || rowind, "rowind is NULL");
  cudaStream_t s = nullptr;
  gb::ScratchSet sc(s);
  uint32_t *rp, *ri, *pm;
  GB_TRY(upload(sc, &rp, rowptr, static_cast<size_t>(nrows) + 1, s));
  GB_TRY(upload(sc, &ri, rowind, nnz, s));
  GB_TRY(sc.get(&pm, nrows));
  GB_TRY(gb::cuthillmckee_device(nrows, rp, ri, max_row, blocks, nblocks, pm, s));
  GB_CUDA_TRY(cudaMemcpyAsync(perm, pm, static_cast<size_t>(nrows) * 4, cudaMemcpyDeviceToHost, s));
  GB_CUDA_TRY(cudaStreamSynchronize(s));
  return GOOSEBERRY_SUCCESS;
}

int gooseberry_permute_sparse(dim_t nrows, dim_t ncols, ind_t * rowptr, dim_t * rowind,
    float * rowval, const dim_t * rowperm, const dim_t * colperm) {
  gb::clear_error();
  return permute_sparse_host(nrows, ncols, rowptr, rowind, rowval, rowperm, colperm);
}

int gooseberry_permute_sparse_f64(dim_t nrows, dim_t ncols, ind_t * rowptr, dim_t * rowind,
    double * rowval, const dim_t * rowperm, const dim_t * colperm) {
  gb::clear_error();
  return permute_sparse_host(nrows, ncols, rowptr, rowind, rowval, rowperm, colperm);
}

int gooseberry_permute_dense(dim_t nrows, dim_t ncols, float * rowval, const dim_t * rowperm,
    const dim_t * colperm) {
  gb::clear_error();
  return permute_dense_host(nrows, ncols, rowval, rowperm, colperm, 0);
}

int gooseberry_permute_dense_f64(dim_t nrows, dim_t ncols, double * rowval,
    const dim_t * rowperm, const dim_t * colperm) {
  gb::clear_error();
  return permute_dense_host(nrows, ncols, rowval, rowperm, colperm, 0);
}

int gooseberry_permute_dense_rev(dim_t nrows, dim_t ncols, float * rowval,
    const dim_t * rowperm, const dim_t * colperm) {
  gb::clear_error();
  return permute_dense_host(nrows, ncols, rowval, rowperm, colperm, 1);
}

int gooseberry_permute_dense_rev_f64(dim_t nrows, dim_t ncols, double * rowval,
    const dim_t * rowperm, const dim_t * colperm) {
  gb::clear_error();
  return permute_dense_host(nrows, ncols, rowval, rowperm, colperm, 1);
}

int gb_csr_cuthillmckee(const gb_csr_t * a, const dim_t * blocks, dim_t nblocks, dim_t * perm,
    gb_stream_t stream) {
  gb::clear_error();
  GB_CHECK_INPUT(a != nullptr, "matrix is NULL");
  GB_CHECK_INPUT(a->nrows == a->ncols,
      "Cuthill-McKee requires a structurally symmetric matrix: Given %ux%u", a->nrows, a->ncols);
  if (blocks && nblocks == 0) return GOOSEBERRY_SUCCESS;
  if (a->nrows == 0) return GOOSEBERRY_SUCCESS;
  GB_CHECK_INPUT(perm != nullptr, "perm is NULL");
  return gb::cuthillmckee_device(a->nrows, a->rowptr, a->rowind, a->plan.max_row, blocks,
      nblocks, perm, static_cast<cudaStream_t>(stream));
}

int gb_csr_permute(const gb_csr_t * a, const dim_t * rowperm, const dim_t * colperm,
    gb_stream_t stream, gb_csr_t ** out) {
  gb::clear_error();
  GB_CHECK_INPUT(a != nullptr && out != nullptr, "NULL argument");
  *out = nullptr;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  uint32_t *prp = nullptr, *pri = nullptr;
  double * pv64 = nullptr;
  float * pv32 = nullptr;
  auto cleanup = [&]() {
    cudaStreamSynchronize(s);
    if (prp) gb::dev_free(prp);
    if (pri) gb::dev_free(pri);
    if (pv64) gb::dev_free(pv64);
    if (pv32) gb::dev_free(pv32);
  };
  int rc = gb::dev_alloc(&prp, (static_cast<size_t>(a->nrows) + 1) * 4);
  if (rc == GOOSEBERRY_SUCCESS)
    rc = gb::dev_alloc(&pri, std::max<size_t>(a->nnz, 1) * 4);
  if (rc == GOOSEBERRY_SUCCESS && a->val64)
    rc = gb::dev_alloc(&pv64, std::max<size_t>(a->nnz, 1) * 8);
  if (rc == GOOSEBERRY_SUCCESS && a->val32)
    rc = gb::dev_alloc(&pv32, std::max<size_t>(a->nnz, 1) * 4);
  if (rc == GOOSEBERRY_SUCCESS)
    rc = gb::permute_sparse_device(a->nrows, a->ncols, a->rowptr, a->rowind, a->val64, a->val32,
        rowperm, colperm, prp, pri, pv64, pv32, s);
  if (rc == GOOSEBERRY_SUCCESS)
    rc = gb::csr_adopt(a->nrows, a->ncols, a->nnz, prp, pri, pv64, pv32, s, out);
  if (rc != GOOSEBERRY_SUCCESS) cleanup();
  return rc;
}

int gb_permute_vector_f64(size_t n, const double * x, const dim_t * perm, int reverse, double * y,
    gb_stream_t stream) {
  GB_CHECK_INPUT(n <= 0xffffffffull, "n too large");
  GB_CHECK_INPUT(n == 0 || (x && perm && y), "NULL argument");
  GB_CHECK_INPUT(n == 0 || x != y, "x and y must not alias");
  if (n == 0) return GOOSEBERRY_SUCCESS;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  gb::pm_vector_kernel<<<gb::grid_for(n, 256), 256, 0, s>>>(x, perm, static_cast<uint32_t>(n),
      reverse, y);
  GB_CUDA_TRY(cudaGetLastError());
  return GOOSEBERRY_SUCCESS;
}

}  // extern "C"
