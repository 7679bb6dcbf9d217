// spmv.cu -- device-resident CSR matrices, the SpMV tile plan, the SpMV /
// SpMM launchers and the schedule autotuner.
//
// Reference path: blas_spmult (src/blas.c:552-606) splits rows evenly over
// OpenMP threads and runs __sparse_mult_dense_block (src/blas.c:67-92), a
// sequential per-row sum.  Here the rows are cut into row-aligned tiles of
// equal rows+nonzeros (balanced whatever the row-length distribution) and
// each tile is reduced on chip by a schedule picked per matrix.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <thread>
#include <tuple>
#include <vector>

#include "gb_internal.h"
#include "spmv_seg.cuh"
#include "spmv_tiles.cuh"

namespace gb {

// ---- plan -------------------------------------------------------------------

namespace {
constexpr uint32_t kDefaultTileItems = 2048;
constexpr uint32_t kChunkTiles = 4;  // a long-row chunk is 4 tiles of nonzeros
}  // namespace

namespace {

// The tiles that start at row r under the greedy rule, appended to `tiles`,
// and the row after them.  A row with more than tile_items - 1 nonzeros is a
// long row: chunk tiles of chunk_nnz nonzeros carrying `lid`, its long-row
// id (*nchunks > 0).  Otherwise one tile of whole rows while rows + nonzeros
// fit in tile_items (*nchunks = 0).  rowptr must be non-decreasing.
uint32_t tile_from(uint32_t r, uint32_t nrows, const uint32_t * rowptr, uint32_t tile_items,
    uint32_t chunk_nnz, uint32_t lid, std::vector<TileDesc> & tiles, uint32_t * nchunks) {
  const uint32_t b = rowptr[r], len = rowptr[r + 1] - b;
  if (static_cast<uint64_t>(len) + 1 > tile_items) {
    const uint32_t nch = (len + chunk_nnz - 1) / chunk_nnz;
    for (uint32_t q = 0; q < nch; ++q)
      tiles.push_back({lid, 0, b + q * chunk_nnz, std::min(chunk_nnz, len - q * chunk_nnz)});
    *nchunks = nch;
    return r + 1;
  }
  uint32_t items = 0, e = r;
  while (e < nrows) {
    const uint32_t l = rowptr[e + 1] - rowptr[e];
    if (static_cast<uint64_t>(l) + 1 > tile_items || items + l + 1 > tile_items) break;
    items += l + 1;
    ++e;
  }
  tiles.push_back({r, e - r, b, rowptr[e] - b});
  *nchunks = 0;
  return e;
}

// Greedy tiles of one segment of rows, planned from its first row as if a
// tile started there; the last step may run past the segment's end.
struct PlanSegment {
  uint32_t begin = 0, end = 0, stop = 0;  // rows [begin, end); steps end at row `stop`
  std::vector<TileDesc> tiles;            // chunk tiles carry segment-local long-row ids
  std::vector<uint32_t> step_row;         // first row of each step (a row tile or a long row)
  std::vector<uint32_t> step_tile;        // its first tile in `tiles`
  std::vector<uint32_t> step_long;        // long rows of the segment before the step
  std::vector<uint32_t> long_step;        // step of each long row
};

void plan_segment(PlanSegment & g, const uint32_t * rowptr, uint32_t nrows,
    uint32_t tile_items, uint32_t chunk_nnz) {
  uint32_t r = g.begin, nlong = 0;
  while (r < g.end) {
    g.step_row.push_back(r);
    g.step_tile.push_back(static_cast<uint32_t>(g.tiles.size()));
    g.step_long.push_back(nlong);
    uint32_t nch = 0;
    r = tile_from(r, nrows, rowptr, tile_items, chunk_nnz, nlong, g.tiles, &nch);
    if (nch) {
      g.long_step.push_back(static_cast<uint32_t>(g.step_row.size() - 1));
      ++nlong;
    }
  }
  g.stop = r;
}

// One tile step of the true plan, at row r; returns the next row.
uint32_t plan_step(Plan & plan, uint32_t r, const uint32_t * rowptr, uint32_t nrows) {
  const uint32_t first = static_cast<uint32_t>(plan.tiles.size());
  uint32_t nch = 0;
  const uint32_t lid = static_cast<uint32_t>(plan.longrows.size());
  const uint32_t next = tile_from(r, nrows, rowptr, plan.tile_items, plan.chunk_nnz, lid,
      plan.tiles, &nch);
  if (nch) plan.longrows.push_back({r, first, nch, 0});
  return next;
}

// body(t) for t in [0, nt), on nt threads (the caller's among them).  A
// thread that cannot be started runs its share inline instead: nothing
// throws through the C interface.
template <class F>
void run_threads(unsigned nt, F && body) {
  std::vector<std::thread> th;
  unsigned t = 1;
  try {
    th.reserve(nt);
    for (; t < nt; ++t) th.emplace_back(body, t);
  } catch (...) {
    for (unsigned u = t; u < nt; ++u) body(u);
  }
  body(0u);
  for (auto & x : th) x.join();
}

}  // namespace

// Tiles in the greedy order from row 0, computed by all host threads for
// large matrices: each thread plans its segment of rows from the segment's
// first row; a sequential pass then follows the true chain of tiles, takes
// over a segment's tiles from the first tile start the chain lands on (from a
// given row the greedy tiles are always the same, and every long row starts
// afresh), and plans tile by tile wherever it does not land on one.  The
// result is the plan the sequential rule gives.
int build_plan(uint32_t nrows, const uint32_t * rowptr, uint32_t nnz,
    uint32_t tile_items, Plan & plan) {
  if (tile_items < 64 || tile_items > 16384)
    GB_CHECK_INPUT(false, "tile_items %u outside [64, 16384]", tile_items);
  GB_CHECK_INPUT(rowptr[nrows] == nnz,
      "rowptr[nrows] = %u but the matrix has %u stored entries", rowptr[nrows], nnz);
  plan.tile_items = tile_items;
  plan.chunk_nnz = tile_items * kChunkTiles;
  plan.tiles.clear();
  plan.longrows.clear();

  constexpr uint32_t kSegmentRows = 32768;  // > the most rows one tile can hold
  const unsigned hw = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
  const unsigned nt = static_cast<unsigned>(std::max<uint64_t>(1,
      std::min<uint64_t>(hw, nrows / kSegmentRows)));

  // row-length histogram (exact counts below 1024, log2 buckets above), the
  // longest row and the first row where rowptr decreases
  struct Hist {
    std::vector<uint64_t> small = std::vector<uint64_t>(1024, 0), big = std::vector<uint64_t>(33, 0);
    uint32_t maxlen = 0, bad = 0xffffffffu;
  };
  std::vector<Hist> hist(nt);
  run_threads(nt, [&](unsigned t) {
    Hist h;  // thread-local until the end: the per-thread slots share cache lines
    const uint32_t a = static_cast<uint32_t>(uint64_t(nrows) * t / nt);
    const uint32_t z = static_cast<uint32_t>(uint64_t(nrows) * (t + 1) / nt);
    uint32_t mx = 0;
    for (uint32_t r = a; r < z; ++r) {
      const uint32_t b = rowptr[r], e = rowptr[r + 1];
      if (e < b) {
        h.bad = r;
        break;
      }
      const uint32_t len = e - b;
      mx = std::max(mx, len);
      if (len < 1024) ++h.small[len]; else ++h.big[32 - __builtin_clz(len)];
    }
    h.maxlen = mx;
    hist[t] = std::move(h);
  });
  std::vector<uint64_t> small(1024, 0), big(33, 0);
  uint32_t maxlen = 0, bad = 0xffffffffu;
  for (const Hist & h : hist) {
    for (int l = 0; l < 1024; ++l) small[l] += h.small[l];
    for (int k = 0; k < 33; ++k) big[k] += h.big[k];
    maxlen = std::max(maxlen, h.maxlen);
    bad = std::min(bad, h.bad);
  }
  GB_CHECK_INPUT(bad == 0xffffffffu, "rowptr decreases at row %u (%u > %u)", bad,
      bad == 0xffffffffu ? 0u : rowptr[bad], bad == 0xffffffffu ? 0u : rowptr[bad + 1]);

  if (nt == 1) {
    for (uint32_t r = 0; r < nrows;) r = plan_step(plan, r, rowptr, nrows);
  } else {
    std::vector<PlanSegment> seg(nt);
    run_threads(nt, [&](unsigned t) {
      PlanSegment g;  // thread-local until the end, as above
      g.begin = static_cast<uint32_t>(uint64_t(nrows) * t / nt);
      g.end = static_cast<uint32_t>(uint64_t(nrows) * (t + 1) / nt);
      plan_segment(g, rowptr, nrows, tile_items, plan.chunk_nnz);
      seg[t] = std::move(g);
    });
    uint32_t r = 0;
    for (unsigned t = 0; t < nt; ++t) {
      const PlanSegment & g = seg[t];
      size_t j = 0;  // first step of g at or after row r
      for (;;) {
        while (j < g.step_row.size() && g.step_row[j] < r) ++j;
        if (r >= g.end || (j < g.step_row.size() && g.step_row[j] == r)) break;
        r = plan_step(plan, r, rowptr, nrows);
      }
      if (r >= g.end) continue;
      // the chain is at step j of this segment: take its tiles from there
      const uint32_t tile0 = static_cast<uint32_t>(plan.tiles.size());
      const uint32_t long0 = static_cast<uint32_t>(plan.longrows.size());
      const uint32_t from_tile = g.step_tile[j], from_long = g.step_long[j];
      for (size_t i = from_tile; i < g.tiles.size(); ++i) {
        TileDesc d = g.tiles[i];
        if (d.row_count == 0) d.row_begin = d.row_begin - from_long + long0;
        plan.tiles.push_back(d);
      }
      for (size_t L = from_long; L < g.long_step.size(); ++L) {
        const uint32_t k = g.long_step[L];
        const uint32_t first = g.step_tile[k];
        const uint32_t last = k + 1 < g.step_tile.size() ? g.step_tile[k + 1]
                                                          : static_cast<uint32_t>(g.tiles.size());
        plan.longrows.push_back({g.step_row[k], tile0 + (first - from_tile), last - first, 0});
      }
      r = g.stop;
    }
  }

  // quantiles (exact below 1024, bucket upper bound above)
  auto quant = [&](double q) -> uint32_t {
    const uint64_t want = static_cast<uint64_t>(std::ceil(q * nrows));
    uint64_t acc = 0;
    for (uint32_t l = 0; l < 1024; ++l) {
      acc += small[l];
      if (acc >= want && want > 0) return l;
    }
    for (uint32_t k = 0; k < 33; ++k) {
      acc += big[k];
      if (acc >= want) return k >= 32 ? 0xffffffffu : ((1u << k) - 1);
    }
    return maxlen;
  };
  plan.max_row = maxlen;
  plan.mean_row = nrows ? static_cast<double>(nnz) / nrows : 0.0;
  plan.p50 = quant(0.50);
  plan.p90 = quant(0.90);
  plan.p99 = quant(0.99);
  return GOOSEBERRY_SUCCESS;
}

uint32_t seg_max_warps(int sm_count) {
  return static_cast<uint32_t>(std::max(sm_count, 1)) * kSegMinBlocks * kSegWarps;
}

// Ranges of a merge-path split of (row ends, nonzeros) into equal shares of
// rows + nonzeros, each range start rounded down to a multiple of 4.  At
// least kSegMinItems items per warp, so small matrices use fewer warps.
void build_seg_plan(uint32_t nrows, const uint32_t * rowptr, uint32_t nnz,
    uint32_t max_warps, Plan & plan) {
  constexpr uint64_t kSegMinItems = 96;
  const uint64_t total = static_cast<uint64_t>(nrows) + nnz;
  const uint32_t W = static_cast<uint32_t>(std::max<uint64_t>(1,
      std::min<uint64_t>(max_warps, total / kSegMinItems)));
  std::vector<uint32_t> nzb(static_cast<size_t>(W) + 1);
  for (uint32_t w = 0; w < W; ++w) {
    const uint64_t d = total * w / W;
    // rows whose end comes before merge position d: the smallest i with
    // rowptr[i + 1] + i >= d (row i's end sits at merge position rowptr[i+1] + i)
    uint64_t lo = d > nnz ? d - nnz : 0, hi = std::min<uint64_t>(d, nrows);
    while (lo < hi) {
      const uint64_t mid = (lo + hi) / 2;
      if (static_cast<uint64_t>(rowptr[mid + 1]) + mid < d) lo = mid + 1; else hi = mid;
    }
    nzb[w] = static_cast<uint32_t>(std::min<uint64_t>(d - lo, nnz)) & ~3u;
  }
  for (uint32_t w = 1; w < W; ++w) nzb[w] = std::max(nzb[w], nzb[w - 1]);
  nzb[W] = nnz;
  // warp holding nonzero p (the last range starting at or before p)
  auto warp_of = [&](uint32_t p) {
    return static_cast<uint32_t>(std::upper_bound(nzb.begin(), nzb.begin() + W, p) -
                                 nzb.begin()) - 1;
  };
  // row holding nonzero p < nnz (the last row starting at or before p)
  auto row_of = [&](uint32_t p) {
    return static_cast<uint32_t>(std::upper_bound(rowptr, rowptr + nrows + 1, p) - rowptr) - 1;
  };
  std::vector<uint32_t> nonempty_before(static_cast<size_t>(W) + 1, 0);
  for (uint32_t w = 0; w < W; ++w)
    nonempty_before[w + 1] = nonempty_before[w] + (nzb[w + 1] > nzb[w] ? 1u : 0u);
  plan.seg.assign(static_cast<size_t>(W) + 1, SegRange{});
  for (uint32_t w = 0; w <= W; ++w) {
    SegRange & g = plan.seg[w];
    g.nz_begin = nzb[w];
    g.head_row = g.head_first = g.tail_last = kSegNone;
    g.span_count = 0;
    if (w == W) continue;
    g.row_begin = static_cast<uint32_t>(
        std::lower_bound(rowptr, rowptr + nrows + 1, nzb[w]) - rowptr);
    if (g.row_begin > nrows) g.row_begin = nrows;
    if (nzb[w + 1] == nzb[w]) continue;  // no nonzeros: no rows to join
    const uint32_t hr = row_of(nzb[w]);
    if (rowptr[hr] < nzb[w]) {
      g.head_row = hr;
      g.head_first = warp_of(rowptr[hr]);
      if (rowptr[hr + 1] <= nzb[w + 1])
        g.span_count = nonempty_before[w + 1] - nonempty_before[g.head_first];
    }
    const uint32_t tr = row_of(nzb[w + 1] - 1);
    if (rowptr[tr + 1] > nzb[w + 1]) g.tail_last = warp_of(rowptr[tr + 1] - 1);
  }
}

void free_plan(Plan & plan) {
  if (plan.d_tiles || plan.d_longrows || plan.d_chunk_partial || plan.d_long_count ||
      plan.d_seg)
    cudaDeviceSynchronize();  // no kernel may still read the old plan
  if (plan.d_tiles) dev_free(plan.d_tiles);
  if (plan.d_longrows) dev_free(plan.d_longrows);
  if (plan.d_chunk_partial) dev_free(plan.d_chunk_partial);
  if (plan.d_long_count) dev_free(plan.d_long_count);
  if (plan.d_seg) dev_free(plan.d_seg);
  if (plan.d_seg_rec) dev_free(plan.d_seg_rec);
  if (plan.d_seg_count) dev_free(plan.d_seg_count);
  plan.d_tiles = nullptr;
  plan.d_longrows = nullptr;
  plan.d_chunk_partial = nullptr;
  plan.d_long_count = nullptr;
  plan.d_seg = nullptr;
  plan.d_seg_rec = nullptr;
  plan.d_seg_count = nullptr;
}

namespace {
// The segmented part of a plan, on the device (plan.seg built on the host).
int upload_seg(Plan & plan, cudaStream_t stream) {
  if (plan.seg.empty()) return GOOSEBERRY_SUCCESS;
  const size_t W = plan.seg.size() - 1;
  GB_TRY(dev_alloc(&plan.d_seg, plan.seg.size() * sizeof(SegRange)));
  GB_TRY(dev_alloc(&plan.d_seg_rec, 2 * W * sizeof(double)));
  GB_TRY(dev_alloc(&plan.d_seg_count, W * sizeof(unsigned int)));
  GB_CUDA_TRY(cudaMemcpyAsync(plan.d_seg, plan.seg.data(), plan.seg.size() * sizeof(SegRange),
      cudaMemcpyHostToDevice, stream));
  GB_CUDA_TRY(cudaMemsetAsync(plan.d_seg_rec, 0, 2 * W * sizeof(double), stream));
  GB_CUDA_TRY(cudaMemsetAsync(plan.d_seg_count, 0, W * sizeof(unsigned int), stream));
  return GOOSEBERRY_SUCCESS;
}
}  // namespace

int upload_plan(Plan & plan, cudaStream_t stream) {
  free_plan(plan);
  const size_t nt = std::max<size_t>(plan.tiles.size(), 1);
  const size_t nl = std::max<size_t>(plan.longrows.size(), 1);
  GB_TRY(dev_alloc(&plan.d_tiles, nt * sizeof(TileDesc)));
  GB_TRY(dev_alloc(&plan.d_longrows, nl * sizeof(LongRowDesc)));
  GB_TRY(dev_alloc(&plan.d_chunk_partial, nt * sizeof(double)));
  GB_TRY(dev_alloc(&plan.d_long_count, nl * sizeof(unsigned int)));
  if (!plan.tiles.empty())
    GB_CUDA_TRY(cudaMemcpyAsync(plan.d_tiles, plan.tiles.data(),
        plan.tiles.size() * sizeof(TileDesc), cudaMemcpyHostToDevice, stream));
  if (!plan.longrows.empty())
    GB_CUDA_TRY(cudaMemcpyAsync(plan.d_longrows, plan.longrows.data(),
        plan.longrows.size() * sizeof(LongRowDesc), cudaMemcpyHostToDevice, stream));
  GB_CUDA_TRY(cudaMemsetAsync(plan.d_long_count, 0, nl * sizeof(unsigned int), stream));
  GB_TRY(upload_seg(plan, stream));
  GB_CUDA_TRY(cudaStreamSynchronize(stream));  // host vectors may change later
  return GOOSEBERRY_SUCCESS;
}

int default_schedule(const Plan & plan) {
  if (plan.max_row <= 16 && plan.mean_row <= 12.0) return GB_SCHED_ROW;
  if (plan.max_row <= 32 && plan.mean_row <= 16.0) return GB_SCHED_THREAD;
  if (plan.p99 <= 2 * plan.p50 + 8 && plan.mean_row <= 40.0) return GB_SCHED_GROUP4;
  if (plan.p99 <= 2 * plan.p50 + 8 && plan.mean_row <= 160.0) return GB_SCHED_GROUP8;
  return GB_SCHED_MERGE;
}

// ---- kernels ----------------------------------------------------------------

template <typename Acc, typename Y>
struct OutStore {
  Y * y;
  uint32_t stride;
  __device__ __forceinline__ void row(uint32_t r, Acc v) {
    y[static_cast<size_t>(r) * stride] = static_cast<Y>(v);
  }
  __device__ __forceinline__ void long_row(uint32_t, uint32_t r, Acc v) { row(r, v); }
  __device__ __forceinline__ void finish() {}
  // per-row operands prefetched by the row schedule (none for a plain store)
  struct Pre {};
  __device__ __forceinline__ Pre pre(uint32_t) const { return Pre{}; }
  __device__ __forceinline__ void row_pre(uint32_t r, Acc v, const Pre &) { row(r, v); }
};

template <typename V, typename Acc, int SCHED, class Gather, class Out, bool DIRECT>
__global__ void __launch_bounds__(DIRECT ? kDirectBlock : kSpmvBlock,
    DIRECT ? kDirectMinBlocks : TileMinBlocks<SCHED, Gather>::value)
spmv_tiles_kernel(const PlanView plan, const uint32_t * __restrict__ rowptr,
    const uint32_t * __restrict__ rowind, const V * __restrict__ val, const Gather gather,
    Out out) {
  spmv_tiles_body<V, Acc, SCHED, DIRECT ? kDirectBlock : kSpmvBlock, Gather, Out, DIRECT>(
      plan, rowptr, rowind, val, gather, out);
}

// The row schedule in one pass, for a matrix whose rows all fit one thread's
// register stage and whose rows all fit one wave of threads: one row per
// thread, every entry of the row loaded at once, every gather in flight
// together, the products summed in the reference's order with unfused
// multiply and add (bit-identical to the pipelined row loop and to
// blas_spmult, src/blas.c:82-91).  The whole SpMV is then three dependent
// memory round trips (rowptr, entries, gathers) in a single wave, where the
// pipelined loop, sized for long grid-stride runs, holds fewer threads.
constexpr int kRow1Block = 128;
constexpr int kRow1Stage = 12;
template <typename V, typename Acc, class Out>
__global__ void __launch_bounds__(kRow1Block) spmv_row1_kernel(uint32_t nrows, uint32_t ncols,
    const uint32_t * __restrict__ rowptr, const uint32_t * __restrict__ rowind,
    const V * __restrict__ val, const Acc * __restrict__ x, Out out) {
  const uint32_t i = blockIdx.x * kRow1Block + threadIdx.x;
  if (i >= nrows) return;
  const uint32_t b = __ldg(rowptr + i), e = __ldg(rowptr + i + 1);
  uint32_t c[kRow1Stage];
  V v[kRow1Stage];
#pragma unroll
  for (int j = 0; j < kRow1Stage; ++j) {
    if (b + j < e) {
      c[j] = ld_l1(rowind + b + j, NoHint{});
      v[j] = ld_l1(val + b + j, NoHint{});
    }
  }
  Acc xv[kRow1Stage];
  const uint32_t cmax = ncols - 1;
#pragma unroll
  for (int j = 0; j < kRow1Stage; ++j)
    if (b + j < e) xv[j] = __ldg(x + min(c[j], cmax));
  Acc sum = Acc(0);
#pragma unroll
  for (int j = 0; j < kRow1Stage; ++j)
    if (b + j < e) sum = add_rn(sum, mul_rn(static_cast<Acc>(v[j]), xv[j]));
  out.row(i, sum);
}

__global__ void max_index_kernel(const uint32_t * __restrict__ ind, uint32_t n,
    unsigned int * out) {
  uint32_t m = 0;
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<size_t>(gridDim.x) * blockDim.x)
    m = max(m, ind[i]);
  m = max(m, __reduce_max_sync(0xffffffffu, m));
  if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

__global__ void round_f32_kernel(const double * __restrict__ in, float * __restrict__ out,
    size_t n) {
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<size_t>(gridDim.x) * blockDim.x)
    out[i] = static_cast<float>(in[i]);
}

// ---- launch helpers ---------------------------------------------------------

// Resident CTAs per SM of a kernel at a dynamic shared-memory size (cached),
// after raising the kernel's dynamic shared-memory limit to cover it (the
// limit only grows: lowering it for a small tile made a later launch at a
// larger, already cached, tile size fail with an invalid argument).
int occupancy(const void * func, size_t smem, int * out, int block = kSpmvBlock) {
  static std::mutex mu;
  static std::map<std::tuple<const void *, size_t, int>, int> cache;
  std::lock_guard<std::mutex> lock(mu);
  int dev = 0;
  GB_CUDA_TRY(cudaGetDevice(&dev));
  auto key = std::make_tuple(func, smem, dev);
  auto it = cache.find(key);
  if (it != cache.end()) {
    *out = it->second;
    return GOOSEBERRY_SUCCESS;
  }
  int max_smem = 0;
  GB_CUDA_TRY(cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  GB_CHECK_INPUT(smem <= static_cast<size_t>(max_smem),
      "this schedule needs %zu bytes of shared memory per CTA at this tile size; the "
      "device allows %d (choose smaller tile_items)", smem, max_smem);
  GB_TRY(raise_smem_limit(func, smem));
  int n = 0;
  GB_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, func, block, smem));
  if (n < 1) {
    set_error("SpMV kernel cannot be resident with %zu bytes of shared memory", smem);
    return GOOSEBERRY_ERROR_UNKNOWN;
  }
  cache[key] = n;
  *out = n;
  return GOOSEBERRY_SUCCESS;
}

template <typename V, typename Acc, int SCHED, class Gather, class Out>
int launch_tiles(const gb_csr & a, const V * val, const Gather & g, const Out & o,
    cudaStream_t stream) {
  if (a.plan.tiles.empty()) return GOOSEBERRY_SUCCESS;
  auto kern = spmv_tiles_kernel<V, Acc, SCHED, Gather, Out, false>;
  size_t smem = spmv_smem_bytes<V, Acc>(SCHED, a.plan.tile_items, kSpmvBlock);
  int block = kSpmvBlock;
  if constexpr (IsPlainGather<Gather>::value && SCHED != SCHED_ROW && SCHED != SCHED_WTILE &&
                SCHED != SCHED_WMERGE) {
    // plain y = A x on CTA tiles: the direct register pipeline when the tile
    // fits its per-thread item budget
    if (a.plan.tile_items <= static_cast<uint32_t>(kDirectKt * kDirectBlock)) {
      kern = spmv_tiles_kernel<V, Acc, SCHED, Gather, Out, true>;
      smem = DirectSmem<Acc>::bytes(a.plan.tile_items);
      block = kDirectBlock;
    }
  }
  int occ = 0;
  GB_TRY(occupancy(reinterpret_cast<const void *>(kern), smem, &occ, block));
  const uint32_t units = spmv_work_units(SCHED, a.nrows,
      static_cast<uint32_t>(a.plan.tiles.size()), block);
  const uint32_t grid = std::min<uint32_t>(units, static_cast<uint32_t>(a.sm_count * occ));
  kern<<<grid, block, smem, stream>>>(plan_view(a), a.rowptr, a.rowind, val, g, o);
  GB_CUDA_TRY(cudaGetLastError());
  return GOOSEBERRY_SUCCESS;
}

template <typename V, typename Acc, class Out>
__global__ void __launch_bounds__(kSegBlock, kSegMinBlocks)
spmv_seg_kernel(const SegView sv, const uint32_t * __restrict__ rowptr,
    const uint32_t * __restrict__ rowind, const V * __restrict__ val,
    const Acc * __restrict__ x, Out out) {
  spmv_seg_body<V, Acc, GB_SEG_K>(sv, rowptr, rowind, val, x, out);
}

// Whether the segmented schedule's 16-byte loads can read these arrays.
bool seg_aligned(const gb_csr & a, const void * val) {
  return (reinterpret_cast<uintptr_t>(a.rowind) & 15u) == 0 &&
         (reinterpret_cast<uintptr_t>(val) & 15u) == 0;
}

template <typename V, typename Acc, class Gather, class Out>
int launch_seg(const gb_csr & a, const V * val, const Gather & g, const Out & o,
    cudaStream_t stream) {
  if constexpr (IsPlainGather<Gather>::value) {
    if (a.nrows == 0) return GOOSEBERRY_SUCCESS;
    GB_CHECK_INPUT(a.plan.d_seg != nullptr, "the matrix has no segmented plan");
    GB_CHECK_INPUT(a.nnz == 0 || seg_aligned(a, val),
        "the segmented schedule needs rowind and values on 16-byte boundaries");
    SegView sv;
    sv.ranges = a.plan.d_seg;
    sv.nwarps = static_cast<uint32_t>(a.plan.seg.size() - 1);
    sv.head_rec = a.plan.d_seg_rec;
    sv.tail_rec = a.plan.d_seg_rec + sv.nwarps;
    sv.count = a.plan.d_seg_count;
    sv.nrows = a.nrows;
    sv.ncols = a.ncols;
    sv.nnz = a.nnz;
    const uint32_t grid = (sv.nwarps + kSegWarps - 1) / kSegWarps;
    spmv_seg_kernel<V, Acc, Out><<<grid, kSegBlock, 0, stream>>>(sv, a.rowptr, a.rowind, val,
        g.x, o);
    GB_CUDA_TRY(cudaGetLastError());
    return GOOSEBERRY_SUCCESS;
  } else {
    set_error("the segmented schedule computes plain SpMV only");
    return GOOSEBERRY_ERROR_INVALIDINPUT;
  }
}

// The one-pass row kernel when the rows fit its stage and one wave holds
// every row; *done = false leaves the launch to the pipelined row loop.
template <typename V, typename Acc, class Gather, class Out>
int launch_row1(const gb_csr & a, const V * val, const Gather & g, const Out & o,
    cudaStream_t stream, bool * done) {
  *done = false;
  if constexpr (IsPlainGather<Gather>::value) {
    if (a.nrows == 0 || a.plan.max_row > static_cast<uint32_t>(kRow1Stage)) return GOOSEBERRY_SUCCESS;
    auto kern = spmv_row1_kernel<V, Acc, Out>;
    int occ = 0;
    GB_TRY(occupancy(reinterpret_cast<const void *>(kern), 0, &occ, kRow1Block));
    const uint64_t wave = static_cast<uint64_t>(a.sm_count) * occ * kRow1Block;
    if (a.nrows > wave) return GOOSEBERRY_SUCCESS;
    kern<<<(a.nrows + kRow1Block - 1) / kRow1Block, kRow1Block, 0, stream>>>(a.nrows, a.ncols,
        a.rowptr, a.rowind, val, g.x, o);
    GB_CUDA_TRY(cudaGetLastError());
    *done = true;
  }
  return GOOSEBERRY_SUCCESS;
}

template <typename V, typename Acc, class Gather, class Out>
int launch_sched(const gb_csr & a, int sched, const V * val, const Gather & g,
    const Out & o, cudaStream_t stream) {
  if (sched == GB_SCHED_ROW) {
    bool done = false;
    GB_TRY((launch_row1<V, Acc>(a, val, g, o, stream, &done)));
    if (done) return GOOSEBERRY_SUCCESS;
  }
  switch (sched) {
    case GB_SCHED_SEG: return launch_seg<V, Acc>(a, val, g, o, stream);
    case GB_SCHED_THREAD: return launch_tiles<V, Acc, SCHED_THREAD>(a, val, g, o, stream);
    case GB_SCHED_GROUP4: return launch_tiles<V, Acc, SCHED_GROUP4>(a, val, g, o, stream);
    case GB_SCHED_GROUP8: return launch_tiles<V, Acc, SCHED_GROUP8>(a, val, g, o, stream);
    case GB_SCHED_WARP: return launch_tiles<V, Acc, SCHED_WARP>(a, val, g, o, stream);
    case GB_SCHED_MERGE: return launch_tiles<V, Acc, SCHED_MERGE>(a, val, g, o, stream);
    case GB_SCHED_ROW: return launch_tiles<V, Acc, SCHED_ROW>(a, val, g, o, stream);
    case GB_SCHED_WTILE: return launch_tiles<V, Acc, SCHED_WTILE>(a, val, g, o, stream);
    case GB_SCHED_WMERGE: return launch_tiles<V, Acc, SCHED_WMERGE>(a, val, g, o, stream);
    default:
      set_error("unknown SpMV schedule %d", sched);
      return GOOSEBERRY_ERROR_INVALIDINPUT;
  }
}

int launch_spmv_f64(const gb_csr & a, int sched, const double * x, double * y,
    uint32_t stride, cudaStream_t stream) {
  GB_CHECK_INPUT(a.val64 != nullptr, "matrix holds no double values");
  GatherPlain<double> g{x};
  OutStore<double, double> o{y, stride};
  return launch_sched<double, double>(a, sched, a.val64, g, o, stream);
}

int launch_spmv_f32(const gb_csr & a, int sched, const float * x, float * y,
    uint32_t stride, cudaStream_t stream) {
  GB_CHECK_INPUT(a.val32 != nullptr, "matrix holds no float values");
  GatherPlain<float> g{x};
  OutStore<float, float> o{y, stride};
  return launch_sched<float, float>(a, sched, a.val32, g, o, stream);
}

int launch_max_index(const uint32_t * rowind, uint32_t nnz, unsigned int * d_out,
    cudaStream_t stream) {
  GB_CUDA_TRY(cudaMemsetAsync(d_out, 0, sizeof(unsigned int), stream));
  if (nnz == 0) return GOOSEBERRY_SUCCESS;
  int sms = 0;
  GB_TRY(sm_count_of_current_device(&sms));
  const uint32_t grid = std::min<uint32_t>((nnz + 255) / 256, static_cast<uint32_t>(sms) * 8);
  max_index_kernel<<<grid, 256, 0, stream>>>(rowind, nnz, d_out);
  GB_CUDA_TRY(cudaGetLastError());
  return GOOSEBERRY_SUCCESS;
}

int launch_round_f32(const double * in, float * out, size_t n, cudaStream_t stream) {
  if (n == 0) return GOOSEBERRY_SUCCESS;
  int sms = 0;
  GB_TRY(sm_count_of_current_device(&sms));
  const size_t grid = std::min<size_t>((n + 255) / 256, static_cast<size_t>(sms) * 8);
  round_f32_kernel<<<static_cast<unsigned>(grid), 256, 0, stream>>>(in, out, n);
  GB_CUDA_TRY(cudaGetLastError());
  return GOOSEBERRY_SUCCESS;
}

// ---- autotuner --------------------------------------------------------------

namespace {

struct TuneKey {
  uint32_t p50, p90, p99, maxlog2, nrows_log2, nnz_log2;
  unsigned width;
  bool operator<(const TuneKey & o) const {
    return std::tie(p50, p90, p99, maxlog2, nrows_log2, nnz_log2, width) <
           std::tie(o.p50, o.p90, o.p99, o.maxlog2, o.nrows_log2, o.nnz_log2, o.width);
  }
};
struct TuneChoice {
  int sched;
  uint32_t tile_items;
};
std::mutex g_tune_mu;
std::map<TuneKey, TuneChoice> g_tune_cache;

uint32_t ilog2(uint64_t v) { return v ? 63u - static_cast<uint32_t>(__builtin_clzll(v)) : 0u; }

TuneKey make_key(const gb_csr & a, unsigned width) {
  TuneKey k;
  k.p50 = a.plan.p50;
  k.p90 = a.plan.p90;
  k.p99 = a.plan.p99;
  k.maxlog2 = ilog2(a.plan.max_row);
  k.nrows_log2 = ilog2(a.nrows);
  k.nnz_log2 = ilog2(a.nnz);
  k.width = width;
  return k;
}

}  // namespace

int rebuild_plan(gb_csr & a, uint32_t tile_items, cudaStream_t stream) {
  if (tile_items == a.plan.tile_items && a.plan.d_tiles) return GOOSEBERRY_SUCCESS;
  std::vector<uint32_t> hrp(static_cast<size_t>(a.nrows) + 1);
  GB_CUDA_TRY(cudaMemcpyAsync(hrp.data(), a.rowptr, hrp.size() * sizeof(uint32_t),
      cudaMemcpyDeviceToHost, stream));
  GB_CUDA_TRY(cudaStreamSynchronize(stream));
  Plan p;
  GB_TRY(build_plan(a.nrows, hrp.data(), a.nnz, tile_items, p));
  GB_TRY(upload_plan(p, stream));
  // the segmented plan does not depend on the tile size: keep it
  p.seg = std::move(a.plan.seg);
  std::swap(p.d_seg, a.plan.d_seg);
  std::swap(p.d_seg_rec, a.plan.d_seg_rec);
  std::swap(p.d_seg_count, a.plan.d_seg_count);
  free_plan(a.plan);
  a.plan = std::move(p);
  return GOOSEBERRY_SUCCESS;
}

// The segmented plan is built the first time the SEG schedule is chosen (by
// gb_csr_set_schedule or the autotuner): it costs a host pass over rowptr
// that most matrices -- every CG operator on the row schedule -- never need.
int ensure_seg_plan(gb_csr & a, cudaStream_t stream) {
  if (a.plan.d_seg || a.nrows == 0) return GOOSEBERRY_SUCCESS;
  std::vector<uint32_t> hrp(static_cast<size_t>(a.nrows) + 1);
  GB_CUDA_TRY(cudaMemcpyAsync(hrp.data(), a.rowptr, hrp.size() * sizeof(uint32_t),
      cudaMemcpyDeviceToHost, stream));
  GB_CUDA_TRY(cudaStreamSynchronize(stream));
  build_seg_plan(a.nrows, hrp.data(), a.nnz, seg_max_warps(a.sm_count), a.plan);
  int rc = upload_seg(a.plan, stream);
  if (rc == GOOSEBERRY_SUCCESS && cudaStreamSynchronize(stream) != cudaSuccess) {
    set_error("segmented plan upload: %s", cudaGetErrorString(cudaGetLastError()));
    rc = GOOSEBERRY_ERROR_UNKNOWN;
  }
  if (rc != GOOSEBERRY_SUCCESS) {  // leave no half-built plan behind
    cudaDeviceSynchronize();
    if (a.plan.d_seg) dev_free(a.plan.d_seg);
    if (a.plan.d_seg_rec) dev_free(a.plan.d_seg_rec);
    if (a.plan.d_seg_count) dev_free(a.plan.d_seg_count);
    a.plan.d_seg = nullptr;
    a.plan.d_seg_rec = nullptr;
    a.plan.d_seg_count = nullptr;
    a.plan.seg.clear();
  }
  return rc;
}

int autotune(gb_csr & a, unsigned width, cudaStream_t stream) {
  const TuneKey key = make_key(a, width);
  {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    auto it = g_tune_cache.find(key);
    if (it != g_tune_cache.end()) {
      GB_TRY(rebuild_plan(a, it->second.tile_items, stream));
      if (it->second.sched == GB_SCHED_SEG) GB_TRY(ensure_seg_plan(a, stream));
      (width == GB_CSR_VALUES_F32 ? a.sched32 : a.sched64) = it->second.sched;
      return GOOSEBERRY_SUCCESS;
    }
  }
  const size_t xb = static_cast<size_t>(a.ncols) * (width == GB_CSR_VALUES_F32 ? 4 : 8);
  const size_t yb = static_cast<size_t>(a.nrows) * (width == GB_CSR_VALUES_F32 ? 4 : 8);
  void * x = nullptr;
  void * y = nullptr;
  GB_TRY(dev_alloc(&x, std::max<size_t>(xb, 8)));
  GB_TRY(dev_alloc(&y, std::max<size_t>(yb, 8)));
  GB_CUDA_TRY(cudaMemsetAsync(x, 0, std::max<size_t>(xb, 8), stream));
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  // (tile_items, schedule) candidates: CTA tiles are large, per-warp tiles
  // small, the row schedule ignores tiles
  struct Cand {
    uint32_t tile;
    int sched;
  };
  std::vector<Cand> cands;
  const bool short_rows = a.plan.p99 <= 64 && a.plan.max_row <= 4096;
  if (short_rows) cands.push_back({1024, GB_SCHED_ROW});
  for (uint32_t t : {128u, 256u, 512u}) cands.push_back({t, GB_SCHED_WTILE});
  cands.push_back({static_cast<uint32_t>(32 * kWmKt), GB_SCHED_WMERGE});
  const void * vals = width == GB_CSR_VALUES_F32 ? static_cast<const void *>(a.val32)
                                                  : static_cast<const void *>(a.val64);
  if (seg_aligned(a, vals)) cands.push_back({kDefaultTileItems, GB_SCHED_SEG});
  for (uint32_t t : {512u, 1024u, 2048u, 4096u}) {
    if (a.plan.p90 <= 64) cands.push_back({t, GB_SCHED_THREAD});
    cands.push_back({t, GB_SCHED_GROUP4});
    cands.push_back({t, GB_SCHED_GROUP8});
    if (a.plan.p50 >= 8) cands.push_back({t, GB_SCHED_WARP});
    cands.push_back({t, GB_SCHED_MERGE});
  }
  float best = 1e30f;
  TuneChoice choice{default_schedule(a.plan), a.plan.tile_items};
  int rc = GOOSEBERRY_SUCCESS;
  for (const Cand & cd : cands) {
    rc = rebuild_plan(a, cd.tile, stream);
    if (rc == GOOSEBERRY_SUCCESS && cd.sched == GB_SCHED_SEG) rc = ensure_seg_plan(a, stream);
    if (rc != GOOSEBERRY_SUCCESS) break;
    {
      const int s = cd.sched;
      const uint32_t ti = cd.tile;
      auto run = [&]() {
        return width == GB_CSR_VALUES_F32
                   ? launch_spmv_f32(a, s, static_cast<const float *>(x),
                         static_cast<float *>(y), 1, stream)
                   : launch_spmv_f64(a, s, static_cast<const double *>(x),
                         static_cast<double *>(y), 1, stream);
      };
      rc = run();  // warm-up
      if (rc != GOOSEBERRY_SUCCESS) break;
      const int reps = 5;
      cudaEventRecord(e0, stream);
      for (int q = 0; q < reps && rc == GOOSEBERRY_SUCCESS; ++q) rc = run();
      cudaEventRecord(e1, stream);
      if (rc != GOOSEBERRY_SUCCESS) break;
      if (cudaEventSynchronize(e1) != cudaSuccess) {
        set_error("autotune timing failed: %s", cudaGetErrorString(cudaGetLastError()));
        rc = GOOSEBERRY_ERROR_UNKNOWN;
        break;
      }
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      if (ms < best) {
        best = ms;
        choice = TuneChoice{s, ti};
      }
    }
    if (rc != GOOSEBERRY_SUCCESS) break;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  dev_free(x);
  dev_free(y);
  GB_TRY(rc);
  GB_TRY(rebuild_plan(a, choice.tile_items, stream));
  (width == GB_CSR_VALUES_F32 ? a.sched32 : a.sched64) = choice.sched;
  std::lock_guard<std::mutex> lock(g_tune_mu);
  g_tune_cache[key] = choice;
  return GOOSEBERRY_SUCCESS;
}

}  // namespace gb

// ---- C ABI ------------------------------------------------------------------

using gb::dev_alloc;
using gb::dev_free;
using gb::set_error;

namespace {

template <typename T>
int alloc_copy(void ** dst, const T * src, size_t n, bool device_src, cudaStream_t s) {
  GB_TRY(dev_alloc(dst, std::max<size_t>(n, 1) * sizeof(T)));
  if (n)
    GB_CUDA_TRY(cudaMemcpyAsync(*dst, src, n * sizeof(T),
        device_src ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s));
  return GOOSEBERRY_SUCCESS;
}

void release(gb_csr * a) {
  if (!a) return;
  // uploads may still be in flight on the creating stream (a creation that
  // failed part-way), and dev_free releases on the pool's own stream
  if (a->own_rowptr || a->own_rowind || a->own_val64 || a->own_val32) cudaDeviceSynchronize();
  gb::free_plan(a->plan);
  if (a->own_rowptr) dev_free(a->own_rowptr);
  if (a->own_rowind) dev_free(a->own_rowind);
  if (a->own_val64) dev_free(a->own_val64);
  if (a->own_val32) dev_free(a->own_val32);
  delete a;
}

int create_impl(dim_t nrows, dim_t ncols, ind_t nnz, const ind_t * rowptr,
    const dim_t * rowind, const double * rowval64, const float * rowval32,
    unsigned flags, cudaStream_t stream, gb_csr * a) {
  const bool dev = (flags & GB_CSR_DEVICE_POINTERS) != 0;
  const bool want64 = (flags & GB_CSR_VALUES_F64) != 0;
  const bool want32 = (flags & GB_CSR_VALUES_F32) != 0;
  GB_CHECK_INPUT(want64 || want32, "flags select no value width");
  GB_CHECK_INPUT(rowptr != nullptr, "rowptr is NULL");
  GB_CHECK_INPUT(nnz == 0 || rowind != nullptr, "rowind is NULL");
  GB_CHECK_INPUT(!want64 || nnz == 0 || rowval64 != nullptr, "double values requested but rowval64 is NULL");
  GB_CHECK_INPUT(!want32 || nnz == 0 || rowval32 != nullptr || rowval64 != nullptr,
      "float values requested but no values given");
  GB_CHECK_INPUT(nrows == 0 || ncols > 0, "matrix with rows but no columns");

  a->nrows = nrows;
  a->ncols = ncols;
  a->nnz = nnz;
  GB_CUDA_TRY(cudaGetDevice(&a->device));
  GB_TRY(gb::sm_count_of_current_device(&a->sm_count));

  // host copy of rowptr for the plan
  std::vector<uint32_t> hrp;
  const uint32_t * rp_host = rowptr;
  if (dev) {
    hrp.resize(static_cast<size_t>(nrows) + 1);
    GB_CUDA_TRY(cudaMemcpyAsync(hrp.data(), rowptr, hrp.size() * sizeof(uint32_t),
        cudaMemcpyDeviceToHost, stream));
    GB_CUDA_TRY(cudaStreamSynchronize(stream));
    rp_host = hrp.data();
  }
  // Host arrays: the uploads are queued first, so that (from pinned memory)
  // the copies run while the host builds the tile plan.  A failure after this
  // point frees the arrays through release(), which synchronises first.
  if (dev) {
    a->rowptr = rowptr;
    a->rowind = rowind;
    a->val64 = want64 ? rowval64 : nullptr;
    a->val32 = (want32 && rowval32) ? rowval32 : nullptr;
  } else {
    GB_TRY(alloc_copy(&a->own_rowptr, rowptr, static_cast<size_t>(nrows) + 1, false, stream));
    GB_TRY(alloc_copy(&a->own_rowind, rowind, nnz, false, stream));
    a->rowptr = static_cast<const uint32_t *>(a->own_rowptr);
    a->rowind = static_cast<const uint32_t *>(a->own_rowind);
    if (want64) {
      GB_TRY(alloc_copy(&a->own_val64, rowval64, nnz, false, stream));
      a->val64 = static_cast<const double *>(a->own_val64);
    }
    if (want32 && rowval32) {
      GB_TRY(alloc_copy(&a->own_val32, rowval32, nnz, false, stream));
      a->val32 = static_cast<const float *>(a->own_val32);
    }
  }
  GB_TRY(gb::build_plan(nrows, rp_host, nnz, gb::kDefaultTileItems, a->plan));
  if (want32 && !a->val32) {
    // round from the double values (already on the device, or upload them)
    const double * src = a->val64;
    void * tmp = nullptr;
    if (!src) {
      GB_TRY(alloc_copy(&tmp, rowval64, nnz, dev, stream));
      src = static_cast<const double *>(tmp);
    }
    GB_TRY(dev_alloc(&a->own_val32, std::max<size_t>(nnz, 1) * sizeof(float)));
    int rc = gb::launch_round_f32(src, static_cast<float *>(a->own_val32), nnz, stream);
    if (tmp) {
      cudaStreamSynchronize(stream);
      dev_free(tmp);
    }
    GB_TRY(rc);
    a->val32 = static_cast<const float *>(a->own_val32);
  }

  // validate column indices on the device
  if (nnz > 0) {
    unsigned int * d_max = nullptr;
    GB_TRY(dev_alloc(&d_max, sizeof(unsigned int)));
    unsigned int hmax = 0;
    int rc = gb::launch_max_index(a->rowind, nnz, d_max, stream);
    if (rc == GOOSEBERRY_SUCCESS) {
      cudaError_t e = cudaMemcpyAsync(&hmax, d_max, sizeof(hmax), cudaMemcpyDeviceToHost, stream);
      if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
      if (e != cudaSuccess) {
        set_error("index validation failed: %s", cudaGetErrorString(e));
        rc = GOOSEBERRY_ERROR_UNKNOWN;
      }
    }
    dev_free(d_max);
    GB_TRY(rc);
    GB_CHECK_INPUT(hmax < ncols, "column index %u out of range for %u columns", hmax, ncols);
  }
  GB_TRY(gb::upload_plan(a->plan, stream));
  a->sched64 = gb::default_schedule(a->plan);
  a->sched32 = a->sched64;
  return GOOSEBERRY_SUCCESS;
}

}  // namespace

namespace gb {

int csr_adopt(uint32_t nrows, uint32_t ncols, uint32_t nnz, uint32_t * rowptr,
    uint32_t * rowind, double * val64, float * val32, cudaStream_t stream, gb_csr ** out) {
  *out = nullptr;
  const unsigned flags = GB_CSR_DEVICE_POINTERS | (val64 ? GB_CSR_VALUES_F64 : 0u) |
                         (val32 ? GB_CSR_VALUES_F32 : 0u);
  gb_csr * a = new gb_csr();
  int rc = create_impl(nrows, ncols, nnz, rowptr, rowind, val64, val32, flags, stream, a);
  if (rc != GOOSEBERRY_SUCCESS) {
    release(a);  // frees only what create_impl allocated itself
    return rc;
  }
  a->own_rowptr = rowptr;
  a->own_rowind = rowind;
  a->own_val64 = val64;
  if (val32) a->own_val32 = val32;
  *out = a;
  return GOOSEBERRY_SUCCESS;
}

}  // namespace gb

extern "C" {

int gb_csr_create(dim_t nrows, dim_t ncols, ind_t nnz, const ind_t * rowptr,
    const dim_t * rowind, const double * rowval64, const float * rowval32,
    unsigned flags, gb_stream_t stream, gb_csr_t ** out) {
  GB_CHECK_INPUT(out != nullptr, "out is NULL");
  *out = nullptr;
  gb_csr * a = new gb_csr();
  int rc = create_impl(nrows, ncols, nnz, rowptr, rowind, rowval64, rowval32, flags,
      static_cast<cudaStream_t>(stream), a);
  if (rc != GOOSEBERRY_SUCCESS) {
    release(a);
    return rc;
  }
  *out = a;
  return GOOSEBERRY_SUCCESS;
}

int gb_csr_destroy(gb_csr_t * a) {
  release(a);
  return GOOSEBERRY_SUCCESS;
}

int gb_csr_get_info(const gb_csr_t * a, gb_csr_info_t * info) {
  GB_CHECK_INPUT(a && info, "NULL argument");
  info->nrows = a->nrows;
  info->ncols = a->ncols;
  info->nnz = a->nnz;
  info->ntiles = static_cast<uint32_t>(a->plan.tiles.size());
  info->nlong = static_cast<uint32_t>(a->plan.longrows.size());
  info->max_row = a->plan.max_row;
  info->mean_row = a->plan.mean_row;
  info->row_p50 = a->plan.p50;
  info->row_p90 = a->plan.p90;
  info->row_p99 = a->plan.p99;
  info->schedule = a->sched64;
  info->schedule_f32 = a->sched32;
  info->tile_items = a->plan.tile_items;
  return GOOSEBERRY_SUCCESS;
}

int gb_csr_set_schedule(gb_csr_t * a, unsigned value_width, int schedule,
    uint32_t tile_items) {
  GB_CHECK_INPUT(a != nullptr, "matrix is NULL");
  GB_CHECK_INPUT(schedule >= GB_SCHED_AUTO && schedule <= GB_SCHED_SEG,
      "unknown schedule %d", schedule);
  GB_CHECK_INPUT(schedule != GB_SCHED_SEG || a->nnz == 0 ||
                     gb::seg_aligned(*a, value_width == GB_CSR_VALUES_F32
                                             ? static_cast<const void *>(a->val32)
                                             : static_cast<const void *>(a->val64)),
      "the segmented schedule needs rowind and values on 16-byte boundaries");
  GB_CHECK_INPUT(value_width == GB_CSR_VALUES_F64 || value_width == GB_CSR_VALUES_F32,
      "value_width must be GB_CSR_VALUES_F64 or GB_CSR_VALUES_F32");
  // per-warp tiles keep two stages per warp in shared memory: they need small
  // tiles, so a plan built for CTA tiles is rebuilt at 256 items
  if (schedule == GB_SCHED_WTILE && tile_items == 0 && a->plan.tile_items > 512)
    tile_items = 256;
  GB_CHECK_INPUT(schedule != GB_SCHED_WTILE || (tile_items ? tile_items : a->plan.tile_items) <= 512,
      "per-warp tiles need tile_items <= 512");
  // per-warp merge tiles: at most kWmKt items per lane
  constexpr uint32_t wm_max = 32 * gb::kWmKt;
  if (schedule == GB_SCHED_WMERGE && tile_items == 0 && a->plan.tile_items > wm_max)
    tile_items = wm_max;
  GB_CHECK_INPUT(schedule != GB_SCHED_WMERGE ||
                     (tile_items ? tile_items : a->plan.tile_items) <= wm_max,
      "per-warp merge tiles need tile_items <= %u", wm_max);
  if (tile_items) GB_TRY(gb::rebuild_plan(*a, tile_items, nullptr));
  if (schedule == GB_SCHED_SEG) GB_TRY(gb::ensure_seg_plan(*a, nullptr));
  const int s = schedule == GB_SCHED_AUTO ? gb::default_schedule(a->plan) : schedule;
  (value_width == GB_CSR_VALUES_F32 ? a->sched32 : a->sched64) = s;
  return GOOSEBERRY_SUCCESS;
}

int gb_csr_autotune(gb_csr_t * a, unsigned value_width, gb_stream_t stream) {
  GB_CHECK_INPUT(a != nullptr, "matrix is NULL");
  GB_CHECK_INPUT(value_width == GB_CSR_VALUES_F64 || value_width == GB_CSR_VALUES_F32,
      "value_width must be GB_CSR_VALUES_F64 or GB_CSR_VALUES_F32");
  GB_CHECK_INPUT(value_width == GB_CSR_VALUES_F64 ? a->val64 != nullptr : a->val32 != nullptr,
      "matrix holds no values of that width");
  return gb::autotune(*a, value_width, static_cast<cudaStream_t>(stream));
}

int gb_plan_tiles_host(dim_t nrows, const ind_t * rowptr, ind_t nnz, uint32_t tile_items,
    uint32_t * tiles, size_t max_tiles, uint32_t * ntiles, uint32_t * nlong,
    gb_csr_info_t * info) {
  GB_CHECK_INPUT(rowptr != nullptr, "rowptr is NULL");
  gb::Plan p;
  GB_TRY(gb::build_plan(nrows, rowptr, nnz, tile_items ? tile_items : 2048u, p));
  if (ntiles) *ntiles = static_cast<uint32_t>(p.tiles.size());
  if (nlong) *nlong = static_cast<uint32_t>(p.longrows.size());
  if (tiles) {
    GB_CHECK_INPUT(max_tiles >= p.tiles.size(), "room for %zu tiles, plan has %zu",
        max_tiles, p.tiles.size());
    for (size_t t = 0; t < p.tiles.size(); ++t) {
      tiles[4 * t + 0] = p.tiles[t].row_begin;
      tiles[4 * t + 1] = p.tiles[t].row_count;
      tiles[4 * t + 2] = p.tiles[t].nnz_begin;
      tiles[4 * t + 3] = p.tiles[t].nnz_count;
    }
  }
  if (info) {
    std::memset(info, 0, sizeof(*info));
    info->nrows = nrows;
    info->ncols = 0;
    info->nnz = nnz;
    info->ntiles = static_cast<uint32_t>(p.tiles.size());
    info->nlong = static_cast<uint32_t>(p.longrows.size());
    info->max_row = p.max_row;
    info->mean_row = p.mean_row;
    info->row_p50 = p.p50;
    info->row_p90 = p.p90;
    info->row_p99 = p.p99;
    info->schedule = gb::default_schedule(p);
    info->schedule_f32 = info->schedule;
    info->tile_items = p.tile_items;
  }
  return GOOSEBERRY_SUCCESS;
}

int gb_spmv_f64(const gb_csr_t * a, const double * x, double * y, gb_stream_t stream) {
  GB_CHECK_INPUT(a != nullptr, "matrix is NULL");
  GB_CHECK_INPUT(a->nrows == 0 || y != nullptr, "y is NULL");
  GB_CHECK_INPUT(a->nnz == 0 || x != nullptr, "x is NULL");
  return gb::launch_spmv_f64(*a, a->sched64, x, y, 1, static_cast<cudaStream_t>(stream));
}

int gb_spmv_f32(const gb_csr_t * a, const float * x, float * y, gb_stream_t stream) {
  GB_CHECK_INPUT(a != nullptr, "matrix is NULL");
  GB_CHECK_INPUT(a->nrows == 0 || y != nullptr, "y is NULL");
  GB_CHECK_INPUT(a->nnz == 0 || x != nullptr, "x is NULL");
  return gb::launch_spmv_f32(*a, a->sched32, x, y, 1, static_cast<cudaStream_t>(stream));
}

int gb_spmm_f64(const gb_csr_t * a, dim_t bncols, const double * b, double * c,
    gb_stream_t stream) {
  GB_CHECK_INPUT(a != nullptr, "matrix is NULL");
  GB_CHECK_INPUT(a->nrows == 0 || bncols == 0 || c != nullptr, "c is NULL");
  GB_CHECK_INPUT(a->nnz == 0 || bncols == 0 || b != nullptr, "b is NULL");
  GB_CHECK_INPUT(a->val64 != nullptr, "matrix holds no double values");
  bool fused = false;
  GB_TRY(gb::launch_spmm_fused<double>(*a, bncols, a->val64, b, c,
      static_cast<cudaStream_t>(stream), &fused));
  if (fused) return GOOSEBERRY_SUCCESS;
  for (dim_t j = 0; j < bncols; ++j)  // one SpMV per column (long rows, or one column)
    GB_TRY(gb::launch_spmv_f64(*a, a->sched64, b + static_cast<size_t>(j) * a->ncols, c + j,
        bncols, static_cast<cudaStream_t>(stream)));
  return GOOSEBERRY_SUCCESS;
}

}  // extern "C"
