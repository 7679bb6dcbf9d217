// pagerank.cu -- PageRank power iteration on the device SpMV: the reference's
// `pagerank` command (src/gooseberry_bin.c:2610-2741) for a square CSR graph
// already in memory (no permutation file, one run).
//
// Normalisation is done on the device with the reference's arithmetic (column
// sums accumulated in row order, every value divided by its column's sum,
// rows without entries are the sinks), so the device matrix holds the same
// values: a stable radix sort of the entries by column keeps each column's
// entries in row order, one thread per column adds them in that order, and
// each value is divided by its column's sum.
// Per iteration on the device: out = A rank (the library SpMV, its matrix's
// schedule); dist = sum of rank over the sinks (fixed-order reduction);
// out = out * damping, then out += (1 - damping)/n + dist (two roundings, as
// blas_scale then blas_add_scalar); every 10th iteration (i % 10 == 0) also
// err = sum (rank - out)^2 in the same kernel, which the host reads to stop.
// rank and out then swap roles.  The reference's semantics are kept as they
// are, quirks included: the whole sink mass is added to every entry (not
// spread over n), and when the iteration limit ends the run the result is the
// second-to-last iterate (the buffer the last swap left in `out`).
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <cmath>
#include <vector>

#include "gb_internal.h"
#include "spmv_tiles.cuh"

namespace gb {
namespace {

constexpr int kPrBlock = 256;

// [begin, end) of CTA b of g over n elements
__device__ __forceinline__ void pr_chunk(size_t n, unsigned b, unsigned g, size_t & s,
    size_t & e) {
  const size_t q = n / g, r = n % g;
  s = b * q + min(static_cast<size_t>(b), r);
  e = s + q + (b < r ? 1 : 0);
}

// partial[b] = sum of rank[sinks[k]] over CTA b's chunk of the sink list
__global__ void __launch_bounds__(kPrBlock) pr_sink_kernel(size_t nsinks,
    const uint32_t * __restrict__ sinks, const double * __restrict__ rank,
    double * __restrict__ partial) {
  __shared__ double red[32];
  size_t s, e;
  pr_chunk(nsinks, blockIdx.x, gridDim.x, s, e);
  double acc = 0.0;
  for (size_t k = s + threadIdx.x; k < e; k += kPrBlock) acc += rank[sinks[k]];
  acc = block_sum(acc, red);
  if (threadIdx.x == 0) partial[blockIdx.x] = acc;
}

// *out = sum of partial[0..g) in index order (one CTA)
__global__ void __launch_bounds__(kPrBlock) pr_final_kernel(unsigned g,
    const double * __restrict__ partial, double * __restrict__ out) {
  __shared__ double red[32];
  double acc = 0.0;
  for (unsigned i = threadIdx.x; i < g; i += kPrBlock) acc += partial[i];
  acc = block_sum(acc, red);
  if (threadIdx.x == 0) *out = acc;
}

// out = out * damping; out += c + dist  (and, when check, partial[b] = sum of
// (rank - out)^2 over CTA b's chunk)
__global__ void __launch_bounds__(kPrBlock) pr_update_kernel(size_t n,
    double * __restrict__ out, const double * __restrict__ rank, double damping, double c,
    const double * __restrict__ dist, int check, double * __restrict__ partial) {
  __shared__ double red[32];
  size_t s, e;
  pr_chunk(n, blockIdx.x, gridDim.x, s, e);
  const double add = __dadd_rn(c, *dist);
  double acc = 0.0;
  for (size_t k = s + threadIdx.x; k < e; k += kPrBlock) {
    const double v = __dadd_rn(__dmul_rn(out[k], damping), add);
    out[k] = v;
    if (check) {
      const double d = __dsub_rn(rank[k], v);
      acc = __dadd_rn(acc, __dmul_rn(d, d));
    }
  }
  if (check) {
    acc = block_sum(acc, red);
    if (threadIdx.x == 0) partial[blockIdx.x] = acc;
  }
}

// partial[b] = sum of (a - b)^2 over CTA b's chunk
__global__ void __launch_bounds__(kPrBlock) pr_diff_kernel(size_t n,
    const double * __restrict__ a, const double * __restrict__ b, double * __restrict__ partial) {
  __shared__ double red[32];
  size_t s, e;
  pr_chunk(n, blockIdx.x, gridDim.x, s, e);
  double acc = 0.0;
  for (size_t k = s + threadIdx.x; k < e; k += kPrBlock) {
    const double d = a[k] - b[k];
    acc += d * d;
  }
  acc = block_sum(acc, red);
  if (threadIdx.x == 0) partial[blockIdx.x] = acc;
}

// ---- normalisation (src/gooseberry_bin.c:2611-2630) --------------------------

__global__ void pr_iota_count_kernel(uint32_t nnz, const uint32_t * __restrict__ rowind,
    uint32_t * __restrict__ iota, uint32_t * __restrict__ count) {
  for (uint32_t l = blockIdx.x * blockDim.x + threadIdx.x; l < nnz; l += gridDim.x * blockDim.x) {
    iota[l] = l;
    atomicAdd(count + rowind[l], 1u);
  }
}

// indeg[c] = sum of the values of column c, entries in row order (the sorted
// entry numbers of a column ascend); the reference's loop adds them in the
// same order without fusing (src/gooseberry_bin.c:2611-2621).
__global__ void pr_colsum_kernel(uint32_t n, const uint32_t * __restrict__ colptr,
    const uint32_t * __restrict__ entry, const double * __restrict__ val,
    double * __restrict__ indeg) {
  for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
    double s = 0.0;
    for (uint32_t j = colptr[c]; j < colptr[c + 1]; ++j) s = __dadd_rn(s, val[entry[j]]);
    indeg[c] = s;
  }
}

// val[l] /= indeg[rowind[l]] (src/gooseberry_bin.c:2622-2630)
__global__ void pr_divide_kernel(uint32_t nnz, const uint32_t * __restrict__ rowind,
    const double * __restrict__ indeg, double * __restrict__ val) {
  for (uint32_t l = blockIdx.x * blockDim.x + threadIdx.x; l < nnz; l += gridDim.x * blockDim.x)
    val[l] = __ddiv_rn(val[l], indeg[rowind[l]]);
}

// Scratch of the normalisation, released together.
struct PrScratch {
  cudaStream_t s;
  std::vector<void *> p;
  explicit PrScratch(cudaStream_t st) : s(st) {}
  template <typename T>
  int get(T ** out, size_t count) {
    void * q = nullptr;
    GB_TRY(scratch_alloc(&q, std::max<size_t>(count, 1) * sizeof(T), s));
    p.push_back(q);
    *out = static_cast<T *>(q);
    return GOOSEBERRY_SUCCESS;
  }
  ~PrScratch() {
    for (void * q : p) scratch_free(q, s);
  }
};

// Normalise the device matrix's values in place.
int normalise_device(gb_csr & a, cudaStream_t st) {
  const uint32_t n = a.nrows, nnz = a.nnz;
  if (nnz == 0) return GOOSEBERRY_SUCCESS;
  double * val = static_cast<double *>(a.own_val64);
  GB_CHECK_INPUT(val != nullptr, "matrix holds no values of its own");
  PrScratch sc(st);
  uint32_t *iota, *keys, *entry, *count, *colptr;
  double * indeg;
  GB_TRY(sc.get(&iota, nnz));
  GB_TRY(sc.get(&keys, nnz));
  GB_TRY(sc.get(&entry, nnz));
  GB_TRY(sc.get(&count, static_cast<size_t>(n) + 1));
  GB_TRY(sc.get(&colptr, static_cast<size_t>(n) + 1));
  GB_TRY(sc.get(&indeg, n));
  int sms = 148;
  GB_TRY(sm_count_of_current_device(&sms));
  const int grid = sms * 8;
  int bits = 1;
  while (bits < 32 && (1ull << bits) < n) ++bits;
  size_t t_sort = 0, t_scan = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, t_sort, a.rowind, keys, iota, entry, nnz, 0, bits,
      st);
  cub::DeviceScan::ExclusiveSum(nullptr, t_scan, count, colptr, n + 1, st);
  unsigned char * tmp;
  GB_TRY(sc.get(&tmp, std::max(t_sort, t_scan)));
  GB_CUDA_TRY(cudaMemsetAsync(count, 0, (static_cast<size_t>(n) + 1) * 4, st));
  pr_iota_count_kernel<<<grid, kPrBlock, 0, st>>>(nnz, a.rowind, iota, count);
  GB_CUDA_TRY(cudaGetLastError());
  // stable: the entries of a column keep their (row) order
  GB_CUDA_TRY(cub::DeviceRadixSort::SortPairs(tmp, t_sort, a.rowind, keys, iota, entry, nnz, 0,
      bits, st));
  GB_CUDA_TRY(cub::DeviceScan::ExclusiveSum(tmp, t_scan, count, colptr, n + 1, st));
  pr_colsum_kernel<<<grid, kPrBlock, 0, st>>>(n, colptr, entry, val, indeg);
  GB_CUDA_TRY(cudaGetLastError());
  pr_divide_kernel<<<grid, kPrBlock, 0, st>>>(nnz, a.rowind, indeg, val);
  GB_CUDA_TRY(cudaGetLastError());
  GB_CUDA_TRY(cudaStreamSynchronize(st));
  return GOOSEBERRY_SUCCESS;
}

__global__ void pr_fill_kernel(size_t n, double * __restrict__ v, double value) {
  for (size_t k = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; k < n;
       k += static_cast<size_t>(gridDim.x) * blockDim.x)
    v[k] = value;
}

struct PrBuffers {
  double * rank = nullptr;
  double * out = nullptr;
  double * partial = nullptr;
  double * scal = nullptr;   // [0] dist, [1] err
  double * h_err = nullptr;  // pinned
  uint32_t * sinks = nullptr;
  cudaStream_t st = nullptr;
  gb_csr_t * a = nullptr;
  ~PrBuffers() {
    if (st) cudaStreamSynchronize(st);
    dev_free(rank);
    dev_free(out);
    dev_free(partial);
    dev_free(scal);
    dev_free(sinks);
    pinned_slot_free(h_err);
    if (a) gb_csr_destroy(a);
    if (st) cudaStreamDestroy(st);
  }
};

int pagerank_f64(dim_t n, const ind_t * rowptr, const dim_t * rowind, const double * rowval,
    double damping, double minerror, size_t niter, double * result, size_t * iterations,
    double * error) {
  GB_CHECK_INPUT(n > 0 && rowptr && result, "NULL array or empty graph");
  const uint32_t nnz = rowptr[n];
  GB_CHECK_INPUT(nnz == 0 || (rowind && rowval), "NULL array");
  GB_CHECK_INPUT(rowptr[0] == 0, "rowptr[0] must be 0");
  // the sinks: rows without entries (src/gooseberry_bin.c:2611-2618)
  std::vector<uint32_t> sinks;
  for (dim_t k = 0; k < n; ++k) {
    GB_CHECK_INPUT(rowptr[k + 1] >= rowptr[k], "rowptr decreases at row %u", k);
    if (rowptr[k] == rowptr[k + 1]) sinks.push_back(k);
  }
  // upload the raw values (gb_csr_create checks the column indices) and
  // normalise them on the device
  PrBuffers B;
  GB_CUDA_TRY(cudaStreamCreateWithFlags(&B.st, cudaStreamNonBlocking));
  GB_TRY(gb_csr_create(n, n, nnz, rowptr, rowind, rowval, nullptr, GB_CSR_VALUES_F64, B.st,
      &B.a));
  GB_TRY(normalise_device(*B.a, B.st));
  int sms = 148;
  GB_TRY(sm_count_of_current_device(&sms));
  const unsigned g = static_cast<unsigned>(std::max<size_t>(1, std::min<size_t>(
      (n + kPrBlock * 4 - 1) / (kPrBlock * 4), static_cast<size_t>(sms) * 4)));
  const unsigned gs = static_cast<unsigned>(std::max<size_t>(1, std::min<size_t>(
      (sinks.size() + kPrBlock * 4 - 1) / (kPrBlock * 4), static_cast<size_t>(sms) * 4)));
  GB_TRY(dev_alloc(&B.rank, n * sizeof(double)));
  GB_TRY(dev_alloc(&B.out, n * sizeof(double)));
  GB_TRY(dev_alloc(&B.partial, std::max(g, gs) * sizeof(double)));
  GB_TRY(dev_alloc(&B.scal, 2 * sizeof(double)));
  GB_CUDA_TRY(cudaMemsetAsync(B.scal, 0, 2 * sizeof(double), B.st));
  GB_TRY(pinned_slot_alloc(sizeof(double), reinterpret_cast<void **>(&B.h_err), nullptr));
  if (!sinks.empty()) {
    GB_TRY(dev_alloc(&B.sinks, sinks.size() * sizeof(uint32_t)));
    GB_CUDA_TRY(cudaMemcpyAsync(B.sinks, sinks.data(), sinks.size() * sizeof(uint32_t),
        cudaMemcpyHostToDevice, B.st));
  }
  pr_fill_kernel<<<g, kPrBlock, 0, B.st>>>(n, B.rank, 1.0 / n);
  GB_CUDA_TRY(cudaGetLastError());
  const double c = (1.0 - damping) / n;
  double * rank = B.rank;
  double * out = B.out;
  size_t i = 0;
  bool done = false;
  for (; niter == 0 || i < niter; ++i) {
    GB_TRY(launch_spmv_f64(*B.a, B.a->sched64, rank, out, 1, B.st));
    if (!sinks.empty()) {
      pr_sink_kernel<<<gs, kPrBlock, 0, B.st>>>(sinks.size(), B.sinks, rank, B.partial);
      pr_final_kernel<<<1, kPrBlock, 0, B.st>>>(gs, B.partial, B.scal);
    }
    const int check = (i % 10 == 0) ? 1 : 0;
    pr_update_kernel<<<g, kPrBlock, 0, B.st>>>(n, out, rank, damping, c, B.scal, check,
        B.partial);
    if (check) {
      pr_final_kernel<<<1, kPrBlock, 0, B.st>>>(g, B.partial, B.scal + 1);
      GB_CUDA_TRY(cudaMemcpyAsync(B.h_err, B.scal + 1, sizeof(double), cudaMemcpyDeviceToHost,
          B.st));
      GB_CUDA_TRY(cudaStreamSynchronize(B.st));
      if (*B.h_err <= minerror * minerror) {
        ++i;
        done = true;
        break;
      }
    }
    std::swap(rank, out);
  }
  GB_CUDA_TRY(cudaGetLastError());
  if (!done) {
    pr_diff_kernel<<<g, kPrBlock, 0, B.st>>>(n, rank, out, B.partial);
    pr_final_kernel<<<1, kPrBlock, 0, B.st>>>(g, B.partial, B.scal + 1);
    GB_CUDA_TRY(cudaMemcpyAsync(B.h_err, B.scal + 1, sizeof(double), cudaMemcpyDeviceToHost,
        B.st));
  }
  GB_CUDA_TRY(cudaMemcpyAsync(result, out, n * sizeof(double), cudaMemcpyDeviceToHost, B.st));
  GB_CUDA_TRY(cudaStreamSynchronize(B.st));
  if (iterations) *iterations = i;
  if (error) *error = std::sqrt(*B.h_err);
  return GOOSEBERRY_SUCCESS;
}

}  // namespace
}  // namespace gb

extern "C" {

int gooseberry_pagerank_f64(dim_t n, const ind_t * rowptr, const dim_t * rowind,
    const double * rowval, double damping, double minerror, size_t niter, double * rank,
    size_t * iterations, double * error) {
  return gb::pagerank_f64(n, rowptr, rowind, rowval, damping, minerror, niter, rank,
      iterations, error);
}

// Float ABI: the iteration runs in double on the device (never less accurate
// than the reference's float build) and rank is rounded back to float.
int gooseberry_pagerank(dim_t n, const ind_t * rowptr, const dim_t * rowind,
    const float * rowval, float damping, float minerror, size_t niter, float * rank,
    size_t * iterations, double * error) {
  GB_CHECK_INPUT(n > 0 && rowptr && rank, "NULL array or empty graph");
  const uint32_t nnz = rowptr[n];
  GB_CHECK_INPUT(nnz == 0 || rowval, "NULL array");
  std::vector<double> v(rowval, rowval + nnz), r(n);
  GB_TRY(gb::pagerank_f64(n, rowptr, rowind, v.data(), damping, minerror, niter, r.data(),
      iterations, error));
  for (dim_t k = 0; k < n; ++k) rank[k] = static_cast<float>(r[k]);
  return GOOSEBERRY_SUCCESS;
}

}  // extern "C"
