// codec.cu -- lossless compressed copies of a matrix's entries for the row
// schedule (ColD16, ValCode8, exact ValPlain<float>; spmv_tiles.cuh).
//
// Built once per solver from the device matrix:
//   * columns: col - row as int16 when every entry lies within 32767 of the
//     diagonal (banded and stencil matrices);
//   * values: an 8-bit code into a table of distinct values when the matrix
//     has at most 256 of them (constant-coefficient operators), else a float
//     copy when every double is exactly a float, else nothing.
// The distinct values are collected in a 1024-slot open-addressing hash set
// in device memory (read before compare-and-swap, so repeated values cost a
// cached read, not an atomic); the set gives up past 256 values.
#include <algorithm>
#include <cstring>
#include <vector>

#include "gb_internal.h"
#include "spmv_tiles.cuh"

namespace gb {
namespace {

constexpr unsigned kSetSlots = 1024;
constexpr unsigned kMaxCodes = 256;
// An empty slot holds this NaN bit pattern; a matrix holding it is not coded.
constexpr unsigned long long kEmpty = 0x7ff4a5a5a5a5a5a5ull;

__device__ __forceinline__ unsigned slot_of(unsigned long long bits) {
  bits ^= bits >> 33;
  bits *= 0xff51afd7ed558ccdull;
  bits ^= bits >> 33;
  return static_cast<unsigned>(bits) & (kSetSlots - 1);
}

// col16[k] = col - row; *bad = 1 if some entry is farther than 32767.
__global__ void codec_delta_kernel(const uint32_t * __restrict__ rowptr,
    const uint32_t * __restrict__ rowind, uint32_t n, int16_t * __restrict__ col16,
    unsigned * bad) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    if (*reinterpret_cast<volatile unsigned *>(bad)) return;
    const uint32_t e = rowptr[i + 1];
    for (uint32_t k = rowptr[i]; k < e; ++k) {
      const long long d = static_cast<long long>(rowind[k]) - static_cast<long long>(i);
      if (d < -32767 || d > 32767) {
        atomicExch(bad, 1u);
        return;
      }
      col16[k] = static_cast<int16_t>(d);
    }
  }
}

// Distinct values into the hash set; *bad = 1 past kMaxCodes values.
__global__ void codec_set_kernel(const double * __restrict__ val, uint32_t nnz,
    unsigned long long * keys, unsigned * count, unsigned * bad) {
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < nnz; k += gridDim.x * blockDim.x) {
    if ((k & 255u) == 0 && *reinterpret_cast<volatile unsigned *>(bad)) return;
    const unsigned long long bits = __double_as_longlong(__ldg(val + k));
    if (bits == kEmpty) {
      atomicExch(bad, 1u);
      return;
    }
    unsigned h = slot_of(bits);
    bool placed = false;
    for (unsigned probe = 0; probe < kSetSlots; ++probe, h = (h + 1) & (kSetSlots - 1)) {
      unsigned long long cur = *reinterpret_cast<volatile unsigned long long *>(keys + h);
      if (cur == bits) {
        placed = true;
        break;
      }
      if (cur == kEmpty) {
        cur = atomicCAS(keys + h, kEmpty, bits);
        if (cur == kEmpty) {
          if (atomicAdd(count, 1u) >= kMaxCodes) atomicExch(bad, 1u);
          placed = true;
          break;
        }
        if (cur == bits) {
          placed = true;
          break;
        }
      }
    }
    if (!placed) {
      atomicExch(bad, 1u);
      return;
    }
  }
}

// code8[k] = code of val[k] (every value is in the set).
__global__ void codec_encode_kernel(const double * __restrict__ val, uint32_t nnz,
    const unsigned long long * __restrict__ keys, const uint8_t * __restrict__ slot_code,
    uint8_t * __restrict__ code8) {
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < nnz; k += gridDim.x * blockDim.x) {
    const unsigned long long bits = __double_as_longlong(__ldg(val + k));
    unsigned h = slot_of(bits);
    for (unsigned probe = 0; probe < kSetSlots; ++probe, h = (h + 1) & (kSetSlots - 1))
      if (__ldg(keys + h) == bits) break;
    code8[k] = __ldg(slot_code + h);
  }
}

// out[k] = (float)val[k]; *bad = 1 if some value is not exactly a float.
__global__ void codec_f32_kernel(const double * __restrict__ val, uint32_t nnz,
    float * __restrict__ out, unsigned * bad) {
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < nnz; k += gridDim.x * blockDim.x) {
    const double v = __ldg(val + k);
    const float f = __double2float_rn(v);
    if (static_cast<double>(f) != v) {
      atomicExch(bad, 1u);
      return;
    }
    out[k] = f;
  }
}

// ---- row patterns (ColPat8) ---------------------------------------------------

// Hash of a row's column offsets from the diagonal (offsets taken mod 2^32, so
// row + offset recovers the column exactly); never the empty-slot value.
__device__ __forceinline__ unsigned long long pattern_hash(const uint32_t * __restrict__ rowind,
    uint32_t b, uint32_t e, uint32_t row) {
  unsigned long long h = 0x9e3779b97f4a7c15ull * (e - b + 1);
  for (uint32_t k = b; k < e; ++k) {
    const unsigned long long d = __ldg(rowind + k) - row;
    h ^= d + 0x9e3779b97f4a7c15ull + (h << 6) + (h >> 2);
    h *= 0xff51afd7ed558ccdull;
    h ^= h >> 33;
  }
  return h == kEmpty ? h ^ 1ull : h;
}

// Distinct row patterns into the hash set, with a row holding each; *bad = 1
// past kMaxCodes patterns or for a row longer than kPatMax.
__global__ void codec_pattern_set_kernel(const uint32_t * __restrict__ rowptr,
    const uint32_t * __restrict__ rowind, uint32_t n, unsigned long long * keys,
    uint32_t * rep, unsigned * count, unsigned * bad) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    if ((i & 255u) == 0 && *reinterpret_cast<volatile unsigned *>(bad)) return;
    const uint32_t b = __ldg(rowptr + i), e = __ldg(rowptr + i + 1);
    if (e - b > static_cast<uint32_t>(kPatMax)) {
      atomicExch(bad, 1u);
      return;
    }
    const unsigned long long h0 = pattern_hash(rowind, b, e, i);
    unsigned h = slot_of(h0);
    bool placed = false;
    for (unsigned probe = 0; probe < kSetSlots; ++probe, h = (h + 1) & (kSetSlots - 1)) {
      unsigned long long cur = *reinterpret_cast<volatile unsigned long long *>(keys + h);
      if (cur == h0) {
        placed = true;
        break;
      }
      if (cur == kEmpty) {
        cur = atomicCAS(keys + h, kEmpty, h0);
        if (cur == kEmpty) {
          rep[h] = i;
          if (atomicAdd(count, 1u) >= kMaxCodes) atomicExch(bad, 1u);
          placed = true;
          break;
        }
        if (cur == h0) {
          placed = true;
          break;
        }
      }
    }
    if (!placed) {
      atomicExch(bad, 1u);
      return;
    }
  }
}

// off[code * kPatMax + j] = offset j of the row that holds each pattern.
__global__ void codec_pattern_table_kernel(const uint32_t * __restrict__ rowptr,
    const uint32_t * __restrict__ rowind, const unsigned long long * __restrict__ keys,
    const uint32_t * __restrict__ rep, const uint8_t * __restrict__ slot_code,
    int32_t * __restrict__ off) {
  const unsigned h = blockIdx.x * blockDim.x + threadIdx.x;
  if (h >= kSetSlots || keys[h] == kEmpty) return;
  const uint32_t row = rep[h], b = rowptr[row], e = rowptr[row + 1];
  const uint32_t c = slot_code[h];
  // pattern rows hold at most kPatMax - 1 entries: the last slot holds the
  // pattern's length (rows that use it need no rowptr for their length)
  for (int j = 0; j + 1 < kPatMax; ++j)
    off[c * kPatMax + j] = b + j < e ? static_cast<int32_t>(rowind[b + j] - row) : 0;
  off[c * kPatMax + kPatMax - 1] = static_cast<int32_t>(e - b);
}

// code8[i] = pattern of row i; then every column is checked against it
// (*bad = 1 on a mismatch, which only a hash collision could cause).
__global__ void codec_pattern_encode_kernel(const uint32_t * __restrict__ rowptr,
    const uint32_t * __restrict__ rowind, uint32_t n, const unsigned long long * __restrict__ keys,
    const uint8_t * __restrict__ slot_code, const int32_t * __restrict__ off,
    uint8_t * __restrict__ code8, unsigned * bad) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint32_t b = __ldg(rowptr + i), e = __ldg(rowptr + i + 1);
    const unsigned long long h0 = pattern_hash(rowind, b, e, i);
    unsigned h = slot_of(h0);
    for (unsigned probe = 0; probe < kSetSlots; ++probe, h = (h + 1) & (kSetSlots - 1))
      if (__ldg(keys + h) == h0) break;
    const uint32_t c = __ldg(slot_code + h);
    code8[i] = static_cast<uint8_t>(c);
    if (e - b != static_cast<uint32_t>(__ldg(off + c * kPatMax + kPatMax - 1))) atomicExch(bad, 1u);
    for (uint32_t k = b; k < e; ++k)
      if (__ldg(rowind + k) != i + static_cast<uint32_t>(__ldg(off + c * kPatMax + (k - b))))
        atomicExch(bad, 1u);
  }
}

int grid_of(const gb_csr & a, size_t items) {
  const size_t want = (items + 255) / 256;
  return static_cast<int>(std::max<size_t>(1, std::min<size_t>(want,
      static_cast<size_t>(std::max(a.sm_count, 1)) * 8)));
}

int read_flag(const unsigned * d, unsigned * h, cudaStream_t s) {
  GB_CUDA_TRY(cudaMemcpyAsync(h, d, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
  GB_CUDA_TRY(cudaStreamSynchronize(s));
  return GOOSEBERRY_SUCCESS;
}

int build_values(const gb_csr & a, RowCodec * c, unsigned * flags, cudaStream_t s) {
  const uint32_t nnz = a.nnz;
  // distinct values
  unsigned long long * keys = nullptr;
  GB_TRY(scratch_alloc(reinterpret_cast<void **>(&keys), kSetSlots * 8 + 64, s));
  unsigned * cnt = reinterpret_cast<unsigned *>(keys + kSetSlots);
  std::vector<unsigned long long> hk(kSetSlots, kEmpty);
  int rc = GOOSEBERRY_SUCCESS;
  unsigned bad = 1, count = 0;
  auto done = [&](int r) {
    scratch_free(keys, s);
    return r;
  };
  if (cudaMemcpyAsync(keys, hk.data(), kSetSlots * 8, cudaMemcpyHostToDevice, s) != cudaSuccess ||
      cudaMemsetAsync(cnt, 0, 8, s) != cudaSuccess || cudaMemsetAsync(flags, 0, 4, s) != cudaSuccess)
    return done(GOOSEBERRY_ERROR_UNKNOWN);
  codec_set_kernel<<<grid_of(a, nnz), 256, 0, s>>>(a.val64, nnz, keys, cnt, flags);
  if ((rc = read_flag(flags, &bad, s)) != GOOSEBERRY_SUCCESS) return done(rc);
  if (!bad) {
    if (cudaMemcpyAsync(hk.data(), keys, kSetSlots * 8, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaMemcpyAsync(&count, cnt, 4, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
      return done(GOOSEBERRY_ERROR_UNKNOWN);
    std::vector<uint8_t> slot_code(kSetSlots, 0);
    std::vector<double> table;
    for (unsigned h = 0; h < kSetSlots; ++h) {
      if (hk[h] == kEmpty) continue;
      slot_code[h] = static_cast<uint8_t>(table.size());
      double v;
      std::memcpy(&v, &hk[h], sizeof v);
      table.push_back(v);
    }
    if (table.size() <= kMaxCodes && table.size() == count) {
      uint8_t * d_slot = nullptr;
      if ((rc = dev_alloc(&c->code8, std::max<size_t>(nnz, 1))) != GOOSEBERRY_SUCCESS ||
          (rc = dev_alloc(&c->table, std::max<size_t>(table.size(), 1) * 8)) !=
              GOOSEBERRY_SUCCESS ||
          (rc = scratch_alloc(reinterpret_cast<void **>(&d_slot), kSetSlots, s)) !=
              GOOSEBERRY_SUCCESS)
        return done(rc);
      c->ntable = static_cast<uint32_t>(table.size());
      cudaError_t e = cudaMemcpyAsync(c->table, table.data(), table.size() * 8,
          cudaMemcpyHostToDevice, s);
      if (e == cudaSuccess)
        e = cudaMemcpyAsync(d_slot, slot_code.data(), kSetSlots, cudaMemcpyHostToDevice, s);
      if (e == cudaSuccess) {
        codec_encode_kernel<<<grid_of(a, nnz), 256, 0, s>>>(a.val64, nnz, keys, d_slot, c->code8);
        e = cudaStreamSynchronize(s);
      }
      scratch_free(d_slot, s);
      if (e != cudaSuccess) {
        set_error("value coding failed: %s", cudaGetErrorString(e));
        return done(GOOSEBERRY_ERROR_UNKNOWN);
      }
      return done(GOOSEBERRY_SUCCESS);
    }
  }
  // exact float copy
  float * f = nullptr;
  if ((rc = dev_alloc(&f, std::max<size_t>(nnz, 1) * 4)) != GOOSEBERRY_SUCCESS) return done(rc);
  if (cudaMemsetAsync(flags, 0, 4, s) != cudaSuccess) return done(GOOSEBERRY_ERROR_UNKNOWN);
  codec_f32_kernel<<<grid_of(a, nnz), 256, 0, s>>>(a.val64, nnz, f, flags);
  if ((rc = read_flag(flags, &bad, s)) != GOOSEBERRY_SUCCESS) return done(rc);
  if (bad) {
    dev_free(f);
  } else {
    c->val32 = f;
  }
  return done(GOOSEBERRY_SUCCESS);
}

}  // namespace

int build_row_patterns(const gb_csr & a, RowPatterns * out, cudaStream_t s) {
  *out = RowPatterns{};
  // rows of at most 7 entries: the row loop's register stage (row_stage_for)
  // then holds a whole row, and pattern rows need no long-row tail
  if (a.nrows == 0 || a.plan.max_row > 7u) return GOOSEBERRY_SUCCESS;
  // set: keys, representative rows, count + flag
  unsigned long long * keys = nullptr;
  GB_TRY(scratch_alloc(reinterpret_cast<void **>(&keys), kSetSlots * 12 + kSetSlots + 64, s));
  uint32_t * rep = reinterpret_cast<uint32_t *>(keys + kSetSlots);
  uint8_t * d_slot = reinterpret_cast<uint8_t *>(rep + kSetSlots);
  unsigned * cnt = reinterpret_cast<unsigned *>(d_slot + kSetSlots);
  unsigned * flags = cnt + 2;
  std::vector<unsigned long long> hk(kSetSlots, kEmpty);
  unsigned bad = 1, count = 0;
  int rc = GOOSEBERRY_SUCCESS;
  auto done = [&](int r) {
    scratch_free(keys, s);
    if (r != GOOSEBERRY_SUCCESS || bad) {
      if (out->code8) dev_free(out->code8);
      if (out->off) dev_free(out->off);
      *out = RowPatterns{};
    }
    return r;
  };
  if (cudaMemcpyAsync(keys, hk.data(), kSetSlots * 8, cudaMemcpyHostToDevice, s) != cudaSuccess ||
      cudaMemsetAsync(cnt, 0, 16, s) != cudaSuccess)
    return done(GOOSEBERRY_ERROR_UNKNOWN);
  codec_pattern_set_kernel<<<grid_of(a, a.nrows), 256, 0, s>>>(a.rowptr, a.rowind, a.nrows, keys,
      rep, cnt, flags);
  if ((rc = read_flag(flags, &bad, s)) != GOOSEBERRY_SUCCESS || bad) return done(rc);
  if (cudaMemcpyAsync(hk.data(), keys, kSetSlots * 8, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaMemcpyAsync(&count, cnt, 4, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return done(GOOSEBERRY_ERROR_UNKNOWN);
  std::vector<uint8_t> slot_code(kSetSlots, 0);
  uint32_t np = 0;
  for (unsigned h = 0; h < kSetSlots; ++h)
    if (hk[h] != kEmpty) slot_code[h] = static_cast<uint8_t>(np++);
  bad = np != count || np > kMaxCodes;
  if (bad) return done(GOOSEBERRY_SUCCESS);
  if ((rc = dev_alloc(&out->code8, a.nrows)) != GOOSEBERRY_SUCCESS ||
      (rc = dev_alloc(&out->off, static_cast<size_t>(std::max(np, 1u)) * kPatMax * 4)) !=
          GOOSEBERRY_SUCCESS)
    return done(rc);
  out->npat = np;
  if (cudaMemcpyAsync(d_slot, slot_code.data(), kSetSlots, cudaMemcpyHostToDevice, s) !=
          cudaSuccess ||
      cudaMemsetAsync(flags, 0, 4, s) != cudaSuccess)
    return done(GOOSEBERRY_ERROR_UNKNOWN);
  codec_pattern_table_kernel<<<kSetSlots / 256, 256, 0, s>>>(a.rowptr, a.rowind, keys, rep,
      d_slot, out->off);
  codec_pattern_encode_kernel<<<grid_of(a, a.nrows), 256, 0, s>>>(a.rowptr, a.rowind, a.nrows,
      keys, d_slot, out->off, out->code8, flags);
  if ((rc = read_flag(flags, &bad, s)) != GOOSEBERRY_SUCCESS) return done(rc);
  return done(GOOSEBERRY_SUCCESS);
}

void free_row_patterns(RowPatterns & p) {
  if (p.code8) dev_free(p.code8);
  if (p.off) dev_free(p.off);
  p = RowPatterns{};
}

int row_stage_for(const gb_csr & a) {
  return a.plan.max_row <= 5 ? 5 : (a.plan.max_row <= 7 ? 7 : 6);
}

int build_col16(const gb_csr & a, int16_t ** out, cudaStream_t s) {
  *out = nullptr;
  if (a.nnz == 0) return GOOSEBERRY_SUCCESS;
  unsigned * flags = nullptr;
  GB_TRY(scratch_alloc(reinterpret_cast<void **>(&flags), 16, s));
  unsigned bad = 1;
  int16_t * col16 = nullptr;
  int rc = dev_alloc(&col16, static_cast<size_t>(a.nnz) * 2);
  if (rc == GOOSEBERRY_SUCCESS && cudaMemsetAsync(flags, 0, 4, s) != cudaSuccess)
    rc = GOOSEBERRY_ERROR_UNKNOWN;
  if (rc == GOOSEBERRY_SUCCESS) {
    codec_delta_kernel<<<grid_of(a, a.nrows), 256, 0, s>>>(a.rowptr, a.rowind, a.nrows, col16,
        flags);
    rc = read_flag(flags, &bad, s);
  }
  scratch_free(flags, s);
  if (rc != GOOSEBERRY_SUCCESS || bad) {
    if (col16) dev_free(col16);
    return rc;
  }
  *out = col16;
  return GOOSEBERRY_SUCCESS;
}

int build_row_codec(const gb_csr & a, RowCodec * c, cudaStream_t s) {
  *c = RowCodec{};
  c->stage = row_stage_for(a);
  if (a.nnz == 0 || !a.val64) return GOOSEBERRY_SUCCESS;
  int rc = build_col16(a, &c->col16, s);
  unsigned * flags = nullptr;
  if (rc == GOOSEBERRY_SUCCESS)
    rc = scratch_alloc(reinterpret_cast<void **>(&flags), 16, s);
  if (rc == GOOSEBERRY_SUCCESS) {
    rc = build_values(a, c, flags, s);
    scratch_free(flags, s);
  }
  if (rc != GOOSEBERRY_SUCCESS) free_row_codec(*c);
  return rc;
}

void free_row_codec(RowCodec & c) {
  if (c.col16) dev_free(c.col16);
  if (c.code8) dev_free(c.code8);
  if (c.table) dev_free(c.table);
  if (c.val32) dev_free(c.val32);
  const int stage = c.stage;
  c = RowCodec{};
  c.stage = stage;
}

}  // namespace gb
