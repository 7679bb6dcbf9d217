// serve.cu -- batched CG serving: many uneven solves resident at once,
// continuous batching, admission by device-memory footprint.
//
// Reference: one cgd call (src/cgd.c:40-129) runs at a time from the CLI
// (src/gooseberry_bin.c:2078-2091).  Here every resident solve owns a slot:
// its CSR matrix and Krylov vectors live in one device pool (first-fit
// allocator, bounded by pool_bytes), and all slots advance together.
//
// Work list: every slot's rows are cut into row-aligned tiles of at most
// kTileItems rows + nonzeros; the tiles of all resident slots form ONE global
// list.  Each kernel is persistent over that list, one warp per tile at a
// time, lane per row (rows hold at most 255 nonzeros).  A tile leaves a
// partial sum; the warp that finishes a slot's last tile (per-slot atomic
// ticket) adds the slot's partials in tile order (deterministic) and updates
// that slot's alpha / beta / stop decision.  So one launch advances a 1k-row
// and a 262k-row solve by one phase each, and the launch cost is shared by
// the whole batch.
//
// Per step (one graph replay): init of newly admitted slots, then
// iters_per_step x { A: SpMV + direction update + p.Ap;  B: x/y, r update +
// r.r;  R (mixed only): reliable FP64 residual update }.  Slot state lives in
// device memory, so the captured graph never changes; between steps the host
// reads the slot table back, retires finished solves (x copied out), admits
// queued requests into freed slots and memory, rebuilds the tile list and
// uploads the table.
//
// Mixed mode is the algorithm of cg_mixed.cu (FP32 values and vectors, FP64
// dots, reliable FP64 updates, convergence on the true residual); F64 mode
// is plain CG like cg.cu (convergence on the recurrence residual, as the
// reference).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <deque>
#include <map>
#include <vector>

#include "gb_internal.h"
#include "spmv_tiles.cuh"
#include "cg_common.cuh"

namespace gb {
namespace {

constexpr uint32_t kTileItems = 256;  // rows + nonzeros per warp tile
constexpr int kSrvBlock = 256;
constexpr int kSrvWarps = kSrvBlock / 32;
constexpr double kSrvDelta = 0.1;     // reliable update trigger (see cg_mixed.cu)
constexpr size_t kMaxTiles = 2u << 20;

struct SrvTile {
  uint32_t slot;
  uint32_t row_begin;
  uint32_t row_count;
  uint32_t pad;
};

struct SrvSlot {
  const uint32_t * rowptr;
  const uint32_t * rowind;
  const double * val64;
  const float * val32;
  const double * b;
  double * x0;
  double * x1;
  void * y;   // T[n] (mixed only)
  void * r;   // T[n]
  void * p0;  // T[n]
  void * p1;  // T[n]
  void * ap;  // T[n]
  uint32_t n, ntiles, tile0, pad;
  double rr_hat, rr_hat_old, alpha, beta, tol, tol_rel, bnorm, rmax, rr_true;
  unsigned long long iter, niter, refinements;
  int live;     // slot holds a solve
  int init;     // needs the init kernel
  int done;     // finished (converged / maxiter / breakdown / nonfinite)
  int status;
  int update;   // reliable update pending
  int final;    // the update is the last one (iteration limit)
  int y_reset;
  int xpar;
  unsigned ticket_a, ticket_b, ticket_r, ticket_i;
};

struct SrvDev {
  SrvSlot * slots;
  const SrvTile * tiles;
  const uint32_t * ntiles;  // device word: tiles in the list
  double * pa;
  double * pb;
  double * pr;
  double * pi0;
  double * pi1;
};

__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// True in every lane of the warp that completes the slot's last tile.
__device__ __forceinline__ bool slot_arrive(unsigned * ticket, unsigned ntiles, int lane) {
  unsigned tk = 0;
  __syncwarp();
  if (lane == 0) {
    __threadfence();
    tk = atomicAdd(ticket, 1u);
  }
  tk = __shfl_sync(0xffffffffu, tk, 0);
  return tk == ntiles - 1;
}

// Sum of part[t0 .. t0+nt) in a fixed order, in every lane.
__device__ __forceinline__ double slot_sum(const double * part, uint32_t t0, uint32_t nt,
    int lane) {
  __threadfence();
  double acc = 0.0;
  for (uint32_t i = lane; i < nt; i += 32) acc += __ldcg(part + t0 + i);
  return warp_sum_d(acc);
}

template <typename T>
__device__ __forceinline__ T ldv(const T * p, uint64_t pol) { return ld_keep(p, pol); }

// ---- init: x = 0, r = b, p = 0 ---------------------------------------------------

template <typename T, bool MIXED>
__global__ void __launch_bounds__(kSrvBlock) srv_init_kernel(const SrvDev d) {
  pdl_wait_and_release();
  const int lane = threadIdx.x & 31;
  const uint32_t nt = *d.ntiles;
  const uint32_t gw = blockIdx.x * kSrvWarps + (threadIdx.x >> 5);
  for (uint32_t t = gw; t < nt; t += gridDim.x * kSrvWarps) {
    const SrvTile tl = d.tiles[t];
    SrvSlot & S = d.slots[tl.slot];
    if (!S.live || !S.init) continue;
    T * r = static_cast<T *>(S.r);
    T * p0 = static_cast<T *>(S.p0);
    double sb = 0.0, sr = 0.0;
    for (uint32_t q = lane; q < tl.row_count; q += 32) {
      const uint32_t i = tl.row_begin + q;
      const double bv = S.b[i];
      const T rv = static_cast<T>(bv);
      S.x0[i] = 0.0;
      r[i] = rv;
      p0[i] = T(0);
      sb += bv * bv;
      sr += static_cast<double>(rv) * static_cast<double>(rv);
    }
    sb = warp_sum_d(sb);
    sr = warp_sum_d(sr);
    if (lane == 0) {
      d.pi0[t] = sb;
      d.pi1[t] = sr;
    }
    if (slot_arrive(&S.ticket_i, S.ntiles, lane)) {
      const double bb = slot_sum(d.pi0, S.tile0, S.ntiles, lane);
      const double rr = slot_sum(d.pi1, S.tile0, S.ntiles, lane);
      if (lane == 0) {
        S.ticket_i = 0;
        S.bnorm = sqrt(bb);
        S.tol = S.tol_rel * S.bnorm;
        S.rr_true = bb;
        S.rr_hat = MIXED ? rr : bb;
        S.rr_hat_old = S.rr_hat;
        S.rmax = sqrt(S.rr_hat);
        S.alpha = 0.0;
        S.beta = 0.0;
        S.iter = 0;
        S.refinements = 0;
        S.xpar = 0;
        S.y_reset = 1;
        S.update = 0;
        S.final = 0;
        S.status = GB_CG_MAXITER;
        S.init = 0;
        if (bb == 0.0) {
          S.done = 1;
          S.status = GB_CG_CONVERGED;
        } else if (!(bb == bb) || isinf(bb)) {
          S.done = 1;
          S.status = GB_CG_NONFINITE;
        }
      }
    }
  }
}

// ---- A: SpMV + direction update + p.Ap --------------------------------------------

template <typename T>
__device__ __forceinline__ const T * values_of(const SrvSlot & S);
template <>
__device__ __forceinline__ const float * values_of<float>(const SrvSlot & S) { return S.val32; }
template <>
__device__ __forceinline__ const double * values_of<double>(const SrvSlot & S) {
  return S.val64;
}

template <typename T>
__global__ void __launch_bounds__(kSrvBlock) srv_a_kernel(const SrvDev d) {
  pdl_wait_and_release();
  const int lane = threadIdx.x & 31;
  const uint64_t pol = policy_evict_last();
  const uint32_t nt = *d.ntiles;
  const uint32_t gw = blockIdx.x * kSrvWarps + (threadIdx.x >> 5);
  for (uint32_t t = gw; t < nt; t += gridDim.x * kSrvWarps) {
    const SrvTile tl = d.tiles[t];
    SrvSlot & S = d.slots[tl.slot];
    if (!S.live || S.init || S.done) continue;
    const T beta = static_cast<T>(S.beta);
    const bool par = (S.iter & 1ull) != 0;
    const T * pold = static_cast<const T *>(par ? S.p1 : S.p0);
    T * pnew = static_cast<T *>(par ? S.p0 : S.p1);
    const T * r = static_cast<const T *>(S.r);
    T * ap = static_cast<T *>(S.ap);
    const T * val = values_of<T>(S);
    const uint32_t * rowptr = S.rowptr;
    const uint32_t * rowind = S.rowind;
    double part = 0.0;
    for (uint32_t q = lane; q < tl.row_count; q += 32) {
      const uint32_t i = tl.row_begin + q;
      const uint32_t b = __ldg(rowptr + i), e = __ldg(rowptr + i + 1);
      const T ri = r[i], pi = pold[i];
      T sum = T(0);
      for (uint32_t base = b; base < e; base += 8) {
        uint32_t c[8];
        T v[8], g[8];
#pragma unroll
        for (int j = 0; j < 8; ++j)
          if (base + j < e) {
            c[j] = __ldg(rowind + base + j);
            v[j] = __ldg(val + base + j);
          }
#pragma unroll
        for (int j = 0; j < 8; ++j)
          if (base + j < e) g[j] = fma(beta, ldv(pold + c[j], pol), ldv(r + c[j], pol));
#pragma unroll
        for (int j = 0; j < 8; ++j)
          if (base + j < e) sum = fma(v[j], g[j], sum);
      }
      ap[i] = sum;
      const T pn = fma(beta, pi, ri);
      pnew[i] = pn;
      part += static_cast<double>(pn) * static_cast<double>(sum);
    }
    part = warp_sum_d(part);
    if (lane == 0) d.pa[t] = part;
    if (slot_arrive(&S.ticket_a, S.ntiles, lane)) {
      const double pap = slot_sum(d.pa, S.tile0, S.ntiles, lane);
      if (lane == 0) {
        S.ticket_a = 0;
        const double rr = S.rr_hat;
        if (!(pap > 0.0)) {
          S.done = 1;
          S.status = (pap == pap && rr == rr) ? GB_CG_BREAKDOWN : GB_CG_NONFINITE;
        } else {
          S.alpha = rr / pap;
        }
      }
    }
  }
}

// ---- B: solution / residual update, r.r, stop or update decision --------------------

template <typename T, bool MIXED>
__global__ void __launch_bounds__(kSrvBlock) srv_b_kernel(const SrvDev d) {
  pdl_wait_and_release();
  const int lane = threadIdx.x & 31;
  const uint32_t nt = *d.ntiles;
  const uint32_t gw = blockIdx.x * kSrvWarps + (threadIdx.x >> 5);
  for (uint32_t t = gw; t < nt; t += gridDim.x * kSrvWarps) {
    const SrvTile tl = d.tiles[t];
    SrvSlot & S = d.slots[tl.slot];
    if (!S.live || S.init || S.done) continue;
    const T alpha = static_cast<T>(S.alpha);
    const bool fresh = S.y_reset != 0;
    const bool par = (S.iter & 1ull) != 0;
    const T * pnew = static_cast<const T *>(par ? S.p0 : S.p1);
    const T * ap = static_cast<const T *>(S.ap);
    T * r = static_cast<T *>(S.r);
    T * y = static_cast<T *>(S.y);
    double part = 0.0;
    for (uint32_t q = lane; q < tl.row_count; q += 32) {
      const uint32_t i = tl.row_begin + q;
      const T pn = pnew[i], av = ap[i], rv = r[i];
      if (MIXED) {
        const T yv = fresh ? T(0) : y[i];
        y[i] = fma(alpha, pn, yv);
      } else {
        S.x0[i] = fma(static_cast<double>(alpha), static_cast<double>(pn), S.x0[i]);
      }
      const T rn = fma(-alpha, av, rv);
      r[i] = rn;
      part += static_cast<double>(rn) * static_cast<double>(rn);
    }
    part = warp_sum_d(part);
    if (lane == 0) d.pb[t] = part;
    if (slot_arrive(&S.ticket_b, S.ntiles, lane)) {
      const double rr = slot_sum(d.pb, S.tile0, S.ntiles, lane);
      if (lane == 0) {
        S.ticket_b = 0;
        S.y_reset = 0;
        S.rr_hat_old = S.rr_hat;
        S.beta = rr / S.rr_hat;
        S.rr_hat = rr;
        const unsigned long long it = S.iter + 1;
        S.iter = it;
        const double rnorm = sqrt(rr);
        S.rmax = fmax(S.rmax, rnorm);
        if (!(rnorm == rnorm) || isinf(rnorm)) {
          S.done = 1;
          S.status = GB_CG_NONFINITE;
        } else if (MIXED) {
          const bool last = S.niter && it >= S.niter;
          if (rnorm <= S.tol || rnorm < kSrvDelta * S.rmax || last) {
            S.update = 1;
            S.final = last ? 1 : 0;
          }
        } else {
          if (rnorm <= S.tol) {
            S.done = 1;
            S.status = GB_CG_CONVERGED;
            S.rr_true = rr;
          } else if (S.niter && it >= S.niter) {
            S.done = 1;
            S.status = GB_CG_MAXITER;
            S.rr_true = rr;
          }
        }
      }
    }
  }
}

// ---- R: reliable update (mixed) ---------------------------------------------------

__global__ void __launch_bounds__(kSrvBlock) srv_r_kernel(const SrvDev d) {
  pdl_wait_and_release();
  const int lane = threadIdx.x & 31;
  const uint64_t pol = policy_evict_last();
  const uint32_t nt = *d.ntiles;
  const uint32_t gw = blockIdx.x * kSrvWarps + (threadIdx.x >> 5);
  for (uint32_t t = gw; t < nt; t += gridDim.x * kSrvWarps) {
    const SrvTile tl = d.tiles[t];
    SrvSlot & S = d.slots[tl.slot];
    if (!S.live || S.init || S.done || !S.update) continue;
    const bool use_y = S.y_reset == 0;
    const double * xold = S.xpar ? S.x1 : S.x0;
    double * xnew = S.xpar ? S.x0 : S.x1;
    const float * y = static_cast<const float *>(S.y);
    float * r32 = static_cast<float *>(S.r);
    double part = 0.0;
    for (uint32_t q = lane; q < tl.row_count; q += 32) {
      const uint32_t i = tl.row_begin + q;
      const uint32_t b = __ldg(S.rowptr + i), e = __ldg(S.rowptr + i + 1);
      double sum = 0.0;
      for (uint32_t k = b; k < e; ++k) {
        const uint32_t c = __ldg(S.rowind + k);
        const double xc = ldv(xold + c, pol) + (use_y ? static_cast<double>(ldv(y + c, pol)) : 0.0);
        sum = fma(__ldg(S.val64 + k), xc, sum);
      }
      xnew[i] = xold[i] + (use_y ? static_cast<double>(y[i]) : 0.0);
      const double rt = S.b[i] - sum;
      r32[i] = static_cast<float>(rt);
      part += rt * rt;
    }
    part = warp_sum_d(part);
    if (lane == 0) d.pr[t] = part;
    if (slot_arrive(&S.ticket_r, S.ntiles, lane)) {
      const double tot = slot_sum(d.pr, S.tile0, S.ntiles, lane);
      if (lane == 0) {
        S.ticket_r = 0;
        S.rr_true = tot;
        S.refinements += 1;
        S.xpar ^= 1;
        S.y_reset = 1;
        S.update = 0;
        const double rnorm = sqrt(tot);
        if (!(rnorm == rnorm) || isinf(rnorm)) {
          S.done = 1;
          S.status = GB_CG_NONFINITE;
        } else if (rnorm <= S.tol) {
          S.done = 1;
          S.status = GB_CG_CONVERGED;
        } else if (S.final) {
          S.done = 1;
          S.status = GB_CG_MAXITER;
        } else {
          S.beta = tot / S.rr_hat_old;
          S.rr_hat = tot;
          S.rmax = rnorm;
        }
      }
    }
  }
}

// ---- host side --------------------------------------------------------------------

// First-fit allocator over [0, size) with coalescing; 256-byte granules.
class Pool {
 public:
  void reset(size_t size) {
    free_.clear();
    free_[0] = size;
  }
  bool alloc(size_t bytes, size_t * off) {
    bytes = (bytes + 255) & ~size_t(255);
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second >= bytes) {
        *off = it->first;
        const size_t rest = it->second - bytes;
        const size_t at = it->first + bytes;
        free_.erase(it);
        if (rest) free_[at] = rest;
        return true;
      }
    }
    return false;
  }
  void release(size_t off, size_t bytes) {
    bytes = (bytes + 255) & ~size_t(255);
    auto it = free_.emplace(off, bytes).first;
    auto nx = std::next(it);
    if (nx != free_.end() && it->first + it->second == nx->first) {
      it->second += nx->second;
      free_.erase(nx);
    }
    if (it != free_.begin()) {
      auto pv = std::prev(it);
      if (pv->first + pv->second == it->first) {
        pv->second += it->second;
        free_.erase(it);
      }
    }
  }
  size_t largest() const {
    size_t m = 0;
    for (const auto & f : free_) m = std::max(m, f.second);
    return m;
  }

 private:
  std::map<size_t, size_t> free_;
};

struct Request {
  uint64_t id = 0;
  uint32_t n = 0, nnz = 0;
  std::vector<uint32_t> rowptr, rowind;
  std::vector<double> val64, b;
  double * x_out = nullptr;
  double tol_rel = 0.0;
  size_t niter = 0;
  double t_submit = 0.0;
  size_t bytes = 0;
  std::vector<SrvTile> tiles;  // slot-relative (slot field filled at admission)
};

struct SlotHost {
  bool used = false;
  uint64_t id = 0;
  uint32_t n = 0;
  size_t off = 0, bytes = 0;
  double * x_out = nullptr;
  double t_submit = 0.0, t_admit = 0.0;
  std::vector<SrvTile> tiles;
};

size_t align256(size_t v) { return (v + 255) & ~size_t(255); }

}  // namespace
}  // namespace gb

struct gb_server {
  gb_server_config_t cfg{};
  bool mixed = true;
  int sm_count = 0;
  unsigned grid = 0;
  std::chrono::steady_clock::time_point t0;
  char * pool = nullptr;
  gb::Pool alloc;
  gb::SrvSlot * d_slots = nullptr;
  gb::SrvSlot * h_slots = nullptr;  // pinned mirror
  gb::SrvTile * d_tiles = nullptr;
  uint32_t * d_ntiles = nullptr;
  uint32_t * h_ntiles = nullptr;    // pinned
  gb::SrvTile * h_tiles = nullptr;  // pinned staging of the tile list
  double * d_part = nullptr;        // 5 * kMaxTiles
  std::vector<gb::SlotHost> slots;
  std::deque<gb::Request> queue;
  std::vector<gb_server_result_t> results;
  size_t total_tiles = 0;
  bool dirty = false;
  cudaStream_t stream = nullptr;
  cudaGraphExec_t graph = nullptr;
  cudaEvent_t step_done = nullptr;
  bool inflight = false;
};

namespace gb {
namespace {

double now_s(const gb_server & s) {
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - s.t0).count();
}

SrvDev dev_view(gb_server & s) {
  SrvDev d;
  d.slots = s.d_slots;
  d.tiles = s.d_tiles;
  d.ntiles = s.d_ntiles;
  d.pa = s.d_part;
  d.pb = s.d_part + kMaxTiles;
  d.pr = s.d_part + 2 * kMaxTiles;
  d.pi0 = s.d_part + 3 * kMaxTiles;
  d.pi1 = s.d_part + 4 * kMaxTiles;
  return d;
}

int capture_graph(gb_server & s) {
  cudaStream_t cs = nullptr;
  GB_CUDA_TRY(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
  cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
  const SrvDev d = dev_view(s);
  if (e == cudaSuccess) {
    e = s.mixed ? launch_k(srv_init_kernel<float, true>, s.grid, kSrvBlock, 0, cs, false, d)
                : launch_k(srv_init_kernel<double, false>, s.grid, kSrvBlock, 0, cs, false, d);
    for (uint32_t k = 0; k < s.cfg.iters_per_step && e == cudaSuccess; ++k) {
      if (s.mixed) {
        e = launch_k(srv_a_kernel<float>, s.grid, kSrvBlock, 0, cs, true, d);
        if (e == cudaSuccess) e = launch_k(srv_b_kernel<float, true>, s.grid, kSrvBlock, 0, cs, true, d);
        if (e == cudaSuccess) e = launch_k(srv_r_kernel, s.grid, kSrvBlock, 0, cs, true, d);
      } else {
        e = launch_k(srv_a_kernel<double>, s.grid, kSrvBlock, 0, cs, true, d);
        if (e == cudaSuccess)
          e = launch_k(srv_b_kernel<double, false>, s.grid, kSrvBlock, 0, cs, true, d);
      }
    }
  }
  cudaGraph_t g = nullptr;
  const cudaError_t e2 = cudaStreamEndCapture(cs, &g);
  if (e == cudaSuccess) e = e2;
  if (e == cudaSuccess) e = cudaGraphInstantiate(&s.graph, g, 0);
  if (g) cudaGraphDestroy(g);
  cudaStreamDestroy(cs);
  GB_CUDA_TRY(e);
  return GOOSEBERRY_SUCCESS;
}

void destroy_server(gb_server * s) {
  if (!s) return;
  if (s->stream) cudaStreamSynchronize(s->stream);
  if (s->graph) cudaGraphExecDestroy(s->graph);
  if (s->step_done) cudaEventDestroy(s->step_done);
  if (s->stream) cudaStreamDestroy(s->stream);
  cudaFree(s->pool);
  cudaFree(s->d_slots);
  cudaFree(s->d_tiles);
  cudaFree(s->d_ntiles);
  cudaFree(s->d_part);
  if (s->h_slots) cudaFreeHost(s->h_slots);
  if (s->h_tiles) cudaFreeHost(s->h_tiles);
  if (s->h_ntiles) cudaFreeHost(s->h_ntiles);
  delete s;
}

int create_server(const gb_server_config_t & cfg, gb_server * s) {
  GB_CHECK_INPUT(cfg.pool_bytes >= (1u << 20), "pool_bytes must be at least 1 MiB");
  GB_CHECK_INPUT(cfg.max_slots >= 1 && cfg.max_slots <= 4096, "max_slots must be in [1, 4096]");
  GB_CHECK_INPUT(cfg.mode == GB_CG_MIXED || cfg.mode == GB_CG_F64, "mode must be GB_CG_MIXED or GB_CG_F64");
  GB_CHECK_INPUT(cfg.iters_per_step >= 1 && cfg.iters_per_step <= 1024,
      "iters_per_step must be in [1, 1024]");
  s->cfg = cfg;
  s->mixed = cfg.mode == GB_CG_MIXED;
  s->t0 = std::chrono::steady_clock::now();
  GB_TRY(sm_count_of_current_device(&s->sm_count));
  int occ = 0;
  GB_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ,
      s->mixed ? reinterpret_cast<const void *>(srv_a_kernel<float>)
               : reinterpret_cast<const void *>(srv_a_kernel<double>), kSrvBlock, 0));
  s->grid = static_cast<unsigned>(s->sm_count * std::max(1, std::min(occ, 4)));
  GB_CUDA_TRY(cudaMalloc(&s->pool, cfg.pool_bytes));
  s->alloc.reset(cfg.pool_bytes);
  GB_CUDA_TRY(cudaMalloc(&s->d_slots, cfg.max_slots * sizeof(SrvSlot)));
  GB_CUDA_TRY(cudaMemset(s->d_slots, 0, cfg.max_slots * sizeof(SrvSlot)));
  GB_CUDA_TRY(cudaMallocHost(&s->h_slots, cfg.max_slots * sizeof(SrvSlot)));
  std::memset(s->h_slots, 0, cfg.max_slots * sizeof(SrvSlot));
  GB_CUDA_TRY(cudaMalloc(&s->d_tiles, kMaxTiles * sizeof(SrvTile)));
  GB_CUDA_TRY(cudaMallocHost(&s->h_tiles, kMaxTiles * sizeof(SrvTile)));
  GB_CUDA_TRY(cudaMalloc(&s->d_ntiles, sizeof(uint32_t)));
  GB_CUDA_TRY(cudaMemset(s->d_ntiles, 0, sizeof(uint32_t)));
  GB_CUDA_TRY(cudaMallocHost(&s->h_ntiles, sizeof(uint32_t)));
  *s->h_ntiles = 0;
  GB_CUDA_TRY(cudaMalloc(&s->d_part, 5 * kMaxTiles * sizeof(double)));
  s->slots.resize(cfg.max_slots);
  GB_CUDA_TRY(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
  GB_CUDA_TRY(cudaEventCreateWithFlags(&s->step_done, cudaEventDisableTiming));
  GB_TRY(capture_graph(*s));
  return GOOSEBERRY_SUCCESS;
}

size_t footprint(bool mixed, uint32_t n, uint32_t nnz) {
  const size_t t = mixed ? 4 : 8;
  size_t b = align256(4ull * (n + 1)) + align256(4ull * nnz) + align256(8ull * nnz) +
             align256(8ull * n) /* b */ + align256(8ull * n) /* x0 */ +
             5 * align256(t * n) /* y r p0 p1 ap */;
  if (mixed) b += align256(4ull * nnz) /* val32 */ + align256(8ull * n) /* x1 */;
  return b;
}

int submit(gb_server & s, uint64_t id, dim_t n, const ind_t * rowptr, const dim_t * rowind,
    const double * rowval, const double * b, double * x_out, double tol_rel, size_t niter) {
  GB_CHECK_INPUT(n > 0 && rowptr && b && x_out, "NULL array or empty system");
  const uint32_t nnz = rowptr[n];
  GB_CHECK_INPUT(nnz == 0 || (rowind && rowval), "NULL array");
  Request q;
  q.id = id;
  q.n = n;
  q.nnz = nnz;
  q.x_out = x_out;
  q.tol_rel = tol_rel;
  q.niter = niter ? niter : std::max<size_t>(1000, 100 * static_cast<size_t>(n));
  q.t_submit = now_s(s);
  q.rowptr.assign(rowptr, rowptr + n + 1);
  GB_CHECK_INPUT(q.rowptr[0] == 0, "rowptr[0] must be 0");
  // row-aligned warp tiles; rows longer than a tile are refused
  uint32_t r = 0;
  while (r < n) {
    SrvTile t{0, r, 0, 0};
    uint32_t items = 0;
    while (r < n) {
      GB_CHECK_INPUT(q.rowptr[r + 1] >= q.rowptr[r], "rowptr decreases at row %u", r);
      const uint32_t l = q.rowptr[r + 1] - q.rowptr[r];
      GB_CHECK_INPUT(l < kTileItems, "row %u has %u nonzeros; the solve server takes at most %u",
          r, l, kTileItems - 1);
      if (items + l + 1 > kTileItems) break;
      items += l + 1;
      ++r;
    }
    t.row_count = r - t.row_begin;
    q.tiles.push_back(t);
  }
  GB_CHECK_INPUT(q.tiles.size() <= kMaxTiles, "request needs %zu tiles, more than %zu",
      q.tiles.size(), kMaxTiles);
  q.rowind.assign(rowind, rowind + nnz);
  for (uint32_t k = 0; k < nnz; ++k)
    GB_CHECK_INPUT(q.rowind[k] < n, "column index %u out of range for %u columns", q.rowind[k], n);
  q.val64.assign(rowval, rowval + nnz);
  q.b.assign(b, b + n);
  q.bytes = footprint(s.mixed, n, nnz);
  GB_CHECK_INPUT(q.bytes <= s.cfg.pool_bytes, "request needs %zu bytes of device memory, "
      "the pool holds %zu", q.bytes, s.cfg.pool_bytes);
  s.queue.push_back(std::move(q));
  return GOOSEBERRY_SUCCESS;
}

template <typename T>
T * carve(char * base, size_t & at, size_t count) {
  T * p = reinterpret_cast<T *>(base + at);
  at += align256(sizeof(T) * count);
  return p;
}

int admit(gb_server & s, Request & q, uint32_t k) {
  size_t off = 0;
  if (!s.alloc.alloc(q.bytes, &off)) return GOOSEBERRY_ERROR_UNKNOWN;  // caller checked
  SlotHost & h = s.slots[k];
  h.used = true;
  h.id = q.id;
  h.n = q.n;
  h.off = off;
  h.bytes = q.bytes;
  h.x_out = q.x_out;
  h.t_submit = q.t_submit;
  h.t_admit = now_s(s);
  h.tiles = std::move(q.tiles);
  for (auto & t : h.tiles) t.slot = k;
  char * base = s.pool + off;
  size_t at = 0;
  SrvSlot S;
  std::memset(&S, 0, sizeof(S));
  uint32_t * rp = carve<uint32_t>(base, at, q.n + 1);
  uint32_t * ri = carve<uint32_t>(base, at, q.nnz);
  double * v64 = carve<double>(base, at, q.nnz);
  double * bb = carve<double>(base, at, q.n);
  double * x0 = carve<double>(base, at, q.n);
  const size_t t = s.mixed ? 4 : 8;
  auto carve_t = [&](size_t count) {
    void * p = base + at;
    at += align256(t * count);
    return p;
  };
  void * y = carve_t(q.n);
  void * r = carve_t(q.n);
  void * p0 = carve_t(q.n);
  void * p1 = carve_t(q.n);
  void * ap = carve_t(q.n);
  float * v32 = nullptr;
  double * x1 = nullptr;
  if (s.mixed) {
    v32 = carve<float>(base, at, q.nnz);
    x1 = carve<double>(base, at, q.n);
  }
  GB_CUDA_TRY(cudaMemcpyAsync(rp, q.rowptr.data(), 4ull * (q.n + 1), cudaMemcpyHostToDevice,
      s.stream));
  if (q.nnz) {
    GB_CUDA_TRY(cudaMemcpyAsync(ri, q.rowind.data(), 4ull * q.nnz, cudaMemcpyHostToDevice,
        s.stream));
    GB_CUDA_TRY(cudaMemcpyAsync(v64, q.val64.data(), 8ull * q.nnz, cudaMemcpyHostToDevice,
        s.stream));
  }
  GB_CUDA_TRY(cudaMemcpyAsync(bb, q.b.data(), 8ull * q.n, cudaMemcpyHostToDevice, s.stream));
  if (s.mixed && q.nnz) GB_TRY(launch_round_f32(v64, v32, q.nnz, s.stream));
  S.rowptr = rp;
  S.rowind = ri;
  S.val64 = v64;
  S.val32 = v32;
  S.b = bb;
  S.x0 = x0;
  S.x1 = x1;
  S.y = y;
  S.r = r;
  S.p0 = p0;
  S.p1 = p1;
  S.ap = ap;
  S.n = q.n;
  S.tol_rel = q.tol_rel;
  S.niter = q.niter;
  S.live = 1;
  S.init = 1;
  S.status = GB_CG_MAXITER;
  s.h_slots[k] = S;
  s.dirty = true;
  return GOOSEBERRY_SUCCESS;
}

int step(gb_server & s, size_t * active, size_t * queued) {
  if (s.inflight) {
    GB_CUDA_TRY(cudaEventSynchronize(s.step_done));
    s.inflight = false;
  }
  // 1. retire finished solves: copy x out, free memory and the slot
  bool any_done = false;
  for (uint32_t k = 0; k < s.cfg.max_slots; ++k) {
    SlotHost & h = s.slots[k];
    const SrvSlot & S = s.h_slots[k];
    if (!h.used || !S.done) continue;
    const double * x = (s.mixed && S.xpar) ? S.x1 : S.x0;
    GB_CUDA_TRY(cudaMemcpyAsync(h.x_out, x, 8ull * h.n, cudaMemcpyDeviceToHost, s.stream));
    any_done = true;
  }
  if (any_done) GB_CUDA_TRY(cudaStreamSynchronize(s.stream));
  for (uint32_t k = 0; k < s.cfg.max_slots; ++k) {
    SlotHost & h = s.slots[k];
    SrvSlot & S = s.h_slots[k];
    if (!h.used || !S.done) continue;
    gb_server_result_t res;
    res.id = h.id;
    res.iterations = S.iter;
    res.refinements = S.refinements;
    res.rnorm = std::sqrt(S.rr_true);
    res.bnorm = S.bnorm;
    res.status = S.status;
    res.t_submit = h.t_submit;
    res.t_admit = h.t_admit;
    res.t_done = now_s(s);
    s.results.push_back(res);
    s.alloc.release(h.off, h.bytes);
    h = SlotHost();
    std::memset(&S, 0, sizeof(S));
    s.dirty = true;
  }
  // 2. admit queued requests (FIFO; a request that does not fit yet lets a
  //    few later, smaller ones through rather than blocking them)
  size_t scanned = 0;
  for (auto it = s.queue.begin(); it != s.queue.end() && scanned < 16;) {
    uint32_t k = 0;
    while (k < s.cfg.max_slots && s.slots[k].used) ++k;
    if (k == s.cfg.max_slots) break;
    if (it->bytes > s.alloc.largest() || s.total_tiles + it->tiles.size() > kMaxTiles) {
      ++it;
      ++scanned;
      continue;
    }
    s.total_tiles += it->tiles.size();
    GB_TRY(admit(s, *it, k));
    it = s.queue.erase(it);
  }
  // 3. rebuild the tile list and upload the slot table
  size_t nact = 0;
  if (s.dirty) {
    size_t nt = 0;
    for (uint32_t k = 0; k < s.cfg.max_slots; ++k) {
      SlotHost & h = s.slots[k];
      if (!h.used) continue;
      s.h_slots[k].tile0 = static_cast<uint32_t>(nt);
      s.h_slots[k].ntiles = static_cast<uint32_t>(h.tiles.size());
      std::memcpy(s.h_tiles + nt, h.tiles.data(), h.tiles.size() * sizeof(SrvTile));
      nt += h.tiles.size();
    }
    s.total_tiles = nt;
    *s.h_ntiles = static_cast<uint32_t>(nt);
    if (nt)
      GB_CUDA_TRY(cudaMemcpyAsync(s.d_tiles, s.h_tiles, nt * sizeof(SrvTile),
          cudaMemcpyHostToDevice, s.stream));
    GB_CUDA_TRY(cudaMemcpyAsync(s.d_ntiles, s.h_ntiles, sizeof(uint32_t), cudaMemcpyHostToDevice,
        s.stream));
    GB_CUDA_TRY(cudaMemcpyAsync(s.d_slots, s.h_slots, s.cfg.max_slots * sizeof(SrvSlot),
        cudaMemcpyHostToDevice, s.stream));
    s.dirty = false;
  }
  for (uint32_t k = 0; k < s.cfg.max_slots; ++k) nact += s.slots[k].used ? 1 : 0;
  // 4. run the step and bring the slot table back
  if (nact) {
    GB_CUDA_TRY(cudaGraphLaunch(s.graph, s.stream));
    GB_CUDA_TRY(cudaMemcpyAsync(s.h_slots, s.d_slots, s.cfg.max_slots * sizeof(SrvSlot),
        cudaMemcpyDeviceToHost, s.stream));
    GB_CUDA_TRY(cudaEventRecord(s.step_done, s.stream));
    s.inflight = true;
  }
  if (active) *active = nact;
  if (queued) *queued = s.queue.size();
  return GOOSEBERRY_SUCCESS;
}

}  // namespace
}  // namespace gb

extern "C" {

int gb_server_create(const gb_server_config_t * cfg, gb_server_t ** out) {
  GB_CHECK_INPUT(cfg && out, "NULL argument");
  *out = nullptr;
  gb_server * s = new gb_server();
  const int rc = gb::create_server(*cfg, s);
  if (rc != GOOSEBERRY_SUCCESS) {
    gb::destroy_server(s);
    return rc;
  }
  *out = s;
  return GOOSEBERRY_SUCCESS;
}

int gb_server_destroy(gb_server_t * s) {
  gb::destroy_server(s);
  return GOOSEBERRY_SUCCESS;
}

int gb_server_submit(gb_server_t * s, uint64_t id, dim_t n, const ind_t * rowptr,
    const dim_t * rowind, const double * rowval, const double * b, double * x_out,
    double tol_rel, size_t niter) {
  GB_CHECK_INPUT(s != nullptr, "server is NULL");
  return gb::submit(*s, id, n, rowptr, rowind, rowval, b, x_out, tol_rel, niter);
}

int gb_server_step(gb_server_t * s, size_t * active, size_t * queued) {
  GB_CHECK_INPUT(s != nullptr, "server is NULL");
  return gb::step(*s, active, queued);
}

int gb_server_poll(gb_server_t * s, gb_server_result_t * out, size_t max, size_t * count) {
  GB_CHECK_INPUT(s && count, "NULL argument");
  const size_t m = std::min(max, s->results.size());
  GB_CHECK_INPUT(m == 0 || out != nullptr, "out is NULL");
  for (size_t i = 0; i < m; ++i) out[i] = s->results[i];
  s->results.erase(s->results.begin(), s->results.begin() + m);
  *count = m;
  return GOOSEBERRY_SUCCESS;
}

double gb_server_clock(const gb_server_t * s) { return s ? gb::now_s(*s) : 0.0; }

}  // extern "C"
