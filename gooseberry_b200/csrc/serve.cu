// serve.cu -- batched CG serving: many uneven solves resident at once,
// continuous batching, admission by device-memory footprint.
//
// Reference: one cgd call (src/cgd.c:40-129) runs at a time from the CLI
// (src/gooseberry_bin.c:2078-2091).  Here every resident solve owns a slot:
// its CSR matrix and Krylov vectors live in one device pool (first-fit
// allocator, bounded by pool_bytes), and all slots advance together.
//
// Work list: every slot's rows are cut into row tiles of 2048 rows (the last
// one shorter); the tiles of all resident slots form ONE global list.  Each kernel is persistent over that list, one
// CTA tile at a time: eight compute warps run the pipelined thread-per-row
// loop of the single-solve kernels over the tile (coalesced row vectors,
// reference summation order), while a ninth, control warp prefetches the
// next tile's descriptor and slot record into the other half of a shared
// double buffer and finishes the previous tile: it publishes the tile's dot
// partial, takes the slot's ticket, and when it is the slot's last tile adds
// the slot's partials in tile order (deterministic) and advances that slot's
// scalar state (alpha / beta / stop decision).  So one launch moves a
// 1k-row and a 262k-row solve forward by one phase each, and the launch
// cost is shared by the whole batch.
//
// Per step (one graph replay): iters_per_step x { A, B }.
//   A: per slot one of  CG   -- SpMV + direction update + p.Ap
//                       INIT -- x = 0, r = b, p = 0, b.b (newly admitted)
//   B: per slot one of  UPDATE   -- x/y and r update + r.r, stop or
//                                   reliable-update decision
//                       RELIABLE -- reliable FP64 residual update (mixed):
//                                   x += y, r = b - A x, true r.r
// A slot idles in the B launch after its INIT and in the A launch before its
// RELIABLE step.  The rare FP64 step rides in the lighter B kernel so that it
// adds nothing to the register demand of the SpMV kernel A, which sets the
// occupancy (3 CTAs of 288 threads per SM).
// Slot state lives in device memory, so the captured graph never changes;
// between steps the host reads the slot table back, retires finished solves
// (x copied out), admits queued requests into freed slots and memory,
// rebuilds the tile list and uploads the table.
//
// Mixed mode is the algorithm of cg_mixed.cu (FP32 values and vectors, FP64
// dots, reliable FP64 updates, convergence on the true residual); F64 mode
// is plain CG like cg.cu (convergence on the recurrence residual, as the
// reference).  A solve's arithmetic depends only on its own rows and tiles,
// so its result is bitwise the same alone or in any mix.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <new>
#include <mutex>
#include <tuple>
#include <vector>

#include "gb_internal.h"
#include "spmv_tiles.cuh"
#include "cg_common.cuh"

namespace gb {
namespace {

constexpr int kSrvComputeWarps = 8;
constexpr int kSrvCompute = kSrvComputeWarps * 32;  // row threads per CTA
constexpr int kSrvThreads = kSrvCompute + 32;       // + the control warp
#ifndef GB_SRV_MIN_BLOCKS
#define GB_SRV_MIN_BLOCKS 3
#endif
#ifndef GB_SRV_MAX_REGS
#define GB_SRV_MAX_REGS 72
#endif
#ifndef GB_SRV_ROW_STAGE
#define GB_SRV_ROW_STAGE 5
#endif
#ifndef GB_SRV_TILE_ROWS
#define GB_SRV_TILE_ROWS 2048  // tile rows when the autotuner cannot run
#endif
constexpr int kSrvMinBlocks = GB_SRV_MIN_BLOCKS;
constexpr int kSrvMaxRegs = GB_SRV_MAX_REGS;  // 3 CTAs of 288 threads per SM at 72
// Row entries loaded ahead per thread: 5 holds a whole row of a 2-D 5-point
// stencil (longer rows finish in the loop's tail); measured 1.3x the solves/s
// of 6 at this register budget.
constexpr int kSrvRowStage = GB_SRV_ROW_STAGE;
constexpr uint32_t kTileRows = GB_SRV_TILE_ROWS;
constexpr uint32_t kMaxRowNnz = 255;      // longer rows belong to the single-solve CG
constexpr double kSrvDelta = 0.1;         // reliable update trigger (see cg_mixed.cu)
constexpr size_t kMaxTiles = 1u << 20;

// What a launch does for a slot.  A: kWorkCg, kWorkInit or kWorkIdle;
// B: kWorkUpdate, kWorkReliable or kWorkIdle.
enum : int { kWorkIdle = 0, kWorkCg = 1, kWorkInit = 2, kWorkUpdate = 3, kWorkReliable = 4 };

struct SrvTile {
  uint32_t slot;
  uint32_t row_begin;
  uint32_t row_count;
  uint32_t pad;
};

struct __align__(16) SrvSlot {
  // written by the host at admission
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
  uint32_t n, ntiles, tile0, pad0;
  double tol_rel;
  unsigned long long niter;
  // written by the kernels (the slot's last tile of a launch)
  double rr_hat, rr_hat_old, alpha, beta, tol, bnorm, rmax, rr_true;
  unsigned long long iter, refinements;
  int live;     // slot holds a solve
  int a_work;   // what the next A launch does for this slot
  int b_work;   // what the next B launch does for this slot
  int done;     // finished (converged / maxiter / breakdown / nonfinite)
  int status;
  int y_reset;
  int xpar;
  int final_update;  // the pending reliable update is the last one (iteration limit)
  unsigned ticket_a, ticket_b, pad1, pad2;
};
static_assert(sizeof(SrvSlot) == 256, "slot record is sixteen 16-byte words");

struct __align__(16) SrvCtx {
  SrvTile tile;
  SrvSlot slot;
};

struct SrvDev {
  SrvSlot * slots;
  const SrvTile * tiles;
  const uint32_t * ntiles;  // device word: tiles in the list
  double2 * pa;             // per tile: A partial sums
  double2 * pb;             // per tile: B partial sums
};

__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Control warp: tile t's descriptor and its slot record into shared memory.
// L2-coherent loads: the record was written by other SMs in earlier launches.
__device__ __forceinline__ void load_ctx(const SrvDev & d, uint32_t t, SrvCtx & c, int lane) {
  const uint4 tv = __ldcg(reinterpret_cast<const uint4 *>(d.tiles + t));
  if (lane == 0) *reinterpret_cast<uint4 *>(&c.tile) = tv;
  if (lane < 16)
    reinterpret_cast<uint4 *>(&c.slot)[lane] =
        __ldcg(reinterpret_cast<const uint4 *>(d.slots + tv.x) + lane);
}

// Control warp, after the tile's rows: publish the tile's sums and take the
// slot's ticket.  True (in every lane) for the slot's last tile; `tot` is
// then the slot's sum over its tiles in tile order.
__device__ __forceinline__ bool slot_finish(double2 * part, uint32_t t, double2 mine,
    unsigned * ticket, uint32_t t0, uint32_t nt, int lane, double2 * tot) {
  unsigned tk = 0;
  if (lane == 0) {
    part[t] = mine;
    __threadfence();
    tk = atomicAdd(ticket, 1u);
  }
  tk = __shfl_sync(0xffffffffu, tk, 0);
  if (tk != nt - 1) return false;
  __threadfence();
  double sx = 0.0, sy = 0.0;
  for (uint32_t i = lane; i < nt; i += 32) {
    const double2 v = __ldcg(part + t0 + i);
    sx += v.x;
    sy += v.y;
  }
  tot->x = warp_sum_d(sx);
  tot->y = warp_sum_d(sy);
  return true;
}

// The persistent tile loop shared by both kernels.  Work supplies
// active(slot), rows(ctx, tid, s0, s1) and finish(d, t, ctx, sums, lane).
template <class Work>
__device__ __forceinline__ void srv_loop(const SrvDev & d, Work & w) {
  __shared__ SrvCtx ctx[2];
  __shared__ double red[2][kSrvComputeWarps][2];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t nt = __ldcg(d.ntiles);
  uint32_t t = blockIdx.x;
  if (t >= nt) return;
  if (warp == kSrvComputeWarps) load_ctx(d, t, ctx[0], lane);
  __syncthreads();
  for (int buf = 0; t < nt; t += gridDim.x, buf ^= 1) {
    const SrvCtx & c = ctx[buf];
    const bool act = Work::active(c.slot);
    if (warp == kSrvComputeWarps) {
      if (t + gridDim.x < nt) load_ctx(d, t + gridDim.x, ctx[buf ^ 1], lane);
    } else if (act) {
      double s0 = 0.0, s1 = 0.0;
      w.rows(c, threadIdx.x, s0, s1);
      s0 = warp_sum_d(s0);
      s1 = warp_sum_d(s1);
      if (lane == 0) {
        red[buf][warp][0] = s0;
        red[buf][warp][1] = s1;
      }
    }
    __syncthreads();
    if (warp == kSrvComputeWarps && act) {
      double2 s = make_double2(0.0, 0.0);
      if (lane == 0)
        for (int k = 0; k < kSrvComputeWarps; ++k) {
          s.x += red[buf][k][0];
          s.y += red[buf][k][1];
        }
      w.finish(d, t, c, s, lane);
      __syncwarp();  // lane 0 is done reading ctx[buf] before it is refilled
    }
  }
}

template <typename T>
__device__ __forceinline__ const T * values_of(const SrvSlot & S);
template <>
__device__ __forceinline__ const float * values_of<float>(const SrvSlot & S) { return S.val32; }
template <>
__device__ __forceinline__ const double * values_of<double>(const SrvSlot & S) {
  return S.val64;
}

// ---- A: CG step / init / reliable update --------------------------------------------

template <typename T>
struct SrvGatherP {  // direction p = r + beta * p_old, rebuilt inside the gather
  const T * r;
  const T * pold;
  T beta;
  template <class P>
  __device__ __forceinline__ T operator()(uint32_t c, P pol) const {
    return fma(beta, ld_keep(pold + c, pol), ld_keep(r + c, pol));
  }
};

template <typename T>
struct SrvOutA {
  T * ap;
  T * pnew;
  const T * r;
  const T * pold;
  T beta;
  double local;
  struct Pre {
    T r, pold;
  };
  __device__ __forceinline__ Pre pre(uint32_t i) const { return Pre{r[i], pold[i]}; }
  __device__ __forceinline__ void row_pre(uint32_t i, T v, const Pre & q) {
    ap[i] = v;
    const T pn = fma(beta, q.pold, q.r);
    pnew[i] = pn;
    local += static_cast<double>(pn) * static_cast<double>(v);
  }
};

struct SrvGatherXY {  // x + y in FP64
  const double * x;
  const float * y;
  bool use_y;
  template <class P>
  __device__ __forceinline__ double operator()(uint32_t c, P pol) const {
    const double xc = ld_keep(x + c, pol);
    return use_y ? xc + static_cast<double>(ld_keep(y + c, pol)) : xc;
  }
};

struct SrvOutR {  // x_new = x + y;  r = b - A (x + y) rounded to FP32
  double * xnew;
  float * r32;
  const double * xold;
  const float * y;
  const double * b;
  bool use_y;
  double local;
  struct Pre {
    double x, b;
    float y;
  };
  __device__ __forceinline__ Pre pre(uint32_t i) const {
    return Pre{xold[i], b[i], use_y ? y[i] : 0.0f};
  }
  __device__ __forceinline__ void row_pre(uint32_t i, double v, const Pre & q) {
    xnew[i] = use_y ? q.x + static_cast<double>(q.y) : q.x;
    const double rt = q.b - v;
    r32[i] = static_cast<float>(rt);
    local += rt * rt;
  }
};

template <typename T, bool MIXED>
struct WorkA {
  uint64_t pol_m, pol_x;
  __device__ __forceinline__ static bool active(const SrvSlot & S) {
    return S.live && !S.done && S.a_work != kWorkIdle;
  }

  __device__ __forceinline__ void rows(const SrvCtx & c, int tid, double & s0, double & s1) {
    const SrvSlot & S = c.slot;
    const uint32_t r0 = c.tile.row_begin, r1 = r0 + c.tile.row_count;
    if (S.a_work == kWorkCg) {
      const bool par = (S.iter & 1ull) != 0;
      const T * pold = static_cast<const T *>(par ? S.p1 : S.p0);
      T * pnew = static_cast<T *>(par ? S.p0 : S.p1);
      const T * r = static_cast<const T *>(S.r);
      const T beta = static_cast<T>(S.beta);
      SrvGatherP<T> g{r, pold, beta};
      SrvOutA<T> o{static_cast<T *>(S.ap), pnew, r, pold, beta, 0.0};
      spmv_row_loop<T, T, kSrvRowStage>(r0 + tid, r1, kSrvCompute, S.n, S.rowptr, S.rowind, values_of<T>(S),
          g, o, pol_m, pol_x);
      s0 = o.local;
    } else {  // kWorkInit
      T * r = static_cast<T *>(S.r);
      T * p0 = static_cast<T *>(S.p0);
      for (uint32_t i = r0 + tid; i < r1; i += kSrvCompute) {
        const double bv = S.b[i];
        const T rv = static_cast<T>(bv);
        S.x0[i] = 0.0;
        r[i] = rv;
        p0[i] = T(0);
        s0 += bv * bv;
        s1 += static_cast<double>(rv) * static_cast<double>(rv);
      }
    }
  }

  __device__ __forceinline__ void finish(const SrvDev & d, uint32_t t, const SrvCtx & c,
      double2 mine, int lane) {
    const SrvSlot & C = c.slot;
    SrvSlot * S = d.slots + c.tile.slot;
    double2 tot;
    if (!slot_finish(d.pa, t, mine, &S->ticket_a, C.tile0, C.ntiles, lane, &tot)) return;
    if (lane != 0) return;
    S->ticket_a = 0;
    if (C.a_work == kWorkCg) {
      const double pap = tot.x;
      S->b_work = kWorkUpdate;
      if (!(pap > 0.0)) {
        S->done = 1;
        S->status = (pap == pap && C.rr_hat == C.rr_hat) ? GB_CG_BREAKDOWN : GB_CG_NONFINITE;
        S->rr_true = C.rr_hat;
      } else {
        S->alpha = C.rr_hat / pap;
      }
    } else {  // kWorkInit
      const double bb = tot.x, rr = MIXED ? tot.y : tot.x;
      S->bnorm = sqrt(bb);
      S->tol = C.tol_rel * sqrt(bb);
      S->rr_true = bb;
      S->rr_hat = rr;
      S->rr_hat_old = rr;
      S->rmax = sqrt(rr);
      S->alpha = 0.0;
      S->beta = 0.0;
      S->iter = 0;
      S->refinements = 0;
      S->xpar = 0;
      S->y_reset = 1;
      S->final_update = 0;
      S->status = GB_CG_MAXITER;
      S->a_work = kWorkCg;
      S->b_work = kWorkIdle;
      if (bb == 0.0) {
        S->done = 1;
        S->status = GB_CG_CONVERGED;
      } else if (!(bb == bb) || isinf(bb)) {
        S->done = 1;
        S->status = GB_CG_NONFINITE;
      }
    }
  }
};

// ---- B: solution / residual update, r.r, stop or update decision;  or the
//      reliable FP64 residual update (mixed) ----------------------------------------------

template <typename T>
struct Vec16;
template <>
struct Vec16<float> {
  using type = float4;
};
template <>
struct Vec16<double> {
  using type = double2;
};

template <typename T, bool MIXED>
struct WorkB {
  uint64_t pol_m, pol_x;
  __device__ __forceinline__ static bool active(const SrvSlot & S) {
    return S.live && !S.done && S.b_work != kWorkIdle;
  }

  __device__ __forceinline__ void rows(const SrvCtx & c, int tid, double & s0, double &) {
    const SrvSlot & S = c.slot;
    const uint32_t r0 = c.tile.row_begin, cnt = c.tile.row_count;
    if (MIXED && S.b_work == kWorkReliable) {
      const bool use_y = S.y_reset == 0;
      const double * xold = S.xpar ? S.x1 : S.x0;
      double * xnew = S.xpar ? S.x0 : S.x1;
      const float * y = static_cast<const float *>(S.y);
      SrvGatherXY g{xold, y, use_y};
      SrvOutR o{xnew, static_cast<float *>(S.r), xold, y, S.b, use_y, 0.0};
      spmv_row_loop<double, double, kSrvRowStage>(r0 + tid, r0 + cnt, kSrvCompute, S.n, S.rowptr, S.rowind,
          S.val64, g, o, pol_m, pol_x);
      s0 = o.local;
      return;
    }
    const T alpha = static_cast<T>(S.alpha);
    const bool fresh = S.y_reset != 0;
    const bool par = (S.iter & 1ull) != 0;
    const T * pnew = static_cast<const T *>(par ? S.p0 : S.p1);
    const T * ap = static_cast<const T *>(S.ap);
    T * r = static_cast<T *>(S.r);
    T * y = static_cast<T *>(S.y);
    // one row's update; s0 += r.r
    auto one = [&](uint32_t i, T pv, T av, T rv, double xv) {
      if (MIXED) {
        y[i] = fma(alpha, pv, static_cast<T>(xv));
      } else {
        S.x0[i] = fma(static_cast<double>(alpha), static_cast<double>(pv), xv);
      }
      const T rn = fma(-alpha, av, rv);
      r[i] = rn;
      s0 += static_cast<double>(rn) * static_cast<double>(rn);
    };
    // 16-byte units (tiles start at multiples of the tile size, and the pool
    // places every vector on a 256-byte boundary); the rows past the last
    // complete unit, or a tile that is not aligned, take one row per thread
    constexpr uint32_t VN = 16 / sizeof(T);
    using V = typename Vec16<T>::type;
    const uint32_t nfull = (r0 % VN == 0) ? cnt / VN : 0u;
    for (uint32_t u = tid; u < nfull; u += kSrvCompute) {
      const uint32_t i = r0 + u * VN;
      const V pv = *reinterpret_cast<const V *>(pnew + i);
      const V av = *reinterpret_cast<const V *>(ap + i);
      const V rv = *reinterpret_cast<const V *>(r + i);
      V yv{};
      double2 xv[VN / 2 > 0 ? VN / 2 : 1];
      if (MIXED) {
        if (!fresh) yv = *reinterpret_cast<const V *>(y + i);
      } else {
#pragma unroll
        for (uint32_t h = 0; h < VN / 2; ++h) xv[h] = reinterpret_cast<const double2 *>(S.x0 + i)[h];
      }
      const T * pp = reinterpret_cast<const T *>(&pv);
      const T * aa = reinterpret_cast<const T *>(&av);
      const T * rr = reinterpret_cast<const T *>(&rv);
      const T * yy = reinterpret_cast<const T *>(&yv);
      const double * xx = reinterpret_cast<const double *>(xv);
#pragma unroll
      for (uint32_t e = 0; e < VN; ++e)
        one(i + e, pp[e], aa[e], rr[e], MIXED ? static_cast<double>(yy[e]) : xx[e]);
    }
    for (uint32_t q = VN * nfull + tid; q < cnt; q += kSrvCompute) {
      const uint32_t i = r0 + q;
      one(i, pnew[i], ap[i], r[i],
          MIXED ? (fresh ? 0.0 : static_cast<double>(y[i])) : S.x0[i]);
    }
  }

  __device__ __forceinline__ void finish(const SrvDev & d, uint32_t t, const SrvCtx & c,
      double2 mine, int lane) {
    const SrvSlot & C = c.slot;
    SrvSlot * S = d.slots + c.tile.slot;
    double2 tot;
    if (!slot_finish(d.pb, t, mine, &S->ticket_b, C.tile0, C.ntiles, lane, &tot)) return;
    if (lane != 0) return;
    S->ticket_b = 0;
    if (MIXED && C.b_work == kWorkReliable) {  // r is now the true residual of x
      const double rr = tot.x;
      const double rnorm = sqrt(rr);
      S->rr_true = rr;
      S->refinements = C.refinements + 1;
      S->xpar = C.xpar ^ 1;
      S->y_reset = 1;
      S->a_work = kWorkCg;
      S->b_work = kWorkIdle;
      if (!(rnorm == rnorm) || isinf(rnorm)) {
        S->done = 1;
        S->status = GB_CG_NONFINITE;
      } else if (rnorm <= C.tol) {
        S->done = 1;
        S->status = GB_CG_CONVERGED;
      } else if (C.final_update) {
        S->done = 1;
        S->status = GB_CG_MAXITER;
      } else {
        S->beta = rr / C.rr_hat_old;
        S->rr_hat = rr;
        S->rmax = rnorm;
      }
      return;
    }
    const double rr = tot.x;
    S->y_reset = 0;
    S->rr_hat_old = C.rr_hat;
    S->beta = rr / C.rr_hat;
    S->rr_hat = rr;
    const unsigned long long it = C.iter + 1;
    S->iter = it;
    const double rnorm = sqrt(rr);
    S->rmax = fmax(C.rmax, rnorm);
    if (!(rnorm == rnorm) || isinf(rnorm)) {
      S->done = 1;
      S->status = GB_CG_NONFINITE;
      S->rr_true = rr;
    } else if (MIXED) {
      const bool last = C.niter && it >= C.niter;
      if (rnorm <= C.tol || rnorm < kSrvDelta * fmax(C.rmax, rnorm) || last) {
        // next launch pair: A idles, B folds y into x and takes the true residual
        S->a_work = kWorkIdle;
        S->b_work = kWorkReliable;
        S->final_update = last ? 1 : 0;
      }
    } else if (rnorm <= C.tol) {
      S->done = 1;
      S->status = GB_CG_CONVERGED;
      S->rr_true = rr;
    } else if (C.niter && it >= C.niter) {
      S->done = 1;
      S->status = GB_CG_MAXITER;
      S->rr_true = rr;
    }
  }
};

// Register budgets: the FP32 kernels are held to 72 so that 3 CTAs fit per
// SM (the rare FP64 reliable step in B spills there, which costs little);
// the FP64 forms get 96 and run with their own grid.
template <typename T, bool MIXED>
struct SrvRegs {
  static constexpr int a = sizeof(T) == 4 ? kSrvMaxRegs : 96;
  static constexpr int b = sizeof(T) == 4 ? kSrvMaxRegs : 96;
};

template <typename T, bool MIXED>
__global__ void __maxnreg__((SrvRegs<T, MIXED>::a)) srv_a_kernel(const SrvDev d) {
  pdl_wait_and_release();
  WorkA<T, MIXED> w{policy_evict_first(), policy_evict_last()};
  srv_loop(d, w);
}

template <typename T, bool MIXED>
__global__ void __maxnreg__((SrvRegs<T, MIXED>::b)) srv_b_kernel(const SrvDev d) {
  pdl_wait_and_release();
  WorkB<T, MIXED> w{policy_evict_first(), policy_evict_last()};
  srv_loop(d, w);
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
  // the request's copy of rowptr, rowind, the values and b: in the server's
  // pinned staging arena when it has room (stage_len > 0), else in `own`
  uint32_t * rowptr = nullptr;
  uint32_t * rowind = nullptr;
  double * val64 = nullptr;
  double * b = nullptr;
  size_t stage_off = 0, stage_len = 0;
  std::unique_ptr<unsigned char[]> own;
  double * x_out = nullptr;
  double tol_rel = 0.0;
  size_t niter = 0;
  double t_submit = 0.0;
  size_t bytes = 0;
  std::vector<SrvTile> tiles;  // slot-relative (slot field filled at admission)
};

struct SlotHost {
  bool used = false;
  bool cancel = false;  // retire at the next step without copying x out
  uint64_t id = 0;
  uint32_t n = 0;
  size_t off = 0, bytes = 0;
  double * x_out = nullptr;
  double t_submit = 0.0, t_admit = 0.0;
  std::vector<SrvTile> tiles;
};

size_t align256(size_t v) { return (v + 255) & ~size_t(255); }

// Host bytes of a queued request's arrays (rowptr, rowind, values, b).
size_t request_host_bytes(uint32_t n, uint32_t nnz) {
  return align256(4ull * (n + 1)) + align256(4ull * nnz) + align256(8ull * nnz) +
         align256(8ull * n);
}

}  // namespace
}  // namespace gb

struct gb_server {
  gb_server_config_t cfg{};
  bool mixed = true;
  int sm_count = 0;
  unsigned grid_a = 0, grid_b = 0;
  std::chrono::steady_clock::time_point t0;
  char * pool = nullptr;
  gb::Pool alloc;
  gb::SrvSlot * d_slots = nullptr;
  gb::SrvSlot * h_slots = nullptr;  // pinned mirror
  gb::SrvTile * d_tiles = nullptr;
  uint32_t * d_ntiles = nullptr;
  uint32_t * h_ntiles = nullptr;    // pinned
  gb::SrvTile * h_tiles = nullptr;  // pinned staging of the tile list
  double2 * d_part = nullptr;       // 2 * kMaxTiles (A and B partial sums)
  // Pinned staging of queued requests: submit copies a request here (memory
  // already faulted in), and admission uploads it with an asynchronous copy
  // instead of a staged one while the device waits.  Regions go back once the
  // copies that read them are done (the next step's wait).
  unsigned char * stage = nullptr;
  gb::Pool stage_alloc;
  std::vector<std::pair<size_t, size_t>> stage_done;
  std::vector<gb::SlotHost> slots;
  std::deque<gb::Request> queue;
  std::vector<gb_server_result_t> results;
  size_t total_tiles = 0;
  bool dirty = false;
  cudaStream_t stream = nullptr;
  cudaGraphExec_t graph = nullptr;
  cudaEvent_t step_start = nullptr;
  cudaEvent_t step_done = nullptr;
  bool inflight = false;
  gb_server_stats_t stats{};
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
  return d;
}

int capture_graph(gb_server & s) {
  cudaStream_t cs = nullptr;
  GB_CUDA_TRY(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
  cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
  const SrvDev d = dev_view(s);
  for (uint32_t k = 0; k < s.cfg.iters_per_step && e == cudaSuccess; ++k) {
    const bool pdl = k > 0;
    if (s.mixed) {
      e = launch_k(srv_a_kernel<float, true>, s.grid_a, kSrvThreads, 0, cs, pdl, d);
      if (e == cudaSuccess)
        e = launch_k(srv_b_kernel<float, true>, s.grid_b, kSrvThreads, 0, cs, true, d);
    } else {
      e = launch_k(srv_a_kernel<double, false>, s.grid_a, kSrvThreads, 0, cs, pdl, d);
      if (e == cudaSuccess)
        e = launch_k(srv_b_kernel<double, false>, s.grid_b, kSrvThreads, 0, cs, true, d);
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
  if (s->step_start) cudaEventDestroy(s->step_start);
  if (s->stream) cudaStreamDestroy(s->stream);
  cudaFree(s->pool);
  cudaFree(s->d_slots);
  cudaFree(s->d_tiles);
  cudaFree(s->d_ntiles);
  cudaFree(s->d_part);
  if (s->h_slots) cudaFreeHost(s->h_slots);
  if (s->h_tiles) cudaFreeHost(s->h_tiles);
  if (s->h_ntiles) cudaFreeHost(s->h_ntiles);
  if (s->stage) cudaFreeHost(s->stage);
  delete s;
}

int create_server(const gb_server_config_t & cfg, gb_server * s) {
  GB_CHECK_INPUT(cfg.pool_bytes >= (1u << 20), "pool_bytes must be at least 1 MiB");
  GB_CHECK_INPUT(cfg.max_slots >= 1 && cfg.max_slots <= 4096, "max_slots must be in [1, 4096]");
  GB_CHECK_INPUT(cfg.mode == GB_CG_MIXED || cfg.mode == GB_CG_F64, "mode must be GB_CG_MIXED or GB_CG_F64");
  GB_CHECK_INPUT(cfg.iters_per_step >= 1 && cfg.iters_per_step <= 1024,
      "iters_per_step must be in [1, 1024]");
  GB_CHECK_INPUT(cfg.tile_rows == 0 || (cfg.tile_rows >= 256 && cfg.tile_rows <= 65536 &&
                                        (cfg.tile_rows & (cfg.tile_rows - 1)) == 0),
      "tile_rows must be 0 (autotuned) or a power of two in [256, 65536]");
  s->cfg = cfg;
  s->mixed = cfg.mode == GB_CG_MIXED;
  s->t0 = std::chrono::steady_clock::now();
  GB_TRY(sm_count_of_current_device(&s->sm_count));
  // each kernel: one resident wave (it is persistent over the tile list)
  int occ_a = 0, occ_b = 0;
  GB_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_a,
      s->mixed ? reinterpret_cast<const void *>(srv_a_kernel<float, true>)
               : reinterpret_cast<const void *>(srv_a_kernel<double, false>), kSrvThreads, 0));
  GB_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_b,
      s->mixed ? reinterpret_cast<const void *>(srv_b_kernel<float, true>)
               : reinterpret_cast<const void *>(srv_b_kernel<double, false>), kSrvThreads, 0));
  s->grid_a = static_cast<unsigned>(s->sm_count * std::max(1, std::min(occ_a, kSrvMinBlocks)));
  s->grid_b = static_cast<unsigned>(s->sm_count * std::max(1, std::min(occ_b, kSrvMinBlocks)));
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
  // the staging arena: an eighth of the device pool, between 64 MiB and
  // 2 GiB; without it (pinning refused) requests are copied to pageable memory
  {
    const size_t want = std::min<size_t>(std::max<size_t>(cfg.pool_bytes / 8, 64ull << 20),
        2ull << 30);
    void * st = nullptr;
    if (cudaHostAlloc(&st, want, cudaHostAllocPortable) == cudaSuccess) {
      s->stage = static_cast<unsigned char *>(st);
      s->stage_alloc.reset(want);
    } else {
      cudaGetLastError();
    }
  }
  *s->h_ntiles = 0;
  GB_CUDA_TRY(cudaMalloc(&s->d_part, 2 * kMaxTiles * sizeof(double2)));
  s->slots.resize(cfg.max_slots);
  GB_CUDA_TRY(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
  GB_CUDA_TRY(cudaEventCreate(&s->step_start));
  GB_CUDA_TRY(cudaEventCreate(&s->step_done));
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

int tile_rows_for(gb_server & s, const Request & q, uint32_t maxrow, uint32_t * out);

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
  const size_t hb = request_host_bytes(n, nnz);
  unsigned char * base = nullptr;
  size_t off = 0;
  if (s.stage && s.stage_alloc.alloc(hb, &off)) {
    base = s.stage + off;
    q.stage_off = off;
    q.stage_len = hb;
  } else {
    q.own.reset(new (std::nothrow) unsigned char[hb]);
    GB_CHECK_INPUT(q.own != nullptr, "no host memory for a request of %zu bytes", hb);
    base = q.own.get();
  }
  size_t at = 0;
  q.rowptr = reinterpret_cast<uint32_t *>(base + at);
  at += align256(4ull * (n + 1));
  q.rowind = reinterpret_cast<uint32_t *>(base + at);
  at += align256(4ull * nnz);
  q.val64 = reinterpret_cast<double *>(base + at);
  at += align256(8ull * nnz);
  q.b = reinterpret_cast<double *>(base + at);
  // checks run on the copy; a refused request hands its staging region back
  uint32_t maxrow = 0;
  const int rc = [&]() -> int {
    std::memcpy(q.rowptr, rowptr, 4ull * (n + 1));
    GB_CHECK_INPUT(q.rowptr[0] == 0, "rowptr[0] must be 0");
    for (uint32_t r = 0; r < n; ++r) {
      GB_CHECK_INPUT(q.rowptr[r + 1] >= q.rowptr[r], "rowptr decreases at row %u", r);
      const uint32_t l = q.rowptr[r + 1] - q.rowptr[r];
      GB_CHECK_INPUT(l <= kMaxRowNnz,
          "row %u has %u nonzeros; the solve server takes at most %u", r, l, kMaxRowNnz);
      maxrow = std::max(maxrow, l);
    }
    if (nnz) std::memcpy(q.rowind, rowind, 4ull * nnz);
    for (uint32_t k = 0; k < nnz; ++k)
      GB_CHECK_INPUT(q.rowind[k] < n, "column index %u out of range for %u columns",
          q.rowind[k], n);
    if (nnz) std::memcpy(q.val64, rowval, 8ull * nnz);
    std::memcpy(q.b, b, 8ull * n);
    q.bytes = footprint(s.mixed, n, nnz);
    GB_CHECK_INPUT(q.bytes <= s.cfg.pool_bytes, "request needs %zu bytes of device memory, "
        "the pool holds %zu", q.bytes, s.cfg.pool_bytes);
    // row tiles (from the request alone, so a solve is cut the same way
    // whatever else is resident)
    uint32_t T = 0;
    GB_TRY(tile_rows_for(s, q, maxrow, &T));
    const size_t ntiles = (static_cast<size_t>(n) + T - 1) / T;
    GB_CHECK_INPUT(ntiles <= kMaxTiles, "request needs %zu tiles, more than %zu", ntiles,
        kMaxTiles);
    for (uint32_t r = 0; r < n; r += T) q.tiles.push_back(SrvTile{0, r, std::min(T, n - r), 0});
    return GOOSEBERRY_SUCCESS;
  }();
  if (rc != GOOSEBERRY_SUCCESS) {
    if (q.stage_len) s.stage_alloc.release(q.stage_off, q.stage_len);
    return rc;
  }
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
  // (from the staging arena these copies are asynchronous)
  GB_CUDA_TRY(cudaMemcpyAsync(rp, q.rowptr, 4ull * (q.n + 1), cudaMemcpyHostToDevice,
      s.stream));
  if (q.nnz) {
    GB_CUDA_TRY(cudaMemcpyAsync(ri, q.rowind, 4ull * q.nnz, cudaMemcpyHostToDevice, s.stream));
    GB_CUDA_TRY(cudaMemcpyAsync(v64, q.val64, 8ull * q.nnz, cudaMemcpyHostToDevice, s.stream));
  }
  GB_CUDA_TRY(cudaMemcpyAsync(bb, q.b, 8ull * q.n, cudaMemcpyHostToDevice, s.stream));
  if (s.mixed && q.nnz) GB_TRY(launch_round_f32(v64, v32, q.nnz, s.stream));
  // the staging region goes back to the arena after the step's wait, when the
  // copies above are done; until every copy is queued the request keeps it
  if (q.stage_len) {
    s.stage_done.emplace_back(q.stage_off, q.stage_len);
    q.stage_len = 0;
  }
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
  S.a_work = kWorkInit;
  S.b_work = kWorkIdle;
  S.status = GB_CG_MAXITER;
  s.h_slots[k] = S;
  s.dirty = true;
  return GOOSEBERRY_SUCCESS;
}

// ---- the tile autotuner ------------------------------------------------------------
//
// Key: server mode, the request's longest row (rows of up to 5, 7, 15, 63 or
// 255 entries) and log2 of its row count.  A new key is tuned on the spot:
// the request is copied into a batch of R replicas (about 8M rows, at most
// 64), each with its own Krylov vectors (the matrix is shared), and for each
// candidate size the batch runs an INIT pair, one untimed CG pair and then
// kTuneIters CG iterations of both kernels, timed with CUDA events; the
// fastest size is cached for the process.

struct TileKey {
  bool mixed;
  uint32_t row_class, log2n;
  bool operator<(const TileKey & o) const {
    return std::tie(mixed, row_class, log2n) < std::tie(o.mixed, o.row_class, o.log2n);
  }
};
std::mutex g_tile_mu;
std::map<TileKey, uint32_t> g_tile_cache;
constexpr int kTuneIters = 6;

TileKey tile_key(bool mixed, uint32_t n, uint32_t maxrow) {
  const uint32_t rc = maxrow <= 5 ? 5 : maxrow <= 7 ? 7 : maxrow <= 15 ? 15 : maxrow <= 63 ? 63
                                                                                      : 255;
  uint32_t lg = 0;
  while ((2u << lg) <= n && lg < 31) ++lg;
  return TileKey{mixed, rc, lg};
}

uint32_t tuned_tile_rows(bool mixed, uint32_t n, uint32_t maxrow) {
  std::lock_guard<std::mutex> lock(g_tile_mu);
  auto it = g_tile_cache.find(tile_key(mixed, n, maxrow));
  return it == g_tile_cache.end() ? 0u : it->second;
}

// Times the candidate tile sizes on replicas of request q (see above).
int tune_tile_rows(gb_server & s, const Request & q, uint32_t * best) {
  const uint32_t n = q.n, nnz = q.nnz;
  std::vector<uint32_t> cands;
  for (uint32_t t = 1024; t <= 16384; t <<= 1) {
    cands.push_back(t);
    if (t >= n) break;
  }
  *best = cands.front();
  if (cands.size() == 1) return GOOSEBERRY_SUCCESS;
  const uint32_t R = static_cast<uint32_t>(std::max<uint64_t>(1, std::min<uint64_t>(64,
      8000000ull / n)));
  const size_t t = s.mixed ? 4 : 8;
  const size_t mat = align256(4ull * (n + 1)) + align256(4ull * nnz) + align256(8ull * nnz) +
                     align256(8ull * n) + (s.mixed ? align256(4ull * nnz) : 0);
  const size_t per = align256(8ull * n) * (s.mixed ? 2 : 1) + 5 * align256(t * n);
  const size_t max_tiles = static_cast<size_t>(R) * ((n + 1023) / 1024);
  const size_t meta = align256(R * sizeof(SrvSlot)) + align256(max_tiles * sizeof(SrvTile)) +
                      align256(2 * max_tiles * sizeof(double2)) + 256;
  char * mem = nullptr;
  GB_TRY(dev_alloc(&mem, mat + R * per + meta));
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  int rc = GOOSEBERRY_SUCCESS;
  auto fail = [&](cudaError_t e) {
    set_error("tile autotuning failed: %s", cudaGetErrorString(e));
    rc = GOOSEBERRY_ERROR_UNKNOWN;
  };
  size_t at = 0;
  uint32_t * rp = carve<uint32_t>(mem, at, n + 1);
  uint32_t * ri = carve<uint32_t>(mem, at, nnz);
  double * v64 = carve<double>(mem, at, nnz);
  double * bb = carve<double>(mem, at, n);
  float * v32 = s.mixed ? carve<float>(mem, at, nnz) : nullptr;
  std::vector<SrvSlot> hs(R);
  for (uint32_t k = 0; k < R; ++k) {
    SrvSlot & S = hs[k];
    std::memset(&S, 0, sizeof(S));
    S.rowptr = rp;
    S.rowind = ri;
    S.val64 = v64;
    S.val32 = v32;
    S.b = bb;
    S.x0 = carve<double>(mem, at, n);
    S.x1 = s.mixed ? carve<double>(mem, at, n) : nullptr;
    for (void ** v : {&S.y, &S.r, &S.p0, &S.p1, &S.ap}) {
      *v = mem + at;
      at += align256(t * n);
    }
    S.n = n;
  }
  SrvSlot * d_slots = carve<SrvSlot>(mem, at, R);
  SrvTile * d_tiles = carve<SrvTile>(mem, at, max_tiles);
  double2 * d_part = carve<double2>(mem, at, 2 * max_tiles);
  uint32_t * d_nt = carve<uint32_t>(mem, at, 1);
  cudaStream_t st = s.stream;
  cudaError_t e = cudaMemcpyAsync(rp, q.rowptr, 4ull * (n + 1), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess && nnz)
    e = cudaMemcpyAsync(ri, q.rowind, 4ull * nnz, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess && nnz)
    e = cudaMemcpyAsync(v64, q.val64, 8ull * nnz, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(bb, q.b, 8ull * n, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaEventCreate(&e0);
  if (e == cudaSuccess) e = cudaEventCreate(&e1);
  if (e != cudaSuccess) fail(e);
  if (rc == GOOSEBERRY_SUCCESS && s.mixed && nnz) rc = launch_round_f32(v64, v32, nnz, st);
  SrvDev d;
  d.slots = d_slots;
  d.tiles = d_tiles;
  d.ntiles = d_nt;
  d.pa = d_part;
  d.pb = d_part + max_tiles;
  std::vector<SrvTile> tiles;
  float best_ms = 1e30f;
  for (uint32_t T : cands) {
    if (rc != GOOSEBERRY_SUCCESS) break;
    tiles.clear();
    for (uint32_t k = 0; k < R; ++k) {
      SrvSlot & S = hs[k];
      S.tile0 = static_cast<uint32_t>(tiles.size());
      for (uint32_t r = 0; r < n; r += T) tiles.push_back(SrvTile{k, r, std::min(T, n - r), 0});
      S.ntiles = static_cast<uint32_t>(tiles.size()) - S.tile0;
      S.tol_rel = 0.0;  // never converges within the trial
      S.niter = ~0ull;
      S.live = 1;
      S.done = 0;
      S.a_work = kWorkInit;
      S.b_work = kWorkIdle;
      S.status = GB_CG_MAXITER;
      S.ticket_a = S.ticket_b = 0;
    }
    const uint32_t nt = static_cast<uint32_t>(tiles.size());
    e = cudaMemcpyAsync(d_slots, hs.data(), R * sizeof(SrvSlot), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(d_tiles, tiles.data(), nt * sizeof(SrvTile), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(d_nt, &nt, sizeof(uint32_t), cudaMemcpyHostToDevice, st);
    for (int k = 0; k < 2 + kTuneIters && e == cudaSuccess; ++k) {
      if (k == 2) e = cudaEventRecord(e0, st);
      if (e != cudaSuccess) break;
      if (s.mixed) {
        e = launch_k(srv_a_kernel<float, true>, s.grid_a, kSrvThreads, 0, st, false, d);
        if (e == cudaSuccess)
          e = launch_k(srv_b_kernel<float, true>, s.grid_b, kSrvThreads, 0, st, false, d);
      } else {
        e = launch_k(srv_a_kernel<double, false>, s.grid_a, kSrvThreads, 0, st, false, d);
        if (e == cudaSuccess)
          e = launch_k(srv_b_kernel<double, false>, s.grid_b, kSrvThreads, 0, st, false, d);
      }
    }
    if (e == cudaSuccess) e = cudaEventRecord(e1, st);
    if (e == cudaSuccess) e = cudaEventSynchronize(e1);
    float ms = 0.f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
    if (e != cudaSuccess) {
      fail(e);
      break;
    }
    if (ms < best_ms) {
      best_ms = ms;
      *best = T;
    }
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  cudaStreamSynchronize(st);  // the trial's memory is released below
  dev_free(mem);
  if (rc == GOOSEBERRY_SUCCESS) s.stats.tunings += 1;
  return rc;
}

// Tile rows for request q: the configured size, else the cached or freshly
// tuned size of its key (kTileRows when tuning cannot run).
int tile_rows_for(gb_server & s, const Request & q, uint32_t maxrow, uint32_t * out) {
  if (s.cfg.tile_rows) {
    *out = s.cfg.tile_rows;
    return GOOSEBERRY_SUCCESS;
  }
  const TileKey key = tile_key(s.mixed, q.n, maxrow);
  {
    std::lock_guard<std::mutex> lock(g_tile_mu);
    auto it = g_tile_cache.find(key);
    if (it != g_tile_cache.end()) {
      *out = it->second;
      return GOOSEBERRY_SUCCESS;
    }
  }
  uint32_t T = kTileRows;
  GB_TRY(tune_tile_rows(s, q, &T));
  std::lock_guard<std::mutex> lock(g_tile_mu);
  *out = g_tile_cache.emplace(key, T).first->second;  // a racing tuner's first entry wins
  return GOOSEBERRY_SUCCESS;
}

int cancel(gb_server & s, uint64_t id) {
  for (auto it = s.queue.begin(); it != s.queue.end(); ++it) {
    if (it->id != id) continue;
    gb_server_result_t res{};
    res.id = id;
    res.status = GB_CG_CANCELLED;
    res.t_submit = it->t_submit;
    res.t_admit = res.t_done = now_s(s);
    s.results.push_back(res);
    if (it->stage_len) s.stage_alloc.release(it->stage_off, it->stage_len);
    s.queue.erase(it);
    return GOOSEBERRY_SUCCESS;
  }
  for (auto & h : s.slots) {
    if (!h.used || h.id != id || h.cancel) continue;
    h.cancel = true;  // the step in flight may still run it; the next step retires it
    return GOOSEBERRY_SUCCESS;
  }
  set_error("no queued or resident request with id %llu", static_cast<unsigned long long>(id));
  return GOOSEBERRY_ERROR_INVALIDINPUT;
}

int step(gb_server & s, size_t * active, size_t * queued) {
  const auto t_in = std::chrono::steady_clock::now();
  double waited = 0.0;
  const bool drained = s.inflight;  // the wait below covers all earlier work on s.stream
  if (s.inflight) {
    GB_CUDA_TRY(cudaEventSynchronize(s.step_done));
    waited = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_in)
                 .count();
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, s.step_start, s.step_done) == cudaSuccess) s.stats.gpu_ms += ms;
    s.stats.wait_ms += waited;
    s.inflight = false;
  }
  if (!s.stage_done.empty()) {  // the admissions' copies ran before the replay waited on
    if (!drained) GB_CUDA_TRY(cudaStreamSynchronize(s.stream));
    for (const auto & r : s.stage_done) s.stage_alloc.release(r.first, r.second);
    s.stage_done.clear();
  }
  // 1. retire finished (or cancelled) solves: copy x out, free memory and
  //    the slot
  bool any_done = false;
  for (uint32_t k = 0; k < s.cfg.max_slots; ++k) {
    SlotHost & h = s.slots[k];
    const SrvSlot & S = s.h_slots[k];
    if (!h.used || !S.done) continue;  // a solve that finished before its cancel keeps x
    const double * x = (s.mixed && S.xpar) ? S.x1 : S.x0;
    GB_CUDA_TRY(cudaMemcpyAsync(h.x_out, x, 8ull * h.n, cudaMemcpyDeviceToHost, s.stream));
    any_done = true;
  }
  if (any_done) GB_CUDA_TRY(cudaStreamSynchronize(s.stream));
  for (uint32_t k = 0; k < s.cfg.max_slots; ++k) {
    SlotHost & h = s.slots[k];
    SrvSlot & S = s.h_slots[k];
    if (!h.used || !(S.done || h.cancel)) continue;
    gb_server_result_t res;
    res.id = h.id;
    res.iterations = S.iter;
    res.refinements = S.refinements;
    res.rnorm = std::sqrt(S.rr_true);
    res.bnorm = S.bnorm;
    res.status = S.done ? S.status : GB_CG_CANCELLED;
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
    GB_CUDA_TRY(cudaEventRecord(s.step_start, s.stream));
    GB_CUDA_TRY(cudaGraphLaunch(s.graph, s.stream));
    GB_CUDA_TRY(cudaMemcpyAsync(s.h_slots, s.d_slots, s.cfg.max_slots * sizeof(SrvSlot),
        cudaMemcpyDeviceToHost, s.stream));
    GB_CUDA_TRY(cudaEventRecord(s.step_done, s.stream));
    s.inflight = true;
    s.stats.steps += 1;
  }
  if (active) *active = nact;
  if (queued) *queued = s.queue.size();
  s.stats.host_ms += std::chrono::duration<double, std::milli>(
                         std::chrono::steady_clock::now() - t_in).count() - waited;
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
  const auto t0 = std::chrono::steady_clock::now();
  const int rc = gb::submit(*s, id, n, rowptr, rowind, rowval, b, x_out, tol_rel, niter);
  s->stats.submit_ms +=
      std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  return rc;
}

int gb_server_stats(const gb_server_t * s, gb_server_stats_t * out) {
  GB_CHECK_INPUT(s && out, "NULL argument");
  *out = s->stats;
  return GOOSEBERRY_SUCCESS;
}

int gb_server_tuned_tile_rows(int mode, uint32_t n, uint32_t max_row_nnz, uint32_t * tile_rows) {
  GB_CHECK_INPUT(tile_rows != nullptr, "NULL argument");
  GB_CHECK_INPUT(mode == GB_CG_MIXED || mode == GB_CG_F64, "mode must be GB_CG_MIXED or GB_CG_F64");
  *tile_rows = gb::tuned_tile_rows(mode == GB_CG_MIXED, n, max_row_nnz);
  return GOOSEBERRY_SUCCESS;
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

int gb_server_cancel(gb_server_t * s, uint64_t id) {
  GB_CHECK_INPUT(s != nullptr, "server is NULL");
  return gb::cancel(*s, id);
}

double gb_server_clock(const gb_server_t * s) { return s ? gb::now_s(*s) : 0.0; }

}  // extern "C"
