// cg.cu -- conjugate gradient on the device (reference cgd, src/cgd.c:40-129).
//
// The reference runs, per iteration, one SpMV, two dots, three scales, two
// add/sub passes and two copies, each its own OpenMP region
// (src/cgd.c:87-120).  Here one iteration is TWO kernels with no host
// round trip:
//
//   A  (SpMV + direction update + p.Ap)
//        p_new[i] = r[i] + beta * p_old[i]        (for every row i it owns)
//        Ap[i]    = sum_k val[k] * (r[c] + beta * p_old[c]),  c = ind[k]
//        partial  += p_new[i] * Ap[i]
//      The gathered p values are recomputed from r and p_old with the same
//      fma, so they equal p_new bit for bit; p is double-buffered so no CTA
//      reads a p value another CTA has already overwritten.  The last CTA to
//      finish (atomic ticket) sums the per-CTA partials in CTA order and
//      sets alpha = rr / p.Ap.
//   B  (solution / residual update + r.r)
//        x += alpha p_new;  r -= alpha Ap;  partial += r.r
//      The last CTA sets rr, beta = rr_new / rr, records ||r|| and decides
//      whether to stop (||r|| <= tol, iteration limit, breakdown, NaN).
//
// Both kernels return at once when the device-side stop flag is set, so a
// CUDA graph of K iterations can be replayed blindly: the host only reads
// the flag between graph launches (two graphs in flight), and the extra
// iterations after convergence cost one empty launch each.
//
// The stopping rule and iteration count follow the reference exactly: the
// first check happens after the first update, iteration k (0-based) is
// counted before its check, and the bound is on the absolute ||r||_2
// (src/cgd.c:87,115-119).
#include <algorithm>
#include <cmath>
#include <vector>

#include "gb_internal.h"
#include "spmv_tiles.cuh"
#include "cg_common.cuh"

namespace gb {

namespace {

struct CgState {
  double rr;         // r.r of the current residual
  double alpha;
  double beta;
  double tol;        // absolute bound on ||r||_2
  double bnorm;      // ||b||_2
  double pap;
  unsigned long long iter;   // iterations done
  unsigned long long niter;  // limit (0 = none)
  int done;          // 1: stop
  int status;        // gb_cg_status_t
  unsigned int ticket_a;
  unsigned int ticket_b;
  unsigned int ticket_i;
  unsigned int pad;
  double * hist;     // optional device history
  unsigned long long hist_len;
};

// Host mirror written by the graph after every chunk.
struct CgStatus {
  int done;
  int status;
  unsigned long long iter;
  double rr;
  double bnorm;
};

// ---- A: SpMV with fused direction update and p.Ap -----------------------------

struct GatherP {
  const double * r;
  const double * pold;
  double beta;
  template <class P>
  __device__ __forceinline__ double operator()(uint32_t c, P pol) const {
    return fma(beta, ld_keep(pold + c, pol), ld_keep(r + c, pol));
  }
};

struct OutCgA {
  double * ap;
  double * pnew;
  const double * r;
  const double * pold;
  double * longdot;
  double * partial;
  CgState * st;
  double beta;
  unsigned nlong;
  double local;
  __device__ __forceinline__ void row(uint32_t i, double v) {
    ap[i] = v;
    const double pn = fma(beta, pold[i], r[i]);
    pnew[i] = pn;
    local += pn * v;
  }
  __device__ __forceinline__ void long_row(uint32_t lid, uint32_t i, double v) {
    ap[i] = v;
    const double pn = fma(beta, pold[i], r[i]);
    pnew[i] = pn;
    longdot[lid] = pn * v;
  }
  struct Pre {
    double r, pold;
  };
  __device__ __forceinline__ Pre pre(uint32_t i) const { return Pre{r[i], pold[i]}; }
  __device__ __forceinline__ void row_pre(uint32_t i, double v, const Pre & q) {
    ap[i] = v;
    const double pn = fma(beta, q.pold, q.r);
    pnew[i] = pn;
    local += pn * v;
  }
  __device__ __forceinline__ void finish() {
    __shared__ double red[32];
    __shared__ bool last;
    const double s = block_sum(local, red);
    if (threadIdx.x == 0) partial[blockIdx.x] = s;
    if (!arrive_last(&st->ticket_a, &last)) return;
    __threadfence();
    double tot = ordered_sum(partial, gridDim.x, red);
    if (threadIdx.x == 0) {
      for (unsigned q = 0; q < nlong; ++q) tot += __ldcg(longdot + q);
      st->ticket_a = 0;
      st->pap = tot;
      const double rr = st->rr;
      if (!(tot > 0.0)) {
        st->done = 1;
        st->status = (tot == tot && rr == rr) ? GB_CG_BREAKDOWN : GB_CG_NONFINITE;
        st->alpha = 0.0;
      } else {
        st->alpha = rr / tot;
      }
    }
  }
};

template <int SCHED, bool HINT>
__global__ void __launch_bounds__(kSpmvBlock, MinBlocks<SCHED>::value) cg_a_kernel(const PlanView plan,
    const uint32_t * __restrict__ rowptr, const uint32_t * __restrict__ rowind,
    const double * __restrict__ val, const double * __restrict__ r,
    const double * __restrict__ pold, double * __restrict__ pnew,
    double * __restrict__ ap, double * __restrict__ longdot,
    double * __restrict__ partial, CgState * st) {
  pdl_wait_and_release();
  if (*reinterpret_cast<volatile int *>(&st->done)) return;
  const double beta = st->beta;
  GatherP g{r, pold, beta};
  // the row schedule finishes long rows through row() like any other row
  OutCgA o{ap, pnew, r, pold, longdot, partial, st, beta,
           SCHED == SCHED_ROW ? 0u : plan.nlong, 0.0};
  spmv_tiles_body<double, double, SCHED, kSpmvBlock, GatherP, OutCgA, false, HINT>(plan, rowptr,
      rowind, val, g, o);
}

// ---- B: x / r update and r.r ----------------------------------------------------

__global__ void __launch_bounds__(kVecBlock, kSpmvMinBlocks) cg_b_kernel(size_t n,
    double * __restrict__ x, double * __restrict__ r, const double * __restrict__ p,
    const double * __restrict__ ap, double * __restrict__ partial, CgState * st) {
  pdl_wait_and_release();
  if (*reinterpret_cast<volatile int *>(&st->done)) return;
  __shared__ double red[32];
  __shared__ bool last;
  const double alpha = st->alpha;
  // contiguous chunk per CTA (2-element units, 16-byte aligned pairs)
  const size_t units = (n + 1) / 2;
  const size_t q = units / gridDim.x, rem = units % gridDim.x;
  const size_t b = blockIdx.x;
  const size_t us = b * q + min(b, rem);
  const size_t ue = us + q + (b < rem ? 1 : 0);
  double acc = 0.0;
  const size_t full = n / 2;  // complete pairs
  const size_t ve = min(ue, full);
  // all loads of a batch are issued before any arithmetic (memory-level
  // parallelism: one round trip per batch)
  constexpr int U = 2;
  for (size_t base = us; base < ve; base += U * kVecBlock) {
    double2 pv[U], av[U], xv[U], rv[U];
#pragma unroll
    for (int j = 0; j < U; ++j) {
      const size_t u = base + threadIdx.x + j * kVecBlock;
      if (u < ve) {
        pv[j] = reinterpret_cast<const double2 *>(p)[u];
        av[j] = reinterpret_cast<const double2 *>(ap)[u];
        xv[j] = reinterpret_cast<const double2 *>(x)[u];
        rv[j] = reinterpret_cast<const double2 *>(r)[u];
      }
    }
#pragma unroll
    for (int j = 0; j < U; ++j) {
      const size_t u = base + threadIdx.x + j * kVecBlock;
      if (u < ve) {
        xv[j].x = fma(alpha, pv[j].x, xv[j].x);
        xv[j].y = fma(alpha, pv[j].y, xv[j].y);
        rv[j].x = fma(-alpha, av[j].x, rv[j].x);
        rv[j].y = fma(-alpha, av[j].y, rv[j].y);
        reinterpret_cast<double2 *>(x)[u] = xv[j];
        reinterpret_cast<double2 *>(r)[u] = rv[j];
        acc += rv[j].x * rv[j].x;
        acc += rv[j].y * rv[j].y;
      }
    }
  }
  if (ue > full && threadIdx.x == 0) {  // odd n: the last element
    const size_t i = 2 * full;
    x[i] = fma(alpha, p[i], x[i]);
    const double rn = fma(-alpha, ap[i], r[i]);
    r[i] = rn;
    acc += rn * rn;
  }
  const double s = block_sum(acc, red);
  if (threadIdx.x == 0) partial[blockIdx.x] = s;
  if (!arrive_last(&st->ticket_b, &last)) return;
  __threadfence();
  const double rr = ordered_sum(partial, gridDim.x, red);
  if (threadIdx.x == 0) {
    st->ticket_b = 0;
    const double rr_old = st->rr;
    st->beta = rr / rr_old;
    st->rr = rr;
    const unsigned long long it = st->iter + 1;
    st->iter = it;
    const double rnorm = sqrt(rr);
    if (st->hist && it <= st->hist_len) st->hist[it - 1] = rnorm;
    if (!(rnorm == rnorm) || isinf(rnorm)) {
      st->done = 1;
      st->status = GB_CG_NONFINITE;
    } else if (rnorm <= st->tol) {
      st->done = 1;
      st->status = GB_CG_CONVERGED;
    } else if (st->niter && it >= st->niter) {
      st->done = 1;
      st->status = GB_CG_MAXITER;
    }
  }
}

// ---- init: x = 0, r = b, p = 0, rr = b.b -----------------------------------------

__global__ void __launch_bounds__(kVecBlock) cg_init_kernel(size_t n,
    const double * __restrict__ b, double * __restrict__ x, double * __restrict__ r,
    double * __restrict__ p0, double * __restrict__ partial, CgState * st,
    int tol_relative) {
  __shared__ double red[32];
  __shared__ bool last;
  const size_t units = (n + 1) / 2;
  const size_t q = units / gridDim.x, rem = units % gridDim.x;
  const size_t bb = blockIdx.x;
  const size_t us = bb * q + min(bb, rem);
  const size_t ue = us + q + (bb < rem ? 1 : 0);
  double acc = 0.0;
  for (size_t u = us + threadIdx.x; u < ue; u += kVecBlock) {
    for (size_t i = 2 * u; i < min(n, 2 * u + 2); ++i) {
      const double bv = b[i];
      x[i] = 0.0;
      r[i] = bv;
      p0[i] = 0.0;
      acc += bv * bv;
    }
  }
  const double s = block_sum(acc, red);
  if (threadIdx.x == 0) partial[blockIdx.x] = s;
  if (!arrive_last(&st->ticket_i, &last)) return;
  __threadfence();
  const double rr = ordered_sum(partial, gridDim.x, red);
  if (threadIdx.x == 0) {
    st->ticket_i = 0;
    st->rr = rr;
    st->bnorm = sqrt(rr);
    st->beta = 0.0;
    st->alpha = 0.0;
    st->iter = 0;
    if (tol_relative) st->tol = st->tol * st->bnorm;
    st->done = 0;
    st->status = GB_CG_MAXITER;
    if (rr == 0.0) {  // b == 0: x = 0 is exact
      st->done = 1;
      st->status = GB_CG_CONVERGED;
    } else if (!(rr == rr) || isinf(rr)) {
      st->done = 1;
      st->status = GB_CG_NONFINITE;
    }
  }
}

// dynamic shared memory of the SpMV phase (the row schedule stages nothing)
size_t spmv_smem(int sched, uint32_t tile_items) {
  return spmv_smem_bytes<double, double>(sched, tile_items, kSpmvBlock);
}

template <int SCHED, bool HINT>
int launch_cg_a_t(const gb_csr & a, const double * r, const double * pold, double * pnew,
    double * ap, double * longdot, double * partial, CgState * st, unsigned grid,
    cudaStream_t s, bool pdl) {
  const size_t smem = spmv_smem(SCHED, a.plan.tile_items);
  auto kern = cg_a_kernel<SCHED, HINT>;
  if (smem > 48 * 1024)
    GB_CUDA_TRY(cudaFuncSetAttribute(reinterpret_cast<const void *>(kern),
        cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
  GB_CUDA_TRY(launch_k(kern, grid, kSpmvBlock, smem, s, pdl, plan_view(a), a.rowptr,
      a.rowind, a.val64, r, pold, pnew, ap, longdot, partial, st));
  return GOOSEBERRY_SUCCESS;
}

template <bool HINT>
int launch_cg_a_h(const gb_csr & a, int sched, const double * r, const double * pold,
    double * pnew, double * ap, double * longdot, double * partial, CgState * st,
    unsigned grid, cudaStream_t s, bool pdl) {
  switch (sched) {
    case GB_SCHED_THREAD:
      return launch_cg_a_t<SCHED_THREAD, HINT>(a, r, pold, pnew, ap, longdot, partial, st, grid, s,
          pdl);
    case GB_SCHED_GROUP4:
      return launch_cg_a_t<SCHED_GROUP4, HINT>(a, r, pold, pnew, ap, longdot, partial, st, grid, s,
          pdl);
    case GB_SCHED_GROUP8:
      return launch_cg_a_t<SCHED_GROUP8, HINT>(a, r, pold, pnew, ap, longdot, partial, st, grid, s,
          pdl);
    case GB_SCHED_WARP:
      return launch_cg_a_t<SCHED_WARP, HINT>(a, r, pold, pnew, ap, longdot, partial, st, grid, s,
          pdl);
    case GB_SCHED_ROW:
      return launch_cg_a_t<SCHED_ROW, HINT>(a, r, pold, pnew, ap, longdot, partial, st, grid, s,
          pdl);
    case GB_SCHED_WTILE:
      return launch_cg_a_t<SCHED_WTILE, HINT>(a, r, pold, pnew, ap, longdot, partial, st, grid, s,
          pdl);
    default:
      return launch_cg_a_t<SCHED_MERGE, HINT>(a, r, pold, pnew, ap, longdot, partial, st, grid, s,
          pdl);
  }
}

// The A kernel with L2-policy loads (hint) or plain loads.
int launch_cg_a(const gb_csr & a, int sched, bool hint, const double * r, const double * pold,
    double * pnew, double * ap, double * longdot, double * partial, CgState * st,
    unsigned grid, cudaStream_t s, bool pdl) {
  return hint ? launch_cg_a_h<true>(a, sched, r, pold, pnew, ap, longdot, partial, st, grid, s,
                                    pdl)
              : launch_cg_a_h<false>(a, sched, r, pold, pnew, ap, longdot, partial, st, grid,
                                     s, pdl);
}

template <int SCHED>
int occupancy_cg_a(size_t smem, int * out) {
  auto kern = cg_a_kernel<SCHED, false>;
  if (smem > 48 * 1024)
    GB_CUDA_TRY(cudaFuncSetAttribute(reinterpret_cast<const void *>(kern),
        cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
  GB_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(out, kern, kSpmvBlock, smem));
  return GOOSEBERRY_SUCCESS;
}

int occupancy_cg_a_sched(int sched, size_t smem, int * out) {
  switch (sched) {
    case GB_SCHED_THREAD: return occupancy_cg_a<SCHED_THREAD>(smem, out);
    case GB_SCHED_GROUP4: return occupancy_cg_a<SCHED_GROUP4>(smem, out);
    case GB_SCHED_GROUP8: return occupancy_cg_a<SCHED_GROUP8>(smem, out);
    case GB_SCHED_WARP: return occupancy_cg_a<SCHED_WARP>(smem, out);
    case GB_SCHED_ROW: return occupancy_cg_a<SCHED_ROW>(smem, out);
    case GB_SCHED_WTILE: return occupancy_cg_a<SCHED_WTILE>(smem, out);
    default: return occupancy_cg_a<SCHED_MERGE>(smem, out);
  }
}

// ---- persistent solve: the whole CG in one cooperative launch -------------------
//
// Every CTA owns a contiguous run of tiles (and so a contiguous run of rows)
// for the whole solve.  Per iteration:
//   phase A  SpMV of its tiles with the fused direction update, p.Ap partial
//   barrier  every CTA then sums the G partials itself, in CTA order, so all
//            CTAs hold the same alpha without a serial last-CTA step
//   phase B  x += alpha p, r -= alpha Ap on its own rows, r.r partial
//   barrier  every CTA sums r.r, forms beta and takes the same stop decision
// Vectors that other CTAs write during the launch (r, p) are read through L2
// (ld.global.cg), never the read-only path.  Barriers wait on a global
// counter with a 2 s limit; on time-out the CTA raises `abort`, every waiting
// CTA leaves, and the solve reports GB_CG_NONFINITE with rnorm = NaN.

constexpr unsigned long long kBarrierTimeoutNs = 2000000000ull;

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned * p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ double ld_cg(const double * p, uint64_t pol) {
  double v;
  asm volatile("ld.global.cg.L2::cache_hint.f64 %0, [%1], %2;" : "=d"(v) : "l"(p), "l"(pol));
  return v;
}

// Grid barrier number `epoch` (1, 2, ...): returns false if it was abandoned.
__device__ __forceinline__ bool grid_barrier(unsigned * counter, int * abort_flag,
    unsigned epoch, int * ok_smem) {
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    atomicAdd(counter, 1u);
    const unsigned target = epoch * gridDim.x;
    const unsigned long long t0 = global_ns();
    int ok = 1;
    unsigned polls = 0;
    while (ld_acquire_u32(counter) < target) {
      if (*reinterpret_cast<volatile int *>(abort_flag)) { ok = 0; break; }
      if (++polls > 64) {
        __nanosleep(64);
        if (global_ns() - t0 > kBarrierTimeoutNs) {
          atomicExch(abort_flag, 1);
          ok = 0;
          break;
        }
      }
    }
    __threadfence();
    *ok_smem = ok;
  }
  __syncthreads();
  return *ok_smem != 0;
}

// Sum of partial[0..n) in index order, identical in every CTA; all threads
// receive the result.
__device__ __forceinline__ double ordered_allsum(const double * partial, unsigned n,
    double * red, double * bcast) {
  const unsigned per = (n + blockDim.x - 1) / blockDim.x;
  const unsigned s = min(n, threadIdx.x * per), e = min(n, s + per);
  double acc = 0.0;
  for (unsigned i = s; i < e; ++i) acc += __ldcg(partial + i);
  acc = block_sum(acc, red);
  if (threadIdx.x == 0) *bcast = acc;
  __syncthreads();
  return *bcast;
}

struct GatherPcg {
  const double * r;
  const double * pold;
  double beta;
  __device__ __forceinline__ double operator()(uint32_t c, uint64_t pol) const {
    return fma(beta, ld_cg(pold + c, pol), ld_cg(r + c, pol));
  }
};

struct OutPersistA {
  double * ap;
  double * pnew;
  const double * r;
  const double * pold;
  double beta;
  double local;
  __device__ __forceinline__ void row(uint32_t i, double v) {
    ap[i] = v;
    const double pn = fma(beta, __ldcg(pold + i), __ldcg(r + i));
    pnew[i] = pn;
    local += pn * v;
  }
  __device__ __forceinline__ void long_row(uint32_t, uint32_t i, double v) { row(i, v); }
  __device__ __forceinline__ void finish() {}
  struct Pre {
    double r, pold;
  };
  __device__ __forceinline__ Pre pre(uint32_t i) const {
    return Pre{__ldcg(r + i), __ldcg(pold + i)};
  }
  __device__ __forceinline__ void row_pre(uint32_t i, double v, const Pre & q) {
    ap[i] = v;
    const double pn = fma(beta, q.pold, q.r);
    pnew[i] = pn;
    local += pn * v;
  }
};

struct PersistArgs {
  PlanView plan;
  const uint32_t * rowptr;
  const uint32_t * rowind;
  const double * val;
  const double * b;
  double * x;
  double * r;
  double * p0;
  double * p1;
  double * ap;
  double * partial_a;
  double * partial_b;
  const uint32_t * cta_tiles;  // [G + 1]
  unsigned * sync;
  int * abort_flag;
  CgState * st;
  int tol_relative;
  int keep_matrix_in_l2;
};

template <int SCHED>
__global__ void __launch_bounds__(kSpmvBlock, MinBlocks<SCHED>::value) cg_persistent_kernel(const PersistArgs a) {
  __shared__ double red[32];
  __shared__ double bcast;
  __shared__ int ok_smem;
  const unsigned G = gridDim.x, cta = blockIdx.x;
  const int tid = threadIdx.x;
  const uint32_t t0 = a.cta_tiles[cta], t1 = a.cta_tiles[cta + 1];
  uint32_t lo = 0, hi = 0;
  if (t0 < t1) {
    lo = a.plan.tiles[t0].row_begin;
    const TileDesc last = a.plan.tiles[t1 - 1];
    hi = last.row_begin + last.row_count;
  }
  const uint64_t pol_x = policy_evict_last();
  const uint64_t pol_m = a.keep_matrix_in_l2 ? policy_evict_last() : policy_evict_first();
  const double tol_in = a.st->tol;
  const unsigned long long niter = a.st->niter;
  double * const hist = a.st->hist;
  const unsigned long long hist_len = a.st->hist_len;

  // phase 0: x = 0, r = b, p = 0, rr = b.b
  double acc = 0.0;
  for (uint32_t i = lo + tid; i < hi; i += kSpmvBlock) {
    const double bv = a.b[i];
    a.x[i] = 0.0;
    a.r[i] = bv;
    a.p0[i] = 0.0;
    acc += bv * bv;
  }
  acc = block_sum(acc, red);
  if (tid == 0) a.partial_b[cta] = acc;
  unsigned epoch = 0;
  int status = GB_CG_MAXITER;
  unsigned long long it = 0;
  double rr = 0.0, bnorm = 0.0, tol = tol_in, beta = 0.0;
  bool aborted = false;
  if (!grid_barrier(a.sync, a.abort_flag, ++epoch, &ok_smem)) {
    aborted = true;
  } else {
    rr = ordered_allsum(a.partial_b, G, red, &bcast);
    bnorm = sqrt(rr);
    if (a.tol_relative) tol = tol_in * bnorm;
    if (rr == 0.0) status = GB_CG_CONVERGED;
    else if (!(rr == rr) || isinf(rr)) status = GB_CG_NONFINITE;
    bool running = (rr != 0.0) && (rr == rr) && !isinf(rr);
    while (running) {
      double * pold = (it & 1) ? a.p1 : a.p0;
      double * pnew = (it & 1) ? a.p0 : a.p1;
      // phase A
      GatherPcg g{a.r, pold, beta};
      OutPersistA o{a.ap, pnew, a.r, pold, beta, 0.0};
      if (SCHED == SCHED_ROW)
        spmv_row_loop<double, double>(lo + tid, hi, kSpmvBlock, a.plan.ncols, a.rowptr,
            a.rowind, a.val, g, o, pol_m, pol_x);
      else if (SCHED == SCHED_WTILE)
        spmv_warp_loop<double, double>(a.plan, t0 + (tid >> 5), t1, kSpmvBlock / 32,
            a.rowptr, a.rowind, a.val, g, o, pol_m, pol_x);
      else
        spmv_tile_loop<double, double, SCHED, kSpmvBlock>(a.plan, t0, t1, 1, a.rowptr,
            a.rowind, a.val, g, o, pol_m, pol_x);
      double s = block_sum(o.local, red);
      if (tid == 0) a.partial_a[cta] = s;
      if (!grid_barrier(a.sync, a.abort_flag, ++epoch, &ok_smem)) { aborted = true; break; }
      const double pap = ordered_allsum(a.partial_a, G, red, &bcast);
      if (!(pap > 0.0)) {
        status = (pap == pap && rr == rr) ? GB_CG_BREAKDOWN : GB_CG_NONFINITE;
        break;
      }
      const double alpha = rr / pap;
      // phase B
      acc = 0.0;
      constexpr int U = 4;
      for (uint32_t base = lo; base < hi; base += U * kSpmvBlock) {
        double pv[U], av[U], xv[U], rv[U];
#pragma unroll
        for (int j = 0; j < U; ++j) {
          const uint32_t i = base + tid + j * kSpmvBlock;
          if (i < hi) {
            pv[j] = __ldcg(pnew + i);
            av[j] = __ldcg(a.ap + i);
            xv[j] = __ldcg(a.x + i);
            rv[j] = __ldcg(a.r + i);
          }
        }
#pragma unroll
        for (int j = 0; j < U; ++j) {
          const uint32_t i = base + tid + j * kSpmvBlock;
          if (i < hi) {
            a.x[i] = fma(alpha, pv[j], xv[j]);
            const double rn = fma(-alpha, av[j], rv[j]);
            a.r[i] = rn;
            acc += rn * rn;
          }
        }
      }
      s = block_sum(acc, red);
      if (tid == 0) a.partial_b[cta] = s;
      if (!grid_barrier(a.sync, a.abort_flag, ++epoch, &ok_smem)) { aborted = true; break; }
      const double rr_new = ordered_allsum(a.partial_b, G, red, &bcast);
      beta = rr_new / rr;
      rr = rr_new;
      ++it;
      const double rnorm = sqrt(rr);
      if (cta == 0 && tid == 0 && hist && it <= hist_len) hist[it - 1] = rnorm;
      if (!(rnorm == rnorm) || isinf(rnorm)) { status = GB_CG_NONFINITE; running = false; }
      else if (rnorm <= tol) { status = GB_CG_CONVERGED; running = false; }
      else if (niter && it >= niter) { status = GB_CG_MAXITER; running = false; }
    }
  }
  if (cta == 0 && tid == 0) {
    CgState * st = a.st;
    st->iter = it;
    st->rr = aborted ? __longlong_as_double(0x7ff8000000000000ll) : rr;
    st->bnorm = bnorm;
    st->tol = tol;
    st->status = aborted ? GB_CG_NONFINITE : status;
    st->done = 1;
  }
}

template <int SCHED>
int persistent_setup_t(size_t smem, int * occ, const void ** fn) {
  auto kern = cg_persistent_kernel<SCHED>;
  *fn = reinterpret_cast<const void *>(kern);
  if (smem > 48 * 1024)
    GB_CUDA_TRY(cudaFuncSetAttribute(*fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
        static_cast<int>(smem)));
  GB_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(occ, kern, kSpmvBlock, smem));
  return GOOSEBERRY_SUCCESS;
}

int persistent_setup(int sched, size_t smem, int * occ, const void ** fn) {
  switch (sched) {
    case GB_SCHED_THREAD: return persistent_setup_t<SCHED_THREAD>(smem, occ, fn);
    case GB_SCHED_GROUP4: return persistent_setup_t<SCHED_GROUP4>(smem, occ, fn);
    case GB_SCHED_GROUP8: return persistent_setup_t<SCHED_GROUP8>(smem, occ, fn);
    case GB_SCHED_WARP: return persistent_setup_t<SCHED_WARP>(smem, occ, fn);
    case GB_SCHED_ROW: return persistent_setup_t<SCHED_ROW>(smem, occ, fn);
    case GB_SCHED_WTILE: return persistent_setup_t<SCHED_WTILE>(smem, occ, fn);
    default: return persistent_setup_t<SCHED_MERGE>(smem, occ, fn);
  }
}

}  // namespace

}  // namespace gb

// ---- solver object ----------------------------------------------------------------

struct gb_cg {
  const gb_csr * a = nullptr;
  int mode = GB_CG_F64;
  size_t n = 0;
  double * x = nullptr;
  double * r = nullptr;
  double * p[2] = {nullptr, nullptr};
  double * ap = nullptr;
  double * partial_a = nullptr;
  double * partial_b = nullptr;
  double * partial_i = nullptr;
  double * longdot = nullptr;
  gb::CgState * st = nullptr;
  gb::CgStatus * host_status = nullptr;  // pinned, [2] slots
  unsigned grid_a = 0, grid_b = 0;
  int sched = GB_SCHED_MERGE;
  uint32_t tile_items = 0;
  int chunk = 32;  // iterations per graph (even)
  cudaStream_t cap_stream = nullptr;
  cudaGraphExec_t graph[2] = {nullptr, nullptr};  // status into slot 0 / slot 1
  // persistent (one cooperative launch per solve) mode
  bool persistent = false;
  unsigned grid_p = 0;
  size_t smem_p = 0;
  const void * fn_p = nullptr;
  uint32_t * cta_tiles = nullptr;
  unsigned * sync = nullptr;  // [0] barrier counter, [1] abort flag
  int keep_l2 = 0;
  bool l2_hint = false;  // A kernel with L2-policy loads (working set fits in L2)
  gb::MixedCg * mixed = nullptr;  // GB_CG_MIXED solver (owns its workspace)
};

namespace gb {
namespace {

void destroy_cg(gb_cg * s) {
  if (!s) return;
  cudaDeviceSynchronize();  // its memory goes back to the pool below
  mixed_destroy(s->mixed);
  for (auto & g : s->graph)
    if (g) cudaGraphExecDestroy(g);
  if (s->cap_stream) cudaStreamDestroy(s->cap_stream);
  dev_free(s->x);
  dev_free(s->r);
  dev_free(s->p[0]);
  dev_free(s->p[1]);
  dev_free(s->ap);
  dev_free(s->partial_a);
  dev_free(s->partial_b);
  dev_free(s->partial_i);
  dev_free(s->longdot);
  dev_free(s->st);
  dev_free(s->cta_tiles);
  dev_free(s->sync);
  if (s->host_status) cudaFreeHost(s->host_status);
  delete s;
}

// One chunk of iterations (A, B per iteration) and the status mirror into
// host_status[slot], on the capture stream cs.
int enqueue_chunk(gb_cg * s, int slot, cudaStream_t cs) {
  int rc = GOOSEBERRY_SUCCESS;
  for (int k = 0; k < s->chunk && rc == GOOSEBERRY_SUCCESS; ++k) {
    const double * pold = s->p[k & 1];
    double * pnew = s->p[(k + 1) & 1];
    rc = launch_cg_a(*s->a, s->sched, s->l2_hint, s->r, pold, pnew, s->ap, s->longdot, s->partial_a,
        s->st, s->grid_a, cs, k > 0);
    if (rc != GOOSEBERRY_SUCCESS) break;
    if (launch_k(cg_b_kernel, s->grid_b, kVecBlock, 0, cs, true, s->n, s->x, s->r,
            static_cast<const double *>(pnew), static_cast<const double *>(s->ap),
            s->partial_b, s->st) != cudaSuccess)
      rc = GOOSEBERRY_ERROR_UNKNOWN;
  }
  if (rc == GOOSEBERRY_SUCCESS) {
    // status mirror: done, status, iter, rr, bnorm
    cudaMemcpyAsync(&s->host_status[slot].done, &s->st->done, sizeof(int),
        cudaMemcpyDeviceToHost, cs);
    cudaMemcpyAsync(&s->host_status[slot].status, &s->st->status, sizeof(int),
        cudaMemcpyDeviceToHost, cs);
    cudaMemcpyAsync(&s->host_status[slot].iter, &s->st->iter, sizeof(unsigned long long),
        cudaMemcpyDeviceToHost, cs);
    cudaMemcpyAsync(&s->host_status[slot].rr, &s->st->rr, sizeof(double),
        cudaMemcpyDeviceToHost, cs);
    cudaMemcpyAsync(&s->host_status[slot].bnorm, &s->st->bnorm, sizeof(double),
        cudaMemcpyDeviceToHost, cs);
  }
  return rc;
}

int capture_chunk(gb_cg * s, int slot) {
  cudaStream_t cs = s->cap_stream;
  GB_CUDA_TRY(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
  const int rc = enqueue_chunk(s, slot, cs);
  cudaGraph_t g = nullptr;
  cudaError_t e = cudaStreamEndCapture(cs, &g);
  if (rc != GOOSEBERRY_SUCCESS) {
    if (g) cudaGraphDestroy(g);
    set_error("CG graph capture failed: %s", cudaGetErrorString(cudaGetLastError()));
    return GOOSEBERRY_ERROR_UNKNOWN;
  }
  GB_CUDA_TRY(e);
  e = cudaGraphInstantiate(&s->graph[slot], g, 0);
  cudaGraphDestroy(g);
  GB_CUDA_TRY(e);
  return GOOSEBERRY_SUCCESS;
}

// One cooperative launch per solve when every row fits a tile (no long rows)
// and all CTAs of the grid can be resident at once.  Tiles are dealt to CTAs
// in contiguous runs of nearly equal rows + nonzeros.
int setup_persistent(const gb_csr * a, gb_cg * s) {
  int dev = 0, coop = 0;
  GB_CUDA_TRY(cudaGetDevice(&dev));
  GB_CUDA_TRY(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
  const size_t ntiles = a->plan.tiles.size();
  if (!coop || !a->plan.longrows.empty() || ntiles == 0) return GOOSEBERRY_SUCCESS;
  s->smem_p = spmv_smem(s->sched, a->plan.tile_items);
  int occ = 0;
  GB_TRY(persistent_setup(s->sched, s->smem_p, &occ, &s->fn_p));
  if (occ < 1) return GOOSEBERRY_SUCCESS;
  const unsigned G = static_cast<unsigned>(std::min<size_t>(ntiles,
      static_cast<size_t>(a->sm_count) * occ));
  std::vector<uint64_t> cum(ntiles + 1, 0);
  for (size_t t = 0; t < ntiles; ++t)
    cum[t + 1] = cum[t] + a->plan.tiles[t].row_count + a->plan.tiles[t].nnz_count;
  std::vector<uint32_t> bounds(G + 1, 0);
  size_t t = 0;
  for (unsigned g = 1; g < G; ++g) {
    const uint64_t want = cum[ntiles] * g / G;
    while (t < ntiles && cum[t] < want) ++t;
    bounds[g] = static_cast<uint32_t>(std::max<size_t>(t, bounds[g - 1]));
  }
  bounds[G] = static_cast<uint32_t>(ntiles);
  GB_TRY(dev_alloc(&s->cta_tiles, (G + 1) * sizeof(uint32_t)));
  GB_CUDA_TRY(cudaMemcpy(s->cta_tiles, bounds.data(), (G + 1) * sizeof(uint32_t),
      cudaMemcpyHostToDevice));
  GB_TRY(dev_alloc(&s->sync, 2 * sizeof(unsigned)));
  // the matrix stays L2-resident across iterations when the working set of
  // one iteration fits in about 3/4 of L2
  int l2 = 0;
  GB_CUDA_TRY(cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, dev));
  const double ws = 4.0 * (a->nrows + 1) + 12.0 * a->nnz + 40.0 * a->nrows;
#ifndef GB_L2_KEEP_FRACTION
#define GB_L2_KEEP_FRACTION 0.75
#endif
  s->keep_l2 = ws <= GB_L2_KEEP_FRACTION * l2 ? 1 : 0;
  s->grid_p = G;
  s->persistent = true;
  return GOOSEBERRY_SUCCESS;
}

int launch_persistent(gb_cg * s, const double * b, int tol_relative, cudaStream_t stream) {
  GB_CUDA_TRY(cudaMemsetAsync(s->sync, 0, 2 * sizeof(unsigned), stream));
  PersistArgs args;
  args.plan = plan_view(*s->a);
  args.rowptr = s->a->rowptr;
  args.rowind = s->a->rowind;
  args.val = s->a->val64;
  args.b = b;
  args.x = s->x;
  args.r = s->r;
  args.p0 = s->p[0];
  args.p1 = s->p[1];
  args.ap = s->ap;
  args.partial_a = s->partial_a;
  args.partial_b = s->partial_b;
  args.cta_tiles = s->cta_tiles;
  args.sync = s->sync;
  args.abort_flag = reinterpret_cast<int *>(s->sync + 1);
  args.st = s->st;
  args.tol_relative = tol_relative;
  args.keep_matrix_in_l2 = s->keep_l2;
  void * kargs[] = {&args};
  GB_CUDA_TRY(cudaLaunchCooperativeKernel(s->fn_p, dim3(s->grid_p), dim3(kSpmvBlock), kargs,
      s->smem_p, stream));
  return GOOSEBERRY_SUCCESS;
}

int create_cg(const gb_csr * a, int mode, gb_cg * s) {
  GB_CHECK_INPUT(a->nrows == a->ncols, "CG needs a square matrix, got %ux%u", a->nrows,
      a->ncols);
  const bool want_persistent = (mode & GB_CG_PERSISTENT) != 0;
  mode &= ~GB_CG_PERSISTENT;
  GB_CHECK_INPUT(mode == GB_CG_F64 || mode == GB_CG_MIXED, "unknown CG mode %d", mode);
  if (mode == GB_CG_MIXED) {
    s->a = a;
    s->mode = mode;
    s->n = a->nrows;
    return mixed_create(a, &s->mixed);
  }
  GB_CHECK_INPUT(a->val64 != nullptr, "CG (FP64) needs double values on the matrix");
  s->a = a;
  s->mode = mode;
  s->n = a->nrows;
  const size_t n = std::max<size_t>(s->n, 2);
  GB_TRY(dev_alloc(&s->x, n * sizeof(double)));
  GB_TRY(dev_alloc(&s->r, n * sizeof(double)));
  GB_TRY(dev_alloc(&s->p[0], n * sizeof(double)));
  GB_TRY(dev_alloc(&s->p[1], n * sizeof(double)));
  GB_TRY(dev_alloc(&s->ap, n * sizeof(double)));
  s->sched = a->sched64;
  s->tile_items = a->plan.tile_items;
  // evict-first/evict-last hints keep an L2-sized working set (matrix, rowptr,
  // r, both p, Ap, x) resident across iterations; beyond L2 the plain loads win
  GB_TRY(l2_fits(4ull * (s->n + 1) + 12ull * a->nnz + 40ull * s->n, &s->l2_hint));
  const size_t smem = spmv_smem(s->sched, a->plan.tile_items);
  int occ = 0;
  GB_TRY(occupancy_cg_a_sched(s->sched, smem, &occ));
  GB_CHECK_INPUT(occ > 0, "CG kernel cannot be resident");
  const unsigned ntiles = static_cast<unsigned>(std::max<size_t>(a->plan.tiles.size(), 1));
  const unsigned work_a = spmv_work_units(s->sched, static_cast<uint32_t>(s->n), ntiles,
      kSpmvBlock);
  s->grid_a = std::min<unsigned>(std::max(work_a, 1u),
      static_cast<unsigned>(a->sm_count * occ));
  const size_t units = (s->n + 1) / 2;
  // vector kernels: one resident wave, each CTA streaming a contiguous chunk
  int occ_b = 0;
  GB_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_b, cg_b_kernel, kVecBlock, 0));
  s->grid_b = static_cast<unsigned>(std::max<size_t>(1, std::min<size_t>(
      (units + kVecBlock - 1) / kVecBlock,
      static_cast<size_t>(a->sm_count) * std::max(occ_b, 1))));
  const unsigned gmax = std::max<unsigned>(std::max(s->grid_a, s->grid_b),
      static_cast<unsigned>(std::min<size_t>(a->plan.tiles.size() + 1,
          static_cast<size_t>(a->sm_count) * 32)));
  GB_TRY(dev_alloc(&s->partial_a, gmax * sizeof(double)));
  GB_TRY(dev_alloc(&s->partial_b, gmax * sizeof(double)));
  GB_TRY(dev_alloc(&s->partial_i, gmax * sizeof(double)));
  GB_TRY(dev_alloc(&s->longdot,
      std::max<size_t>(a->plan.longrows.size(), 1) * sizeof(double)));
  GB_TRY(dev_alloc(&s->st, sizeof(CgState)));
  GB_CUDA_TRY(cudaMemset(s->st, 0, sizeof(CgState)));
  GB_CUDA_TRY(cudaMallocHost(&s->host_status, 2 * sizeof(CgStatus)));
  if (want_persistent) GB_TRY(setup_persistent(a, s));
  if (!s->persistent) {
    GB_CUDA_TRY(cudaStreamCreateWithFlags(&s->cap_stream, cudaStreamNonBlocking));
    GB_TRY(capture_chunk(s, 0));
    GB_TRY(capture_chunk(s, 1));
  }
  return GOOSEBERRY_SUCCESS;
}

int start_solve(gb_cg * s, const double * b, double tol, int tol_relative, size_t niter,
    double * dhist, size_t hl, cudaStream_t stream) {
  // niter == 0 means "no limit" as in the reference; a solve that can never
  // reach its tolerance is still stopped after max(1000, 100 n) iterations so
  // the caller cannot hang.
  const size_t cap = std::max<size_t>(1000, 100 * s->n);
  CgState init{};
  init.tol = tol;
  init.niter = niter ? niter : cap;
  init.hist = dhist;
  init.hist_len = hl;
  GB_CUDA_TRY(cudaMemcpyAsync(s->st, &init, sizeof(CgState), cudaMemcpyHostToDevice, stream));
  if (s->persistent) return launch_persistent(s, b, tol_relative, stream);
  cg_init_kernel<<<s->grid_b, kVecBlock, 0, stream>>>(s->n, b, s->x, s->r, s->p[0],
      s->partial_i, s->st, tol_relative);
  GB_CUDA_TRY(cudaGetLastError());
  return GOOSEBERRY_SUCCESS;
}

int solve_cg(gb_cg * s, const double * b, double * x, double tol, int tol_relative,
    size_t niter, double * history, size_t history_len, gb_cg_result_t * res,
    cudaStream_t stream) {
  if (s->mixed)
    return mixed_solve(s->mixed, b, x, tol, tol_relative, niter, history, history_len, res,
        stream);
  GB_CHECK_INPUT(s->n == 0 || (b && x), "NULL vector");
  GB_CHECK_INPUT(s->a->sched64 == s->sched && s->a->plan.tile_items == s->tile_items,
      "matrix schedule changed after the solver was created");
  if (s->n == 0) {
    if (res) *res = gb_cg_result_t{0, 0, 0.0, 0.0, GB_CG_CONVERGED, 0};
    return GOOSEBERRY_SUCCESS;
  }
  double * dhist = nullptr;
  const size_t hl = history ? std::min(history_len, niter ? niter : history_len) : 0;
  if (hl) GB_TRY(scratch_alloc(reinterpret_cast<void **>(&dhist), hl * sizeof(double), stream));
  GB_TRY(start_solve(s, b, tol, tol_relative, niter, dhist, hl, stream));
  size_t launches = 1;

  // two graphs in flight; the host reads the status mirror of the older one
  cudaEvent_t ev[2];
  GB_CUDA_TRY(cudaEventCreateWithFlags(&ev[0], cudaEventDisableTiming));
  GB_CUDA_TRY(cudaEventCreateWithFlags(&ev[1], cudaEventDisableTiming));
  int rc = GOOSEBERRY_SUCCESS;
  s->host_status[0].done = s->host_status[1].done = 0;
  auto launch = [&](int slot) -> int {
    cudaError_t e = cudaGraphLaunch(s->graph[slot], stream);
    if (e == cudaSuccess) e = cudaEventRecord(ev[slot], stream);
    launches += 2 * static_cast<size_t>(s->chunk);
    if (e != cudaSuccess) {
      set_error("CG graph launch failed: %s", cudaGetErrorString(e));
      return GOOSEBERRY_ERROR_UNKNOWN;
    }
    return GOOSEBERRY_SUCCESS;
  };
  if (!s->persistent) {
    rc = launch(0);
    if (rc == GOOSEBERRY_SUCCESS) rc = launch(1);
  }
  int slot = 0;
  while (rc == GOOSEBERRY_SUCCESS && !s->persistent) {
    cudaError_t e = cudaEventSynchronize(ev[slot]);
    if (e != cudaSuccess) {
      set_error("CG solve failed: %s", cudaGetErrorString(e));
      rc = GOOSEBERRY_ERROR_UNKNOWN;
      break;
    }
    if (s->host_status[slot].done) break;
    rc = launch(slot);
    slot ^= 1;
  }
  cudaError_t e = cudaStreamSynchronize(stream);
  cudaEventDestroy(ev[0]);
  cudaEventDestroy(ev[1]);
  if (rc == GOOSEBERRY_SUCCESS && e != cudaSuccess) {
    set_error("CG solve failed: %s", cudaGetErrorString(e));
    rc = GOOSEBERRY_ERROR_UNKNOWN;
  }
  if (rc == GOOSEBERRY_SUCCESS) {
    CgState fin{};
    e = cudaMemcpy(&fin, s->st, sizeof(CgState), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpyAsync(x, s->x, s->n * sizeof(double),
        cudaMemcpyDeviceToDevice, stream);
    if (e == cudaSuccess && hl && fin.iter)
      e = cudaMemcpyAsync(history, dhist, std::min<size_t>(hl, fin.iter) * sizeof(double),
          cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    unsigned flags[2] = {0, 0};
    if (e == cudaSuccess && s->persistent)
      e = cudaMemcpy(flags, s->sync, sizeof(flags), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) {
      set_error("CG result copy failed: %s", cudaGetErrorString(e));
      rc = GOOSEBERRY_ERROR_UNKNOWN;
    } else if (flags[1]) {
      set_error("CG solve abandoned: a grid barrier timed out");
      rc = GOOSEBERRY_ERROR_UNKNOWN;
    } else if (res) {
      res->iterations = fin.iter;
      res->refinements = 0;
      res->rnorm = std::sqrt(fin.rr);
      res->bnorm = fin.bnorm;
      res->status = fin.status;
      res->kernel_launches = launches;
    }
  }
  if (dhist) scratch_free(dhist, stream);
  return rc;
}

int profile_cg(gb_cg * s, const double * b, size_t iterations, double * ms, size_t ms_len,
    size_t * nkernels, cudaStream_t stream) {
  GB_CHECK_INPUT(s->n > 0 && b != nullptr, "profile needs a non-empty system and b");
  GB_CHECK_INPUT(iterations > 0, "iterations must be positive");
  if (s->mixed) return mixed_profile(s->mixed, b, iterations, ms, ms_len, nkernels, stream);
  if (s->persistent) {
    // one launch runs every iteration: time it and report ms per iteration
    if (nkernels) *nkernels = 1;
    cudaEvent_t e0, e1;
    GB_CUDA_TRY(cudaEventCreate(&e0));
    GB_CUDA_TRY(cudaEventCreate(&e1));
    GB_CUDA_TRY(cudaEventRecord(e0, stream));
    int rc = start_solve(s, b, 0.0, 0, iterations, nullptr, 0, stream);
    cudaEventRecord(e1, stream);
    cudaError_t e = cudaEventSynchronize(e1);
    float t = 0.f;
    if (rc == GOOSEBERRY_SUCCESS && e == cudaSuccess) cudaEventElapsedTime(&t, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    GB_TRY(rc);
    GB_CUDA_TRY(e);
    if (ms && ms_len > 0) ms[0] = static_cast<double>(t) / iterations;
    return GOOSEBERRY_SUCCESS;
  }
  if (nkernels) *nkernels = 2;
  GB_TRY(start_solve(s, b, 0.0, 0, 0, nullptr, 0, stream));
  std::vector<cudaEvent_t> ev(3 * iterations);
  for (auto & e : ev) GB_CUDA_TRY(cudaEventCreate(&e));
  int rc = GOOSEBERRY_SUCCESS;
  for (size_t k = 0; k < iterations && rc == GOOSEBERRY_SUCCESS; ++k) {
    const double * pold = s->p[k & 1];
    double * pnew = s->p[(k + 1) & 1];
    cudaEventRecord(ev[3 * k], stream);
    rc = launch_cg_a(*s->a, s->sched, s->l2_hint, s->r, pold, pnew, s->ap, s->longdot, s->partial_a,
        s->st, s->grid_a, stream, false);
    cudaEventRecord(ev[3 * k + 1], stream);
    cg_b_kernel<<<s->grid_b, kVecBlock, 0, stream>>>(s->n, s->x, s->r, pnew, s->ap,
        s->partial_b, s->st);
    cudaEventRecord(ev[3 * k + 2], stream);
  }
  cudaError_t e = cudaStreamSynchronize(stream);
  if (rc == GOOSEBERRY_SUCCESS && e != cudaSuccess) {
    set_error("CG profile failed: %s", cudaGetErrorString(e));
    rc = GOOSEBERRY_ERROR_UNKNOWN;
  }
  double ta = 0.0, tb = 0.0;
  if (rc == GOOSEBERRY_SUCCESS) {
    for (size_t k = 0; k < iterations; ++k) {
      float a = 0.f, bb = 0.f;
      cudaEventElapsedTime(&a, ev[3 * k], ev[3 * k + 1]);
      cudaEventElapsedTime(&bb, ev[3 * k + 1], ev[3 * k + 2]);
      ta += a;
      tb += bb;
    }
    if (ms && ms_len > 0) ms[0] = ta / iterations;
    if (ms && ms_len > 1) ms[1] = tb / iterations;
  }
  for (auto & ee : ev) cudaEventDestroy(ee);
  return rc;
}

}  // namespace
}  // namespace gb

extern "C" {

int gb_cg_create(const gb_csr_t * a, int mode, gb_cg_t ** out) {
  GB_CHECK_INPUT(a && out, "NULL argument");
  *out = nullptr;
  gb_cg * s = new gb_cg();
  int rc = gb::create_cg(a, mode, s);
  if (rc != GOOSEBERRY_SUCCESS) {
    gb::destroy_cg(s);
    return rc;
  }
  *out = s;
  return GOOSEBERRY_SUCCESS;
}

int gb_cg_destroy(gb_cg_t * s) {
  gb::destroy_cg(s);
  return GOOSEBERRY_SUCCESS;
}

int gb_cg_solve(gb_cg_t * s, const double * b, double * x, double tol, int tol_relative,
    size_t niter, double * history, size_t history_len, gb_cg_result_t * result,
    gb_stream_t stream) {
  GB_CHECK_INPUT(s != nullptr, "solver is NULL");
  return gb::solve_cg(s, b, x, tol, tol_relative, niter, history, history_len, result,
      static_cast<cudaStream_t>(stream));
}

int gb_cg_profile(gb_cg_t * s, const double * b, size_t iterations, double * ms,
    size_t ms_len, size_t * nkernels, gb_stream_t stream) {
  GB_CHECK_INPUT(s != nullptr, "solver is NULL");
  return gb::profile_cg(s, b, iterations, ms, ms_len, nkernels,
      static_cast<cudaStream_t>(stream));
}

}  // extern "C"
