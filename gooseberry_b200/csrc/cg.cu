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

constexpr int kVecBlock = 256;

// Returns true in thread 0 of the last CTA to arrive (ticket pattern).
__device__ __forceinline__ bool arrive_last(unsigned int * ticket, bool * flag) {
  __threadfence();
  if (threadIdx.x == 0) {
    const unsigned prev = atomicAdd(ticket, 1u);
    *flag = (prev == gridDim.x - 1);
  }
  __syncthreads();
  return *flag;
}

// Sum of partial[0..n) in index order, by one CTA; result valid in thread 0.
__device__ __forceinline__ double ordered_sum(const double * partial, unsigned n,
    double * red) {
  // each thread sums a contiguous run, then runs are summed in thread order
  const unsigned per = (n + blockDim.x - 1) / blockDim.x;
  const unsigned s = min(n, threadIdx.x * per), e = min(n, s + per);
  double acc = 0.0;
  for (unsigned i = s; i < e; ++i) acc += __ldcg(partial + i);
  // ordered combine: warp tree is order-fixed as well
  return block_sum(acc, red);
}

// ---- A: SpMV with fused direction update and p.Ap -----------------------------

struct GatherP {
  const double * r;
  const double * pold;
  double beta;
  __device__ __forceinline__ double operator()(uint32_t c, uint64_t pol) const {
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

template <int SCHED>
__global__ void __launch_bounds__(kSpmvBlock) cg_a_kernel(const PlanView plan,
    const uint32_t * __restrict__ rowptr, const uint32_t * __restrict__ rowind,
    const double * __restrict__ val, const double * __restrict__ r,
    const double * __restrict__ pold, double * __restrict__ pnew,
    double * __restrict__ ap, double * __restrict__ longdot,
    double * __restrict__ partial, CgState * st) {
  if (*reinterpret_cast<volatile int *>(&st->done)) return;
  const double beta = st->beta;
  GatherP g{r, pold, beta};
  OutCgA o{ap, pnew, r, pold, longdot, partial, st, beta, plan.nlong, 0.0};
  spmv_tiles_body<double, double, SCHED, kSpmvBlock>(plan, rowptr, rowind, val, g, o);
}

// ---- B: x / r update and r.r ----------------------------------------------------

__global__ void __launch_bounds__(kVecBlock) cg_b_kernel(size_t n,
    double * __restrict__ x, double * __restrict__ r, const double * __restrict__ p,
    const double * __restrict__ ap, double * __restrict__ partial, CgState * st) {
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
  for (size_t u = us + threadIdx.x; u < ue; u += kVecBlock) {
    if (u < full) {
      const double2 pv = reinterpret_cast<const double2 *>(p)[u];
      const double2 av = reinterpret_cast<const double2 *>(ap)[u];
      double2 xv = reinterpret_cast<double2 *>(x)[u];
      double2 rv = reinterpret_cast<double2 *>(r)[u];
      xv.x = fma(alpha, pv.x, xv.x);
      xv.y = fma(alpha, pv.y, xv.y);
      rv.x = fma(-alpha, av.x, rv.x);
      rv.y = fma(-alpha, av.y, rv.y);
      reinterpret_cast<double2 *>(x)[u] = xv;
      reinterpret_cast<double2 *>(r)[u] = rv;
      acc += rv.x * rv.x;
      acc += rv.y * rv.y;
    } else {
      const size_t i = 2 * u;  // odd tail element
      x[i] = fma(alpha, p[i], x[i]);
      const double rn = fma(-alpha, ap[i], r[i]);
      r[i] = rn;
      acc += rn * rn;
    }
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

template <int SCHED>
int launch_cg_a_t(const gb_csr & a, const double * r, const double * pold, double * pnew,
    double * ap, double * longdot, double * partial, CgState * st, unsigned grid,
    cudaStream_t s) {
  const size_t smem = TileSmem<double>::bytes(a.plan.tile_items);
  auto kern = cg_a_kernel<SCHED>;
  if (smem > 48 * 1024)
    GB_CUDA_TRY(cudaFuncSetAttribute(reinterpret_cast<const void *>(kern),
        cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
  kern<<<grid, kSpmvBlock, smem, s>>>(plan_view(a), a.rowptr, a.rowind, a.val64, r, pold,
      pnew, ap, longdot, partial, st);
  GB_CUDA_TRY(cudaGetLastError());
  return GOOSEBERRY_SUCCESS;
}

int launch_cg_a(const gb_csr & a, int sched, const double * r, const double * pold,
    double * pnew, double * ap, double * longdot, double * partial, CgState * st,
    unsigned grid, cudaStream_t s) {
  switch (sched) {
    case GB_SCHED_THREAD:
      return launch_cg_a_t<SCHED_THREAD>(a, r, pold, pnew, ap, longdot, partial, st, grid, s);
    case GB_SCHED_GROUP4:
      return launch_cg_a_t<SCHED_GROUP4>(a, r, pold, pnew, ap, longdot, partial, st, grid, s);
    case GB_SCHED_GROUP8:
      return launch_cg_a_t<SCHED_GROUP8>(a, r, pold, pnew, ap, longdot, partial, st, grid, s);
    case GB_SCHED_WARP:
      return launch_cg_a_t<SCHED_WARP>(a, r, pold, pnew, ap, longdot, partial, st, grid, s);
    default:
      return launch_cg_a_t<SCHED_MERGE>(a, r, pold, pnew, ap, longdot, partial, st, grid, s);
  }
}

template <int SCHED>
int occupancy_cg_a(size_t smem, int * out) {
  auto kern = cg_a_kernel<SCHED>;
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
    default: return occupancy_cg_a<SCHED_MERGE>(smem, out);
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
};

namespace gb {
namespace {

void destroy_cg(gb_cg * s) {
  if (!s) return;
  for (auto & g : s->graph)
    if (g) cudaGraphExecDestroy(g);
  if (s->cap_stream) cudaStreamDestroy(s->cap_stream);
  cudaFree(s->x);
  cudaFree(s->r);
  cudaFree(s->p[0]);
  cudaFree(s->p[1]);
  cudaFree(s->ap);
  cudaFree(s->partial_a);
  cudaFree(s->partial_b);
  cudaFree(s->partial_i);
  cudaFree(s->longdot);
  cudaFree(s->st);
  if (s->host_status) cudaFreeHost(s->host_status);
  delete s;
}

int capture_chunk(gb_cg * s, int slot) {
  cudaStream_t cs = s->cap_stream;
  GB_CUDA_TRY(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
  int rc = GOOSEBERRY_SUCCESS;
  for (int k = 0; k < s->chunk && rc == GOOSEBERRY_SUCCESS; ++k) {
    const double * pold = s->p[k & 1];
    double * pnew = s->p[(k + 1) & 1];
    rc = launch_cg_a(*s->a, s->sched, s->r, pold, pnew, s->ap, s->longdot, s->partial_a,
        s->st, s->grid_a, cs);
    if (rc != GOOSEBERRY_SUCCESS) break;
    cg_b_kernel<<<s->grid_b, kVecBlock, 0, cs>>>(s->n, s->x, s->r, pnew, s->ap,
        s->partial_b, s->st);
    if (cudaGetLastError() != cudaSuccess) rc = GOOSEBERRY_ERROR_UNKNOWN;
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

int create_cg(const gb_csr * a, int mode, gb_cg * s) {
  GB_CHECK_INPUT(a->nrows == a->ncols, "CG needs a square matrix, got %ux%u", a->nrows,
      a->ncols);
  GB_CHECK_INPUT(mode == GB_CG_F64, "CG mode %d is not available", mode);
  GB_CHECK_INPUT(a->val64 != nullptr, "CG (FP64) needs double values on the matrix");
  s->a = a;
  s->mode = mode;
  s->n = a->nrows;
  const size_t n = std::max<size_t>(s->n, 2);
  GB_CUDA_TRY(cudaMalloc(&s->x, n * sizeof(double)));
  GB_CUDA_TRY(cudaMalloc(&s->r, n * sizeof(double)));
  GB_CUDA_TRY(cudaMalloc(&s->p[0], n * sizeof(double)));
  GB_CUDA_TRY(cudaMalloc(&s->p[1], n * sizeof(double)));
  GB_CUDA_TRY(cudaMalloc(&s->ap, n * sizeof(double)));
  s->sched = a->sched64;
  s->tile_items = a->plan.tile_items;
  const size_t smem = TileSmem<double>::bytes(a->plan.tile_items);
  int occ = 0;
  GB_TRY(occupancy_cg_a_sched(s->sched, smem, &occ));
  GB_CHECK_INPUT(occ > 0, "CG kernel cannot be resident");
  const unsigned ntiles = static_cast<unsigned>(std::max<size_t>(a->plan.tiles.size(), 1));
  s->grid_a = std::min<unsigned>(ntiles, static_cast<unsigned>(a->sm_count * occ));
  const size_t units = (s->n + 1) / 2;
  s->grid_b = static_cast<unsigned>(std::max<size_t>(1, std::min<size_t>(
      (units + kVecBlock * 2 - 1) / (kVecBlock * 2), static_cast<size_t>(a->sm_count) * 8)));
  const unsigned gmax = std::max(s->grid_a, s->grid_b);
  GB_CUDA_TRY(cudaMalloc(&s->partial_a, gmax * sizeof(double)));
  GB_CUDA_TRY(cudaMalloc(&s->partial_b, gmax * sizeof(double)));
  GB_CUDA_TRY(cudaMalloc(&s->partial_i, gmax * sizeof(double)));
  GB_CUDA_TRY(cudaMalloc(&s->longdot,
      std::max<size_t>(a->plan.longrows.size(), 1) * sizeof(double)));
  GB_CUDA_TRY(cudaMalloc(&s->st, sizeof(CgState)));
  GB_CUDA_TRY(cudaMemset(s->st, 0, sizeof(CgState)));
  GB_CUDA_TRY(cudaMallocHost(&s->host_status, 2 * sizeof(CgStatus)));
  GB_CUDA_TRY(cudaStreamCreateWithFlags(&s->cap_stream, cudaStreamNonBlocking));
  GB_TRY(capture_chunk(s, 0));
  GB_TRY(capture_chunk(s, 1));
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
  cg_init_kernel<<<s->grid_b, kVecBlock, 0, stream>>>(s->n, b, s->x, s->r, s->p[0],
      s->partial_i, s->st, tol_relative);
  GB_CUDA_TRY(cudaGetLastError());
  return GOOSEBERRY_SUCCESS;
}

int solve_cg(gb_cg * s, const double * b, double * x, double tol, int tol_relative,
    size_t niter, double * history, size_t history_len, gb_cg_result_t * res,
    cudaStream_t stream) {
  GB_CHECK_INPUT(s->n == 0 || (b && x), "NULL vector");
  GB_CHECK_INPUT(s->a->sched64 == s->sched && s->a->plan.tile_items == s->tile_items,
      "matrix schedule changed after the solver was created");
  if (s->n == 0) {
    if (res) *res = gb_cg_result_t{0, 0, 0.0, 0.0, GB_CG_CONVERGED, 0};
    return GOOSEBERRY_SUCCESS;
  }
  double * dhist = nullptr;
  const size_t hl = history ? std::min(history_len, niter ? niter : history_len) : 0;
  if (hl) GB_CUDA_TRY(cudaMallocAsync(reinterpret_cast<void **>(&dhist), hl * sizeof(double),
      stream));
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
  rc = launch(0);
  if (rc == GOOSEBERRY_SUCCESS) rc = launch(1);
  int slot = 0;
  while (rc == GOOSEBERRY_SUCCESS) {
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
    if (e != cudaSuccess) {
      set_error("CG result copy failed: %s", cudaGetErrorString(e));
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
  if (dhist) cudaFreeAsync(dhist, stream);
  return rc;
}

int profile_cg(gb_cg * s, const double * b, size_t iterations, double * ms, size_t ms_len,
    size_t * nkernels, cudaStream_t stream) {
  GB_CHECK_INPUT(s->n > 0 && b != nullptr, "profile needs a non-empty system and b");
  GB_CHECK_INPUT(iterations > 0, "iterations must be positive");
  if (nkernels) *nkernels = 2;
  GB_TRY(start_solve(s, b, 0.0, 0, 0, nullptr, 0, stream));
  std::vector<cudaEvent_t> ev(3 * iterations);
  for (auto & e : ev) GB_CUDA_TRY(cudaEventCreate(&e));
  int rc = GOOSEBERRY_SUCCESS;
  for (size_t k = 0; k < iterations && rc == GOOSEBERRY_SUCCESS; ++k) {
    const double * pold = s->p[k & 1];
    double * pnew = s->p[(k + 1) & 1];
    cudaEventRecord(ev[3 * k], stream);
    rc = launch_cg_a(*s->a, s->sched, s->r, pold, pnew, s->ap, s->longdot, s->partial_a,
        s->st, s->grid_a, stream);
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
