// cg_mixed.cu -- mixed-precision CG: FP32 inner iterations, FP64 refinement.
//
// Same iteration as the reference's cgd (src/cgd.c:87-120), but the matrix
// values and the Krylov vectors of the inner loop are FP32 (half the bytes of
// an FP64 iteration), while everything that decides accuracy stays FP64:
//
//   * the dots p.Ap and r.r are accumulated in FP64 (alpha, beta, ||r||);
//   * the solution is x (FP64) + y (FP32 correction since the last update);
//   * a "reliable update" (Sleijpen & van der Vorst, 1996) replaces the
//     iterated FP32 residual by the true one whenever ||r|| has dropped by
//     kDelta below its largest value since the last update, or looks
//     converged:  x <- x + y,  r = b - A x  computed with the FP64 values and
//     FP64 accumulation, then rounded to FP32.  The search direction is kept,
//     so the Krylov process continues instead of restarting, and convergence
//     is only ever declared on the true FP64 residual.
//
// Per iteration two kernels, graph-captured 32 at a time with programmatic
// dependent launch:
//   A32  the iteration's scalar step from B32's r.r partials (beta, ||r||, the
//        stop test and the reliable-update decision, identical in every CTA),
//        then the FP32 SpMV with the fused direction update and p.Ap in FP64;
//   B32  alpha from A32's partials; y += alpha p, r -= alpha Ap, r.r in FP64.
// A reliable update takes one pair of launches of its own: A32 decides it and
// does no SpMV, and B32 computes r = b - A (x + y) with the FP64 values and
// FP64 accumulation over its rows, x <- x + y (into the other x buffer, so no
// CTA reads an x another CTA already changed), the FP32 rounding of r and the
// true r.r partials, which the next A32 turns into the true ||r||, the
// convergence test and beta.  No kernel has a serial last-CTA step: every CTA
// of the next kernel sums the per-CTA partials itself in the same fixed
// order, so all CTAs hold the same alpha / beta / decision.  The scalars are
// kept in two versions: A32 launch k reads version k & 1 and its CTA 0 writes
// version (k + 1) & 1, which B32 launch k reads, so no CTA reads a value
// another CTA of the same kernel is rewriting.  The R kernel (FP64 residual
// over the matrix's SpMV schedule) folds a pending correction into x when a
// solve stops at its iteration limit, and times the FP64 residual for the
// profiler.
#include <algorithm>
#include <cmath>
#include <vector>

#include "gb_internal.h"
#include "spmv_tiles.cuh"
#include "cg_common.cuh"

namespace gb {

namespace {

constexpr double kDelta = 0.1;  // reliable update when ||r|| < kDelta * max ||r||

// The scalars of one iteration (two versions, see above).
// What the pair of launches governed by a version does.
enum : int { kPhaseCg = 0, kPhaseRefresh = 1, kPhaseFirst = 2 };

struct MixScalars {
  double rr_hat;      // ||r||^2 of the FP32 residual the directions are built on
  double rr_hat_old;  // its value one iteration earlier
  double beta;
  double rmax;        // largest ||r|| since the last reliable update
  unsigned long long iter;
  int phase;          // kPhaseCg: a CG iteration; kPhaseRefresh: a reliable
                      // update (B32 recomputes r in FP64); kPhaseFirst: the
                      // init kernel's version (A32 takes no step from it)
  int y_reset;        // y was folded into x: the next B starts y afresh
};

struct MixState {
  MixScalars sv[2];
  double tol;         // absolute bound on the true ||b - A x||
  double bnorm;
  double rr_true;     // ||b - A x||^2 at the last reliable update
  unsigned long long iter;  // iterations done (host mirror; written by A32's CTA 0)
  unsigned long long niter;
  unsigned long long refinements;
  int done;
  int status;
  int xpar;           // index of the current x buffer
  int ver;            // the version the last A32 wrote (the current one)
  unsigned ticket_r, ticket_i;
  double * hist;
  unsigned long long hist_len;
};

// R launch modes: the final fold the host requests when a solve stops with a
// pending FP32 correction, and the profiler's (the FP64 residual alone).
enum : int { kRFold = 1, kRProfile = 2 };

// The stop flag, read once per CTA so that all of its threads agree.
__device__ __forceinline__ bool mix_cta_done(const MixState * st) {
  __shared__ int s_done;
  if (threadIdx.x == 0) s_done = *reinterpret_cast<const volatile int *>(&st->done);
  __syncthreads();
  return s_done != 0;
}

struct MixStatus {
  int done;
  int status;
  unsigned long long iter;
};

// ---- A32 ----------------------------------------------------------------------

// The scalar step of A32 launch k from B32 launch k-1's partials: version
// `par` in, version par ^ 1 out (CTA 0 writes it).  Identical in every CTA.
// Returns true when this launch runs the CG SpMV (beta in *beta); false when
// the solve stopped or this pair of launches is a reliable update.
__device__ __forceinline__ bool mix_a_step(MixState * st, int par,
    const double * __restrict__ partial_b, unsigned nb, float * beta) {
  __shared__ double red[32];
  __shared__ double s_rr;
  const MixScalars cur = st->sv[par];
  MixScalars nv = cur;
  int stop = -1;
  if (cur.phase != kPhaseFirst) {
    const double rr_sum = ordered_sum(partial_b, nb, red);
    if (threadIdx.x == 0) s_rr = rr_sum;
    __syncthreads();
    const double rr = s_rr;
    const double rnorm = sqrt(rr);
    const bool finite = rnorm == rnorm && !isinf(rnorm);
    if (cur.phase == kPhaseRefresh) {
      // B32 recomputed r = b - A x in FP64 (src/cgd.c:115-119 stops on it):
      // continue from the true residual, keeping the search direction
      nv.phase = kPhaseCg;
      nv.y_reset = 1;
      nv.beta = rr / cur.rr_hat_old;
      nv.rr_hat = rr;
      nv.rmax = rnorm;
      if (!finite) stop = GB_CG_NONFINITE;
      else if (rnorm <= st->tol) stop = GB_CG_CONVERGED;
      else if (st->niter && cur.iter >= st->niter) stop = GB_CG_MAXITER;
      if (blockIdx.x == 0 && threadIdx.x == 0) {
        st->rr_true = rr;
        st->refinements += 1;
        st->xpar ^= 1;
        if (st->hist && cur.iter >= 1 && cur.iter <= st->hist_len) st->hist[cur.iter - 1] = rnorm;
      }
    } else {
      // a CG iteration finished: beta, ||r|| and the reliable-update test
      const unsigned long long it = cur.iter + 1;
      nv.phase = kPhaseCg;
      nv.y_reset = 0;
      nv.iter = it;
      nv.rr_hat_old = cur.rr_hat;
      nv.beta = rr / cur.rr_hat;
      nv.rr_hat = rr;
      nv.rmax = fmax(cur.rmax, rnorm);
      if (!finite) stop = GB_CG_NONFINITE;
      else if (rnorm <= st->tol || rnorm < kDelta * nv.rmax) nv.phase = kPhaseRefresh;
      else if (st->niter && it >= st->niter) stop = GB_CG_MAXITER;
      if (blockIdx.x == 0 && threadIdx.x == 0) {
        st->iter = it;
        if (st->hist && it <= st->hist_len) st->hist[it - 1] = rnorm;
      }
    }
  } else {
    nv.phase = kPhaseCg;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    st->sv[par ^ 1] = nv;
    st->ver = par ^ 1;
    if (stop >= 0) {
      st->status = stop;
      st->done = 1;
    }
  }
  *beta = static_cast<float>(nv.beta);
  return stop < 0 && nv.phase == kPhaseCg;
}

struct GatherP32 {
  const float * r;
  const float * pold;
  float beta;
  template <class P>
  __device__ __forceinline__ float operator()(uint32_t c, P pol) const {
    return fmaf(beta, ld_keep(pold + c, pol), ld_keep(r + c, pol));
  }
};

struct OutA32 {
  float * ap;
  float * pnew;
  const float * r;
  const float * pold;
  double * longdot;
  double * partial;
  MixState * st;
  float beta;
  unsigned nlong;
  double local;
  __device__ __forceinline__ void row(uint32_t i, float v) {
    ap[i] = v;
    const float pn = fmaf(beta, pold[i], r[i]);
    pnew[i] = pn;
    local += static_cast<double>(pn) * static_cast<double>(v);
  }
  __device__ __forceinline__ void long_row(uint32_t lid, uint32_t i, float v) {
    ap[i] = v;
    const float pn = fmaf(beta, pold[i], r[i]);
    pnew[i] = pn;
    longdot[lid] = static_cast<double>(pn) * static_cast<double>(v);
  }
  struct Pre {
    float r, pold;
  };
  __device__ __forceinline__ Pre pre(uint32_t i) const { return Pre{r[i], pold[i]}; }
  __device__ __forceinline__ void row_pre(uint32_t i, float v, const Pre & q) {
    ap[i] = v;
    const float pn = fmaf(beta, q.pold, q.r);
    pnew[i] = pn;
    local += static_cast<double>(pn) * static_cast<double>(v);
  }
  __device__ __forceinline__ void finish() {
    __shared__ double red[32];
    const double s = block_sum(local, red);
    if (threadIdx.x == 0) partial[blockIdx.x] = s;
  }
};

template <int SCHED, bool HINT>
__global__ void __launch_bounds__(kSpmvBlock, MinBlocks<SCHED>::value) cg_a32_kernel(
    const PlanView plan, const uint32_t * __restrict__ rowptr,
    const uint32_t * __restrict__ rowind, const float * __restrict__ val,
    const float * __restrict__ r, const float * __restrict__ pold, float * __restrict__ pnew,
    float * __restrict__ ap, double * __restrict__ longdot, double * __restrict__ partial,
    MixState * st, int par, const double * __restrict__ partial_b, unsigned nb) {
  pdl_wait_and_release();
  if (mix_cta_done(st)) return;
  float beta;
  if (!mix_a_step(st, par, partial_b, nb, &beta)) return;
  GatherP32 g{r, pold, beta};
  OutA32 o{ap, pnew, r, pold, longdot, partial, st, beta,
           SCHED == SCHED_ROW ? 0u : plan.nlong, 0.0};
  spmv_tiles_body<float, float, SCHED, kSpmvBlock, GatherP32, OutA32, false, HINT>(plan, rowptr,
      rowind, val, g, o);
}

// A32 on the row schedule over compressed columns: a pattern byte per row
// (ColPat8, stencils) or 16-bit column distances (ColD16): the same products
// and sums as cg_a32_kernel<SCHED_ROW>, 4 or 2 bytes less per nonzero.  Four
// CTAs per SM (64 registers, no spills): the FP32 rows are short chains of
// dependent loads, and more of them in flight measured 4 % faster than three
// CTAs (five spill).
#ifndef GB_MIX_PAT_MIN_BLOCKS
#define GB_MIX_PAT_MIN_BLOCKS 5
#endif
// Over row patterns the stage holds one code per row instead of a column per
// entry: 48 registers, five CTAs per SM.
template <class IC>
struct MixAMinBlocks {
  static constexpr int value = IC::kPerRow ? GB_MIX_PAT_MIN_BLOCKS : 4;
};

template <class IC, bool HINT, int STAGE>
__global__ void __launch_bounds__(kSpmvBlock, MixAMinBlocks<IC>::value) cg_a32_c_kernel(
    const PlanView plan, const uint32_t * __restrict__ rowptr, IC ic,
    const int32_t * __restrict__ pat_off, uint32_t npat, const float * __restrict__ val,
    const float * __restrict__ r, const float * __restrict__ pold, float * __restrict__ pnew,
    float * __restrict__ ap, double * __restrict__ longdot, double * __restrict__ partial,
    MixState * st, int par, const double * __restrict__ partial_b, unsigned nb) {
  if constexpr (IC::kPerRow) {
    __shared__ int32_t s_pat[256 * kPatMax];
    for (uint32_t i = threadIdx.x; i < npat * kPatMax; i += kSpmvBlock) s_pat[i] = pat_off[i];
    ic.off = s_pat;
    __syncthreads();
  }
  pdl_wait_and_release();
  if (mix_cta_done(st)) return;
  float beta;
  if (!mix_a_step(st, par, partial_b, nb, &beta)) return;
  GatherP32 g{r, pold, beta};
  OutA32 o{ap, pnew, r, pold, longdot, partial, st, beta, 0u, 0.0};
  spmv_row_loop_c<float, STAGE>(blockIdx.x * kSpmvBlock + threadIdx.x, plan.nrows,
      gridDim.x * kSpmvBlock, plan.ncols, rowptr, ic, ValPlain<float>{val}, g, o,
      L2Pol<HINT>::stream(), L2Pol<HINT>::keep());
  o.finish();
}

#ifndef GB_MIX_ELL
#define GB_MIX_ELL 1
#endif
// A32 over row patterns with the FP32 values in rows of 8 (ELL): row i's
// values at v8[8 i ...], zero-padded, its length and column offsets from the
// pattern table.  No rowptr: a row's values arrive with two 16-byte loads
// whose address depends on nothing but i.  The same products, sums, epilogue
// and partials as cg_a32_c_kernel<ColPat8>, so the iterates are identical.
// On the 160^3 operator A32 went from 54.7 to 46.0 us (the same bytes: the
// padding costs what rowptr saved; the row's loads no longer wait on rowptr
// and there are 9 fewer load instructions per row).
__global__ void ell_values_kernel(uint32_t n, const uint32_t * __restrict__ rowptr,
    const float * __restrict__ val, float4 * __restrict__ v8) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint32_t b = __ldg(rowptr + i), e = __ldg(rowptr + i + 1);
    float v[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) v[j] = b + j < e ? __ldg(val + b + j) : 0.0f;
    v8[2 * static_cast<size_t>(i)] = make_float4(v[0], v[1], v[2], v[3]);
    v8[2 * static_cast<size_t>(i) + 1] = make_float4(v[4], v[5], v[6], v[7]);
  }
}

template <bool HINT, int STAGE>
__global__ void __launch_bounds__(kSpmvBlock, GB_MIX_PAT_MIN_BLOCKS) cg_a32_ell_kernel(
    uint32_t nrows, const uint8_t * __restrict__ code, const int32_t * __restrict__ pat_off,
    uint32_t npat, const float4 * __restrict__ v8, const float * __restrict__ r,
    const float * __restrict__ pold, float * __restrict__ pnew, float * __restrict__ ap,
    double * __restrict__ partial, MixState * st, int par, const double * __restrict__ partial_b,
    unsigned nb) {
  __shared__ __align__(16) int32_t s_pat[256 * kPatMax];
  for (uint32_t i = threadIdx.x; i < npat * kPatMax; i += kSpmvBlock) s_pat[i] = pat_off[i];
  __syncthreads();
  pdl_wait_and_release();
  if (mix_cta_done(st)) return;
  float beta;
  if (!mix_a_step(st, par, partial_b, nb, &beta)) return;
  const auto pm = L2Pol<HINT>::stream();
  const auto px = L2Pol<HINT>::keep();
  double local = 0.0;
  const uint32_t step = gridDim.x * kSpmvBlock;
  uint32_t i = blockIdx.x * kSpmvBlock + threadIdx.x;
  if (i < nrows) {
    // stage: the next row's code, values and own-row operands, one row ahead
    uint32_t c_cur = ld_l1_u8(code + i, pm);
    float4 va = v8[2 * static_cast<size_t>(i)], vb = v8[2 * static_cast<size_t>(i) + 1];
    float r_cur = r[i], p_cur = pold[i];
    for (; i < nrows; i += step) {
      const uint32_t i1 = i + step;
      uint32_t c_nx = 0;
      float4 na = make_float4(0.f, 0.f, 0.f, 0.f), nb4 = na;
      float r_nx = 0.f, p_nx = 0.f;
      if (i1 < nrows) {
        c_nx = ld_l1_u8(code + i1, pm);
        na = v8[2 * static_cast<size_t>(i1)];
        nb4 = v8[2 * static_cast<size_t>(i1) + 1];
        r_nx = r[i1];
        p_nx = pold[i1];
      }
      const int32_t * po = s_pat + c_cur * kPatMax;
      const int len = po[kPatMax - 1];
      const float v[8] = {va.x, va.y, va.z, va.w, vb.x, vb.y, vb.z, vb.w};
      float xv[STAGE];
#pragma unroll
      for (int j = 0; j < STAGE; ++j)
        if (j < len) {
          const uint32_t c = i + static_cast<uint32_t>(po[j]);
          xv[j] = fmaf(beta, ld_keep(pold + c, px), ld_keep(r + c, px));
        }
      float sum = 0.0f;
#pragma unroll
      for (int j = 0; j < STAGE; ++j)
        if (j < len) sum = add_rn(sum, mul_rn(v[j], xv[j]));
      ap[i] = sum;
      const float pn = fmaf(beta, p_cur, r_cur);
      pnew[i] = pn;
      local += static_cast<double>(pn) * static_cast<double>(sum);
      c_cur = c_nx;
      va = na;
      vb = nb4;
      r_cur = r_nx;
      p_cur = p_nx;
    }
  }
  __shared__ double red[32];
  const double bs = block_sum(local, red);
  if (threadIdx.x == 0) partial[blockIdx.x] = bs;
}

// ---- B32 ----------------------------------------------------------------------

// The reliable update of B32's rows (a kPhaseRefresh pair): r = b - A (x + y)
// with the FP64 values, each row summed in the reference's order
// (src/blas.c:82-91, unfused multiply and add), x <- x + y into the other x
// buffer, r rounded to FP32, and the true r.r partial of the CTA.  The search
// direction is kept: A32 wrote no new one in this pair, so it is carried into
// the buffer the next A32 reads (pnew <- pold).  One thread per row: the
// reliable update is rare, and this keeps the FP64 loop out of the SpMV
// kernel's register budget.
__device__ __forceinline__ void mix_refresh_rows(size_t s, size_t e,
    const uint32_t * __restrict__ rowptr, const uint32_t * __restrict__ rowind,
    const double * __restrict__ val, const double * __restrict__ b,
    const double * __restrict__ xold, double * __restrict__ xnew, const float * __restrict__ y,
    float * __restrict__ r, const float * __restrict__ pold, float * __restrict__ pnew,
    bool use_y, double * __restrict__ partial, double * red) {
  double acc = 0.0;
  for (size_t i = s + threadIdx.x; i < e; i += kVecBlock) {
    pnew[i] = pold[i];
    const uint32_t kb = __ldg(rowptr + i), ke = __ldg(rowptr + i + 1);
    double ax = 0.0;
    for (uint32_t k = kb; k < ke; ++k) {
      const uint32_t c = __ldg(rowind + k);
      const double xc = use_y ? xold[c] + static_cast<double>(y[c]) : xold[c];
      ax = add_rn(ax, mul_rn(__ldg(val + k), xc));
    }
    xnew[i] = use_y ? xold[i] + static_cast<double>(y[i]) : xold[i];
    const double rt = b[i] - ax;
    r[i] = static_cast<float>(rt);
    acc += rt * rt;
  }
  const double bs = block_sum(acc, red);
  if (threadIdx.x == 0) partial[blockIdx.x] = bs;
}

// Every CTA first sums A32's p.Ap partials (then the long-row terms) in order
// and forms alpha = rr_hat / p.Ap; a breakdown (p.Ap <= 0) or NaN stops the
// solve before anything is updated.  In a reliable-update pair it computes
// the FP64 residual of its rows instead (mix_refresh_rows).  Six CTAs per SM
// (40 registers, no spills): the update streams six vectors, and at four CTAs
// (54 registers) it ran 21.2 us instead of 18.6 on the 160^3 operator.
// Units of four elements per thread per pass: at one unit the update loads
// 16 bytes per vector (21.0 -> 18.6 us on the 160^3 operator against the
// former four scalar elements); two units spill at this register budget (21.5 us).
#ifndef GB_B32_UNITS
#define GB_B32_UNITS 1
#endif
__global__ void __launch_bounds__(kVecBlock, 6) cg_b32_kernel(size_t n,
    float * __restrict__ y, float * __restrict__ r, float * __restrict__ p,
    const float * __restrict__ pold,
    const float * __restrict__ ap, const double * __restrict__ partial_a, unsigned na,
    const double * __restrict__ longdot, unsigned nlong, double * __restrict__ partial,
    MixState * st, int par, const uint32_t * __restrict__ rowptr,
    const uint32_t * __restrict__ rowind, const double * __restrict__ val64,
    const double * __restrict__ bvec, double * x0, double * x1) {
  pdl_wait_and_release();
  if (mix_cta_done(st)) return;
  __shared__ double red[32];
  __shared__ double s_pap;
  if (st->sv[par].phase == kPhaseRefresh) {
    const size_t q = n / gridDim.x, rem = n % gridDim.x;
    const size_t cb = blockIdx.x;
    const size_t s = cb * q + min(cb, rem);
    const size_t e = s + q + (cb < rem ? 1 : 0);
    const int xp = st->xpar;
    mix_refresh_rows(s, e, rowptr, rowind, val64, bvec, xp ? x1 : x0, xp ? x0 : x1, y, r,
        pold, p, st->sv[par].y_reset == 0, partial, red);
    return;
  }
  double tot = ordered_sum(partial_a, na, red);
  if (threadIdx.x == 0) {
    for (unsigned q = 0; q < nlong; ++q) tot += __ldcg(longdot + q);
    s_pap = tot;
  }
  __syncthreads();
  const double pap = s_pap;
  const double rr_hat = st->sv[par].rr_hat;
  if (!(pap > 0.0)) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      st->status = (pap == pap && rr_hat == rr_hat) ? GB_CG_BREAKDOWN : GB_CG_NONFINITE;
      st->done = 1;
    }
    return;
  }
  const float alpha = static_cast<float>(rr_hat / pap);
  const bool fresh = st->sv[par].y_reset != 0;
  // contiguous chunk per CTA in units of four elements (16-byte loads); all
  // loads of a pass are issued before any arithmetic
  const size_t units = (n + 3) / 4;
  const size_t q = units / gridDim.x, rem = units % gridDim.x;
  const size_t b = blockIdx.x;
  const size_t us = b * q + min(b, rem);
  const size_t ue = us + q + (b < rem ? 1 : 0);
  const size_t full = n / 4;  // complete units
  const size_t ve = min(ue, full);
  const float4 * p4 = reinterpret_cast<const float4 *>(p);
  const float4 * a4 = reinterpret_cast<const float4 *>(ap);
  float4 * y4 = reinterpret_cast<float4 *>(y);
  float4 * r4 = reinterpret_cast<float4 *>(r);
  double acc = 0.0;
  constexpr int U = GB_B32_UNITS;
  for (size_t base = us; base < ve; base += U * kVecBlock) {
    float4 pv[U], av[U], yv[U], rv[U];
#pragma unroll
    for (int j = 0; j < U; ++j) {
      const size_t u = base + threadIdx.x + j * kVecBlock;
      if (u < ve) {
        pv[j] = p4[u];
        av[j] = a4[u];
        yv[j] = fresh ? make_float4(0.f, 0.f, 0.f, 0.f) : y4[u];
        rv[j] = r4[u];
      }
    }
#pragma unroll
    for (int j = 0; j < U; ++j) {
      const size_t u = base + threadIdx.x + j * kVecBlock;
      if (u < ve) {
        float4 yn, rn;
        yn.x = fmaf(alpha, pv[j].x, yv[j].x);
        yn.y = fmaf(alpha, pv[j].y, yv[j].y);
        yn.z = fmaf(alpha, pv[j].z, yv[j].z);
        yn.w = fmaf(alpha, pv[j].w, yv[j].w);
        rn.x = fmaf(-alpha, av[j].x, rv[j].x);
        rn.y = fmaf(-alpha, av[j].y, rv[j].y);
        rn.z = fmaf(-alpha, av[j].z, rv[j].z);
        rn.w = fmaf(-alpha, av[j].w, rv[j].w);
        y4[u] = yn;
        r4[u] = rn;
        acc += static_cast<double>(rn.x) * static_cast<double>(rn.x);
        acc += static_cast<double>(rn.y) * static_cast<double>(rn.y);
        acc += static_cast<double>(rn.z) * static_cast<double>(rn.z);
        acc += static_cast<double>(rn.w) * static_cast<double>(rn.w);
      }
    }
  }
  if (ue > full && threadIdx.x == 0) {  // n % 4 elements past the last complete unit
    for (size_t i = 4 * full; i < n; ++i) {
      y[i] = fmaf(alpha, p[i], fresh ? 0.0f : y[i]);
      const float rn = fmaf(-alpha, ap[i], r[i]);
      r[i] = rn;
      acc += static_cast<double>(rn) * static_cast<double>(rn);
    }
  }
  const double bs = block_sum(acc, red);
  if (threadIdx.x == 0) partial[blockIdx.x] = bs;
}

// ---- R: reliable update -------------------------------------------------------

struct GatherXY {
  const double * x;
  const float * y;
  bool use_y;
  template <class P>
  __device__ __forceinline__ double operator()(uint32_t c, P pol) const {
    const double xv = ld_keep(x + c, pol);
    return use_y ? xv + static_cast<double>(ld_keep(y + c, pol)) : xv;
  }
};

struct OutR {
  const double * b;
  const double * xold;
  double * xnew;
  const float * y;
  float * r32;
  double * longdot;
  double * partial;
  MixState * st;
  bool use_y;
  unsigned nlong;
  double local;
  MixScalars * sv;  // the version this R step writes
  bool forced;      // fold and measure only: the iteration does not continue
  __device__ __forceinline__ double fold(uint32_t i, double ax) {
    xnew[i] = use_y ? xold[i] + static_cast<double>(y[i]) : xold[i];
    const double rt = b[i] - ax;
    r32[i] = static_cast<float>(rt);
    return rt * rt;
  }
  __device__ __forceinline__ void row(uint32_t i, double v) { local += fold(i, v); }
  __device__ __forceinline__ void long_row(uint32_t lid, uint32_t i, double v) {
    longdot[lid] = fold(i, v);
  }
  struct Pre {};
  __device__ __forceinline__ Pre pre(uint32_t) const { return Pre{}; }
  __device__ __forceinline__ void row_pre(uint32_t i, double v, const Pre &) { row(i, v); }
  __device__ __forceinline__ void finish() {
    __shared__ double red[32];
    __shared__ bool last;
    const double s = block_sum(local, red);
    if (threadIdx.x == 0) partial[blockIdx.x] = s;
    if (!arrive_last(&st->ticket_r, &last)) return;
    __threadfence();
    double tot = ordered_sum(partial, gridDim.x, red);
    if (threadIdx.x == 0) {
      for (unsigned q = 0; q < nlong; ++q) tot += __ldcg(longdot + q);
      st->ticket_r = 0;
      st->rr_true = tot;
      st->refinements += 1;
      st->xpar ^= 1;
      sv->y_reset = 1;
      sv->phase = kPhaseCg;
      const double rnorm = sqrt(tot);
      // written by CTA 0 during this launch: read through L2
      const unsigned long long it = __ldcg(&st->iter);
      if (st->hist && it >= 1 && it <= st->hist_len) st->hist[it - 1] = rnorm;
      if (!(rnorm == rnorm) || isinf(rnorm)) {
        st->done = 1;
        st->status = GB_CG_NONFINITE;
      } else if (rnorm <= st->tol) {
        st->done = 1;
        st->status = GB_CG_CONVERGED;
      } else if (!forced) {
        // continue from the true residual, keeping the search direction
        sv->beta = tot / __ldcg(&sv->rr_hat_old);
        sv->rr_hat = tot;
        sv->rmax = rnorm;
        if (st->niter && it >= st->niter) {
          st->done = 1;
          st->status = GB_CG_MAXITER;
        }
      }
    }
  }
};

// R: the FP64 residual r = b - A (x + y) over the matrix's SpMV schedule,
// x <- x + y into the other x buffer; kRFold folds a pending correction when a
// solve stopped (version `par`, the current one), kRProfile times the step.
template <int SCHED, bool HINT>
__global__ void __launch_bounds__(kSpmvBlock, MinBlocks<SCHED>::value) cg_r_kernel(
    const PlanView plan, const uint32_t * __restrict__ rowptr,
    const uint32_t * __restrict__ rowind, const double * __restrict__ val,
    const double * __restrict__ b, const double * __restrict__ x0, double * __restrict__ x1,
    const float * __restrict__ y, float * __restrict__ r32, double * __restrict__ longdot,
    double * __restrict__ partial, MixState * st, int par, int mode) {
  pdl_wait_and_release();
  MixScalars * sv = &st->sv[par];
  const int xpar = st->xpar;
  // a fold uses y only if no update has consumed it yet
  const bool use_y = mode != kRFold || sv->y_reset == 0;
  const double * xold = xpar ? x1 : x0;
  double * xnew = xpar ? const_cast<double *>(x0) : x1;
  GatherXY g{xold, y, use_y};
  OutR o{b, xold, xnew, y, r32, longdot, partial, st, use_y,
         SCHED == SCHED_ROW ? 0u : plan.nlong, 0.0, sv, true};
  spmv_tiles_body<double, double, SCHED, kSpmvBlock, GatherXY, OutR, false, HINT>(plan, rowptr,
      rowind, val, g, o);
}

// ---- init -----------------------------------------------------------------------

__global__ void __launch_bounds__(kVecBlock) cg_mixed_init_kernel(size_t n,
    const double * __restrict__ b, double * __restrict__ x0, float * __restrict__ r32,
    float * __restrict__ p0, double * __restrict__ partial, MixState * st,
    int tol_relative) {
  __shared__ double red[32];
  __shared__ double red2[32];
  __shared__ bool last;
  double acc = 0.0, acc32 = 0.0;
  for (size_t i = blockIdx.x * static_cast<size_t>(kVecBlock) + threadIdx.x; i < n;
       i += static_cast<size_t>(gridDim.x) * kVecBlock) {
    const double bv = b[i];
    const float rv = static_cast<float>(bv);
    x0[i] = 0.0;
    r32[i] = rv;
    p0[i] = 0.0f;
    acc += bv * bv;
    acc32 += static_cast<double>(rv) * static_cast<double>(rv);
  }
  const double s = block_sum(acc, red);
  const double s32 = block_sum(acc32, red2);
  if (threadIdx.x == 0) {
    partial[2 * blockIdx.x] = s;
    partial[2 * blockIdx.x + 1] = s32;
  }
  if (!arrive_last(&st->ticket_i, &last)) return;
  __threadfence();
  // ordered sums of the even (b.b) and odd (r32.r32) entries
  double bb = 0.0, rr = 0.0;
  if (threadIdx.x == 0) {
    for (unsigned i = 0; i < gridDim.x; ++i) {
      bb += __ldcg(partial + 2 * i);
      rr += __ldcg(partial + 2 * i + 1);
    }
    st->ticket_i = 0;
    st->bnorm = sqrt(bb);
    st->rr_true = bb;
    MixScalars v0;
    v0.rr_hat = rr;
    v0.rr_hat_old = rr;
    v0.rmax = sqrt(rr);
    v0.beta = 0.0;
    v0.iter = 0;
    v0.y_reset = 1;
    v0.phase = kPhaseFirst;
    st->sv[0] = v0;
    st->ver = 0;
    st->iter = 0;
    st->refinements = 0;
    st->xpar = 0;
    if (tol_relative) st->tol = st->tol * st->bnorm;
    st->done = 0;
    st->status = GB_CG_MAXITER;
    if (bb == 0.0) {
      st->done = 1;
      st->status = GB_CG_CONVERGED;
    } else if (!(bb == bb) || isinf(bb)) {
      st->done = 1;
      st->status = GB_CG_NONFINITE;
    }
  }
}

// ---- launch helpers ----------------------------------------------------------------

size_t smem_of(int sched, uint32_t tile_items, size_t value_bytes) {
  return value_bytes == 4 ? spmv_smem_bytes<float, float>(sched, tile_items, kSpmvBlock)
                          : spmv_smem_bytes<double, double>(sched, tile_items, kSpmvBlock);
}

template <typename K>
int prep_kernel(K kern, size_t smem, int * occ) {
  GB_TRY(raise_smem_limit(reinterpret_cast<const void *>(kern), smem));
  if (occ)
    GB_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(occ, kern, kSpmvBlock, smem));
  return GOOSEBERRY_SUCCESS;
}

template <int SCHED, bool HINT>
int launch_a32_t(const gb_csr & a, unsigned grid, cudaStream_t s, bool pdl,
    const float * r, const float * pold, float * pnew, float * ap, double * longdot,
    double * partial, MixState * st, int par, const double * partial_b, unsigned nb) {
  const size_t smem = smem_of(SCHED, a.plan.tile_items, 4);
  auto kern = cg_a32_kernel<SCHED, HINT>;
  GB_TRY(prep_kernel(kern, smem, nullptr));
  GB_CUDA_TRY(launch_k(kern, grid, kSpmvBlock, smem, s, pdl, plan_view(a), a.rowptr,
      a.rowind, a.val32, r, pold, pnew, ap, longdot, partial, st, par, partial_b, nb));
  return GOOSEBERRY_SUCCESS;
}

template <int SCHED, bool HINT>
int launch_r_t(const gb_csr & a, unsigned grid, cudaStream_t s, bool pdl, const double * b,
    const double * x0, double * x1, const float * y, float * r32, double * longdot,
    double * partial, MixState * st, int par, int mode) {
  const size_t smem = smem_of(SCHED, a.plan.tile_items, 8);
  auto kern = cg_r_kernel<SCHED, HINT>;
  GB_TRY(prep_kernel(kern, smem, nullptr));
  GB_CUDA_TRY(launch_k(kern, grid, kSpmvBlock, smem, s, pdl, plan_view(a), a.rowptr,
      a.rowind, a.val64, b, x0, x1, y, r32, longdot, partial, st, par, mode));
  return GOOSEBERRY_SUCCESS;
}

#define GB_SCHED_SWITCH(sched, CALL)                                            \
  switch (sched) {                                                              \
    case GB_SCHED_THREAD: return CALL(SCHED_THREAD);                            \
    case GB_SCHED_GROUP4: return CALL(SCHED_GROUP4);                            \
    case GB_SCHED_GROUP8: return CALL(SCHED_GROUP8);                            \
    case GB_SCHED_WARP: return CALL(SCHED_WARP);                                \
    case GB_SCHED_ROW: return CALL(SCHED_ROW);                                  \
    case GB_SCHED_WTILE: return CALL(SCHED_WTILE);                              \
    default: return CALL(SCHED_MERGE);                                          \
  }

template <class IC, bool HINT>
int launch_a32_c_t(const gb_csr & a, const IC & ic, const RowPatterns & pat, int stage,
    unsigned grid, cudaStream_t s, bool pdl, const float * r, const float * pold, float * pnew,
    float * ap, double * longdot, double * partial, MixState * st, int par,
    const double * partial_b, unsigned nb, int * occ) {
  auto kern = stage == 5   ? cg_a32_c_kernel<IC, HINT, 5>
              : stage == 7 ? cg_a32_c_kernel<IC, HINT, 7>
                           : cg_a32_c_kernel<IC, HINT, kRowStage>;
  if (occ) return prep_kernel(kern, 0, occ);
  GB_CUDA_TRY(launch_k(kern, grid, kSpmvBlock, 0, s, pdl, plan_view(a), a.rowptr, ic,
      static_cast<const int32_t *>(pat.off), pat.npat, a.val32, r, pold, pnew, ap, longdot,
      partial, st, par, partial_b, nb));
  return GOOSEBERRY_SUCCESS;
}

// The row-schedule A32 over the solver's compressed columns (patterns, else
// 16-bit distances).
template <bool HINT>
int launch_a32_d16_t(const gb_csr & a, const RowPatterns & pat, const int16_t * col16,
    int stage, unsigned grid, cudaStream_t s, bool pdl, const float * r, const float * pold,
    float * pnew, float * ap, double * longdot, double * partial, MixState * st, int par,
    const double * partial_b, unsigned nb, int * occ) {
  if (pat.code8)
    return launch_a32_c_t<ColPat8, HINT>(a, ColPat8{pat.code8, nullptr}, pat, stage, grid, s,
        pdl, r, pold, pnew, ap, longdot, partial, st, par, partial_b, nb, occ);
  return launch_a32_c_t<ColD16, HINT>(a, ColD16{col16}, pat, stage, grid, s, pdl, r, pold, pnew,
      ap, longdot, partial, st, par, partial_b, nb, occ);
}

template <int SCHED>
int occ_a32_t(size_t smem, int * occ) {
  return prep_kernel(cg_a32_kernel<SCHED, false>, smem, occ);
}
template <int SCHED>
int occ_r_t(size_t smem, int * occ) { return prep_kernel(cg_r_kernel<SCHED, false>, smem, occ); }

}  // namespace

// ---- the solver ------------------------------------------------------------------

struct MixedCg {
  const gb_csr * a = nullptr;
  size_t n = 0;
  int sched32 = GB_SCHED_MERGE, sched64 = GB_SCHED_MERGE;
  uint32_t tile_items = 0;
  double * x[2] = {nullptr, nullptr};
  double * b = nullptr;
  float * y = nullptr;
  float * r = nullptr;
  float * p[2] = {nullptr, nullptr};
  float * ap = nullptr;
  float * v8 = nullptr;  // FP32 values in rows of 8 (pattern matrices, GB_MIX_ELL)
  double * partial_a = nullptr;
  double * partial_b = nullptr;
  double * partial_r = nullptr;
  double * partial_i = nullptr;
  double * longdot = nullptr;
  MixState * st = nullptr;
  MixStatus * host_status = nullptr;
  unsigned grid_a = 0, grid_b = 0, grid_r = 0;
  bool l2_hint = false;  // L2-policy loads (the FP32 working set fits in L2)
  // row schedule: columns as row patterns, else column - row in 16 bits
  RowPatterns pat;
  int16_t * col16 = nullptr;
  int stage = 6;
  int chunk = 32;
  cudaStream_t cap_stream = nullptr;
  cudaGraphExec_t graph[2] = {nullptr, nullptr};
};

namespace {

int launch_a32(MixedCg * m, cudaStream_t s, bool pdl, int k) {
  const float * pold = m->p[k & 1];
  float * pnew = m->p[(k + 1) & 1];
  if (m->v8) {
    auto kern = m->stage == 5 ? (m->l2_hint ? cg_a32_ell_kernel<true, 5> : cg_a32_ell_kernel<false, 5>)
                              : (m->l2_hint ? cg_a32_ell_kernel<true, 7> : cg_a32_ell_kernel<false, 7>);
    GB_CUDA_TRY(launch_k(kern, m->grid_a, kSpmvBlock, 0, s, pdl, static_cast<uint32_t>(m->n),
        static_cast<const uint8_t *>(m->pat.code8), static_cast<const int32_t *>(m->pat.off),
        m->pat.npat, static_cast<const float4 *>(reinterpret_cast<float4 *>(m->v8)),
        static_cast<const float *>(m->r), pold, pnew, m->ap, m->partial_a, m->st, k & 1,
        static_cast<const double *>(m->partial_b), m->grid_b));
    return GOOSEBERRY_SUCCESS;
  }
  if (m->pat.code8 || m->col16)
    return m->l2_hint ? launch_a32_d16_t<true>(*m->a, m->pat, m->col16, m->stage, m->grid_a, s,
                            pdl, m->r, pold, pnew, m->ap, m->longdot, m->partial_a, m->st,
                            k & 1, m->partial_b, m->grid_b, nullptr)
                      : launch_a32_d16_t<false>(*m->a, m->pat, m->col16, m->stage, m->grid_a, s,
                            pdl, m->r, pold, pnew, m->ap, m->longdot, m->partial_a, m->st,
                            k & 1, m->partial_b, m->grid_b, nullptr);
#define GB_CALL(S)                                                                      \
  (m->l2_hint ? launch_a32_t<S, true>(*m->a, m->grid_a, s, pdl, m->r, pold, pnew, m->ap,   \
                                      m->longdot, m->partial_a, m->st, k & 1,              \
                                      m->partial_b, m->grid_b)                             \
              : launch_a32_t<S, false>(*m->a, m->grid_a, s, pdl, m->r, pold, pnew, m->ap,  \
                                       m->longdot, m->partial_a, m->st, k & 1,             \
                                       m->partial_b, m->grid_b))
  GB_SCHED_SWITCH(m->sched32, GB_CALL)
#undef GB_CALL
}

// R over version par (kRFold: the current version).
int launch_r(MixedCg * m, cudaStream_t s, bool pdl, int par, int mode) {
#define GB_CALL(S)                                                                      \
  (m->l2_hint ? launch_r_t<S, true>(*m->a, m->grid_r, s, pdl, m->b, m->x[0], m->x[1], m->y,  \
                                    m->r, m->longdot, m->partial_r, m->st, par, mode)       \
              : launch_r_t<S, false>(*m->a, m->grid_r, s, pdl, m->b, m->x[0], m->x[1], m->y, \
                                     m->r, m->longdot, m->partial_r, m->st, par, mode))
  GB_SCHED_SWITCH(m->sched64, GB_CALL)
#undef GB_CALL
}

// B32 of A32 launch k: it reads the version A32 k wrote, (k + 1) & 1.
int launch_b32(MixedCg * m, cudaStream_t s, bool pdl, int k) {
  float * pnew = m->p[(k + 1) & 1];
  // the row schedule sums long rows like any other row: no long-row terms
  const unsigned nlong = m->sched32 == GB_SCHED_ROW ? 0u
                         : static_cast<unsigned>(m->a->plan.longrows.size());
  GB_CUDA_TRY(launch_k(cg_b32_kernel, m->grid_b, kVecBlock, 0, s, pdl, m->n, m->y, m->r,
      pnew, static_cast<const float *>(m->p[k & 1]), static_cast<const float *>(m->ap),
      static_cast<const double *>(m->partial_a), m->grid_a,
      static_cast<const double *>(m->longdot), nlong, m->partial_b, m->st, (k + 1) & 1,
      m->a->rowptr, m->a->rowind, static_cast<const double *>(m->a->val64),
      static_cast<const double *>(m->b), m->x[0], m->x[1]));
  return GOOSEBERRY_SUCCESS;
}

int iteration(MixedCg * m, cudaStream_t s, bool pdl_first, int k) {
  GB_TRY(launch_a32(m, s, pdl_first, k));
  GB_TRY(launch_b32(m, s, true, k));
  return GOOSEBERRY_SUCCESS;
}

int capture(MixedCg * m, int slot) {
  cudaStream_t cs = m->cap_stream;
  GB_CUDA_TRY(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
  int rc = GOOSEBERRY_SUCCESS;
  for (int k = 0; k < m->chunk && rc == GOOSEBERRY_SUCCESS; ++k) rc = iteration(m, cs, k > 0, k);
  if (rc == GOOSEBERRY_SUCCESS) {
    cudaMemcpyAsync(&m->host_status[slot].done, &m->st->done, sizeof(int),
        cudaMemcpyDeviceToHost, cs);
    cudaMemcpyAsync(&m->host_status[slot].iter, &m->st->iter, sizeof(unsigned long long),
        cudaMemcpyDeviceToHost, cs);
  }
  cudaGraph_t g = nullptr;
  cudaError_t e = cudaStreamEndCapture(cs, &g);
  if (rc != GOOSEBERRY_SUCCESS) {
    if (g) cudaGraphDestroy(g);
    return rc;
  }
  GB_CUDA_TRY(e);
  e = cudaGraphInstantiate(&m->graph[slot], g, 0);
  cudaGraphDestroy(g);
  GB_CUDA_TRY(e);
  return GOOSEBERRY_SUCCESS;
}

int grid_of(const gb_csr * a, int sched, size_t smem, bool f32, unsigned * grid) {
  int occ = 0;
  if (f32) {
#define GB_CALL(S) occ_a32_t<S>(smem, &occ)
    int rc;
    switch (sched) {
      case GB_SCHED_THREAD: rc = GB_CALL(SCHED_THREAD); break;
      case GB_SCHED_GROUP4: rc = GB_CALL(SCHED_GROUP4); break;
      case GB_SCHED_GROUP8: rc = GB_CALL(SCHED_GROUP8); break;
      case GB_SCHED_WARP: rc = GB_CALL(SCHED_WARP); break;
      case GB_SCHED_ROW: rc = GB_CALL(SCHED_ROW); break;
      case GB_SCHED_WTILE: rc = GB_CALL(SCHED_WTILE); break;
      default: rc = GB_CALL(SCHED_MERGE); break;
    }
#undef GB_CALL
    GB_TRY(rc);
  } else {
#define GB_CALL(S) occ_r_t<S>(smem, &occ)
    int rc;
    switch (sched) {
      case GB_SCHED_THREAD: rc = GB_CALL(SCHED_THREAD); break;
      case GB_SCHED_GROUP4: rc = GB_CALL(SCHED_GROUP4); break;
      case GB_SCHED_GROUP8: rc = GB_CALL(SCHED_GROUP8); break;
      case GB_SCHED_WARP: rc = GB_CALL(SCHED_WARP); break;
      case GB_SCHED_ROW: rc = GB_CALL(SCHED_ROW); break;
      case GB_SCHED_WTILE: rc = GB_CALL(SCHED_WTILE); break;
      default: rc = GB_CALL(SCHED_MERGE); break;
    }
#undef GB_CALL
    GB_TRY(rc);
  }
  GB_CHECK_INPUT(occ > 0, "mixed CG kernel cannot be resident");
  const unsigned ntiles = static_cast<unsigned>(std::max<size_t>(a->plan.tiles.size(), 1));
  const unsigned work = spmv_work_units(sched, a->nrows, ntiles, kSpmvBlock);
  *grid = std::min<unsigned>(std::max(work, 1u), static_cast<unsigned>(a->sm_count * occ));
  return GOOSEBERRY_SUCCESS;
}

}  // namespace

void mixed_destroy(MixedCg * m) {
  if (!m) return;
  cudaDeviceSynchronize();  // its memory goes back to the pool below
  for (auto & g : m->graph)
    if (g) cudaGraphExecDestroy(g);
  if (m->cap_stream) cudaStreamDestroy(m->cap_stream);
  dev_free(m->x[0]);
  dev_free(m->x[1]);
  dev_free(m->b);
  dev_free(m->y);
  dev_free(m->r);
  dev_free(m->p[0]);
  dev_free(m->p[1]);
  dev_free(m->ap);
  dev_free(m->partial_a);
  dev_free(m->partial_b);
  dev_free(m->partial_r);
  dev_free(m->partial_i);
  dev_free(m->longdot);
  dev_free(m->st);
  if (m->col16) dev_free(m->col16);
  if (m->v8) dev_free(m->v8);
  free_row_patterns(m->pat);
  pinned_slot_free(m->host_status);
  delete m;
}

// Stored bytes A32 streams per nonzero and per row: rows of 8 padded values
// and a pattern byte (ELL: nothing per nonzero, no rowptr), else rowptr plus a
// pattern byte and a float per nonzero, 16-bit distances, or plain columns.
size_t mixed_entry_bytes(const MixedCg * m) {
  return m->v8 ? 0 : (m->pat.code8 ? 4 : (m->col16 ? 6 : 8));
}

size_t mixed_row_bytes(const MixedCg * m) { return m->v8 ? 33 : (m->pat.code8 ? 5 : 4); }

int mixed_create(const gb_csr * a, bool plain_entries, MixedCg ** out) {
  GB_CHECK_INPUT(a->val64 && a->val32,
      "mixed-precision CG needs both double and float values on the matrix "
      "(GB_CSR_VALUES_F64 | GB_CSR_VALUES_F32)");
  MixedCg * m = new MixedCg();
  *out = m;
  m->a = a;
  m->n = a->nrows;
  m->sched32 = a->sched32;
  m->sched64 = a->sched64;
  m->tile_items = a->plan.tile_items;
  // the row schedule reads a pattern byte per row when the rows form at most
  // 256 column patterns (stencils), else 16-bit column distances when every
  // entry lies within 32767 of the diagonal (banded matrices)
  if (m->sched32 == GB_SCHED_ROW && !plain_entries) {
    GB_TRY(build_row_patterns(*a, &m->pat, nullptr));
    if (!m->pat.code8) GB_TRY(build_col16(*a, &m->col16, nullptr));
    m->stage = row_stage_for(*a);
    if (GB_MIX_ELL && m->pat.code8 && (m->stage == 5 || m->stage == 7)) {
      GB_TRY(dev_alloc(&m->v8, std::max<size_t>(m->n, 1) * 8 * sizeof(float)));
      const unsigned g = static_cast<unsigned>(std::max<size_t>(1, std::min<size_t>(
          (m->n + 255) / 256, static_cast<size_t>(a->sm_count) * 8)));
      ell_values_kernel<<<g, 256>>>(static_cast<uint32_t>(m->n), a->rowptr, a->val32,
          reinterpret_cast<float4 *>(m->v8));
      GB_CUDA_TRY(cudaGetLastError());
      GB_CUDA_TRY(cudaDeviceSynchronize());
    }
  }
  // L2-policy loads only when the FP32 iteration's working set (rowptr,
  // indices, float values, r, both p, Ap, y) fits in L2
  GB_TRY(l2_fits(mixed_row_bytes(m) * (m->n + 1) + mixed_entry_bytes(m) * a->nnz +
      24ull * m->n, &m->l2_hint));
  const size_t n = std::max<size_t>(m->n, 2);
  GB_TRY(dev_alloc(&m->x[0], n * sizeof(double)));
  GB_TRY(dev_alloc(&m->x[1], n * sizeof(double)));
  GB_TRY(dev_alloc(&m->b, n * sizeof(double)));
  GB_TRY(dev_alloc(&m->y, n * sizeof(float)));
  GB_TRY(dev_alloc(&m->r, n * sizeof(float)));
  GB_TRY(dev_alloc(&m->p[0], n * sizeof(float)));
  GB_TRY(dev_alloc(&m->p[1], n * sizeof(float)));
  GB_TRY(dev_alloc(&m->ap, n * sizeof(float)));
  if (m->pat.code8 || m->col16) {
    int occ = 0;
    GB_TRY(launch_a32_d16_t<false>(*a, m->pat, m->col16, m->stage, 0, nullptr, false, nullptr,
        nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, 0, nullptr, 0, &occ));
    GB_CHECK_INPUT(occ > 0, "CG kernel cannot be resident");
    const size_t rows_units = (m->n + kSpmvBlock - 1) / kSpmvBlock;
    m->grid_a = static_cast<unsigned>(std::max<size_t>(1, std::min<size_t>(rows_units,
        static_cast<size_t>(a->sm_count) * occ)));
  } else {
    GB_TRY(grid_of(a, m->sched32, smem_of(m->sched32, m->tile_items, 4), true, &m->grid_a));
  }
  GB_TRY(grid_of(a, m->sched64, smem_of(m->sched64, m->tile_items, 8), false, &m->grid_r));
  int occ_b = 0;
  GB_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_b, cg_b32_kernel, kVecBlock, 0));
  m->grid_b = static_cast<unsigned>(std::max<size_t>(1, std::min<size_t>(
      (m->n + kVecBlock - 1) / kVecBlock, static_cast<size_t>(a->sm_count) * std::max(occ_b, 1))));
  const unsigned gmax = std::max({m->grid_a, m->grid_b, m->grid_r, 1u});
  GB_TRY(dev_alloc(&m->partial_a, gmax * sizeof(double)));
  GB_TRY(dev_alloc(&m->partial_b, gmax * sizeof(double)));
  GB_TRY(dev_alloc(&m->partial_r, gmax * sizeof(double)));
  GB_TRY(dev_alloc(&m->partial_i, 2 * gmax * sizeof(double)));
  GB_TRY(dev_alloc(&m->longdot,
      std::max<size_t>(a->plan.longrows.size(), 1) * sizeof(double)));
  GB_TRY(dev_alloc(&m->st, sizeof(MixState)));
  GB_CUDA_TRY(cudaMemset(m->st, 0, sizeof(MixState)));
  GB_TRY(pinned_slot_alloc(2 * sizeof(MixStatus), reinterpret_cast<void **>(&m->host_status),
      nullptr));
  GB_CUDA_TRY(cudaStreamCreateWithFlags(&m->cap_stream, cudaStreamNonBlocking));
  GB_TRY(capture(m, 0));
  GB_TRY(capture(m, 1));
  return GOOSEBERRY_SUCCESS;
}

namespace {

int mixed_start(MixedCg * m, const double * b, double tol, int tol_relative, size_t niter,
    double * dhist, size_t hl, cudaStream_t stream) {
  const size_t cap = std::max<size_t>(1000, 100 * m->n);
  MixState init{};
  init.tol = tol;
  init.niter = niter ? niter : cap;
  init.hist = dhist;
  init.hist_len = hl;
  GB_CUDA_TRY(cudaMemcpyAsync(m->st, &init, sizeof(MixState), cudaMemcpyHostToDevice, stream));
  GB_CUDA_TRY(cudaMemcpyAsync(m->b, b, m->n * sizeof(double), cudaMemcpyDeviceToDevice,
      stream));
  cg_mixed_init_kernel<<<m->grid_b, kVecBlock, 0, stream>>>(m->n, m->b, m->x[0], m->r,
      m->p[0], m->partial_i, m->st, tol_relative);
  GB_CUDA_TRY(cudaGetLastError());
  return GOOSEBERRY_SUCCESS;
}

}  // namespace

int mixed_solve(MixedCg * m, const double * b, double * x, double tol, int tol_relative,
    size_t niter, double * history, size_t history_len, gb_cg_result_t * res,
    cudaStream_t stream, const int * cancel) {
  GB_CHECK_INPUT(m->n == 0 || (b && x), "NULL vector");
  GB_CHECK_INPUT(m->a->sched32 == m->sched32 && m->a->sched64 == m->sched64 &&
                 m->a->plan.tile_items == m->tile_items,
      "matrix schedule changed after the solver was created");
  if (m->n == 0) {
    if (res) *res = gb_cg_result_t{0, 0, 0.0, 0.0, GB_CG_CONVERGED, 0};
    return GOOSEBERRY_SUCCESS;
  }
  double * dhist = nullptr;
  const size_t hl = history ? std::min(history_len, niter ? niter : history_len) : 0;
  if (hl) GB_TRY(scratch_alloc(reinterpret_cast<void **>(&dhist), hl * sizeof(double), stream));
  GB_TRY(mixed_start(m, b, tol, tol_relative, niter, dhist, hl, stream));
  size_t launches = 1;
  cudaEvent_t ev[2];
  GB_CUDA_TRY(cudaEventCreateWithFlags(&ev[0], cudaEventDisableTiming));
  GB_CUDA_TRY(cudaEventCreateWithFlags(&ev[1], cudaEventDisableTiming));
  m->host_status[0].done = m->host_status[1].done = 0;
  int rc = GOOSEBERRY_SUCCESS;
  auto launch = [&](int slot) -> int {
    cudaError_t e = cudaGraphLaunch(m->graph[slot], stream);
    if (e == cudaSuccess) e = cudaEventRecord(ev[slot], stream);
    launches += 2 * static_cast<size_t>(m->chunk);
    if (e != cudaSuccess) {
      set_error("mixed CG graph launch failed: %s", cudaGetErrorString(e));
      return GOOSEBERRY_ERROR_UNKNOWN;
    }
    return GOOSEBERRY_SUCCESS;
  };
  rc = launch(0);
  if (rc == GOOSEBERRY_SUCCESS) rc = launch(1);
  int slot = 0;
  bool cancelled = false;
  while (rc == GOOSEBERRY_SUCCESS) {
    cudaError_t e = cudaEventSynchronize(ev[slot]);
    if (e != cudaSuccess) {
      set_error("mixed CG solve failed: %s", cudaGetErrorString(e));
      rc = GOOSEBERRY_ERROR_UNKNOWN;
      break;
    }
    if (m->host_status[slot].done) break;
    if (cancel && __atomic_load_n(cancel, __ATOMIC_ACQUIRE)) {  // no new graph starts
      cancelled = true;
      break;
    }
    rc = launch(slot);
    slot ^= 1;
  }
  cudaError_t e = cudaStreamSynchronize(stream);
  cudaEventDestroy(ev[0]);
  cudaEventDestroy(ev[1]);
  if (rc == GOOSEBERRY_SUCCESS && e != cudaSuccess) {
    set_error("mixed CG solve failed: %s", cudaGetErrorString(e));
    rc = GOOSEBERRY_ERROR_UNKNOWN;
  }
  MixState fin{};
  if (rc == GOOSEBERRY_SUCCESS) {
    e = cudaMemcpy(&fin, m->st, sizeof(MixState), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && fin.status != GB_CG_CONVERGED && fin.status != GB_CG_NONFINITE &&
        fin.sv[fin.ver].y_reset == 0) {
      // stopped on the iteration limit (or breakdown) with a pending FP32
      // correction: fold it into x once more and measure the true residual
      rc = launch_r(m, stream, false, fin.ver, kRFold);
      launches += 1;
      if (e == cudaSuccess && rc == GOOSEBERRY_SUCCESS) e = cudaStreamSynchronize(stream);
      if (e == cudaSuccess && rc == GOOSEBERRY_SUCCESS)
        e = cudaMemcpy(&fin, m->st, sizeof(MixState), cudaMemcpyDeviceToHost);
    }
    if (e == cudaSuccess && rc == GOOSEBERRY_SUCCESS)
      e = cudaMemcpyAsync(x, m->x[fin.xpar], m->n * sizeof(double), cudaMemcpyDeviceToDevice,
          stream);
    if (e == cudaSuccess && rc == GOOSEBERRY_SUCCESS && hl && fin.iter)
      e = cudaMemcpyAsync(history, dhist, std::min<size_t>(hl, fin.iter) * sizeof(double),
          cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess && rc == GOOSEBERRY_SUCCESS) e = cudaStreamSynchronize(stream);
    if (rc == GOOSEBERRY_SUCCESS && e != cudaSuccess) {
      set_error("mixed CG result copy failed: %s", cudaGetErrorString(e));
      rc = GOOSEBERRY_ERROR_UNKNOWN;
    }
  }
  if (rc == GOOSEBERRY_SUCCESS && res) {
    res->iterations = fin.iter;
    res->refinements = fin.refinements;
    res->rnorm = std::sqrt(fin.rr_true);
    res->bnorm = fin.bnorm;
    res->status = cancelled && fin.status != GB_CG_CONVERGED ? GB_CG_CANCELLED : fin.status;
    res->kernel_launches = launches;
  }
  if (dhist) scratch_free(dhist, stream);
  return rc;
}

int mixed_profile(MixedCg * m, const double * b, size_t iterations, double * ms,
    size_t ms_len, size_t * nkernels, cudaStream_t stream) {
  GB_CHECK_INPUT(m->n > 0 && b != nullptr, "profile needs a non-empty system and b");
  GB_CHECK_INPUT(iterations > 0, "iterations must be positive");
  if (nkernels) *nkernels = 3;  // A32, B32, and the FP64 residual of a reliable update
  GB_TRY(mixed_start(m, b, 0.0, 0, 0, nullptr, 0, stream));
  std::vector<cudaEvent_t> ev(4 * iterations);
  for (auto & e : ev) GB_CUDA_TRY(cudaEventCreate(&e));
  int rc = GOOSEBERRY_SUCCESS;
  for (size_t k = 0; k < iterations && rc == GOOSEBERRY_SUCCESS; ++k) {
    cudaEventRecord(ev[4 * k], stream);
    rc = launch_a32(m, stream, false, static_cast<int>(k));
    cudaEventRecord(ev[4 * k + 1], stream);
    if (rc == GOOSEBERRY_SUCCESS) rc = launch_b32(m, stream, false, static_cast<int>(k));
    cudaEventRecord(ev[4 * k + 2], stream);
    // the FP64 residual of a reliable update runs every iteration here, so
    // every iteration times it (the solve runs it only when an update is due)
    if (rc == GOOSEBERRY_SUCCESS)
      rc = launch_r(m, stream, false, static_cast<int>((k + 1) & 1), kRProfile);
    cudaEventRecord(ev[4 * k + 3], stream);
  }
  cudaError_t e = cudaStreamSynchronize(stream);
  if (rc == GOOSEBERRY_SUCCESS && e != cudaSuccess) {
    set_error("mixed CG profile failed: %s", cudaGetErrorString(e));
    rc = GOOSEBERRY_ERROR_UNKNOWN;
  }
  if (rc == GOOSEBERRY_SUCCESS) {
    double t[3] = {0, 0, 0};
    for (size_t k = 0; k < iterations; ++k)
      for (int j = 0; j < 3; ++j) {
        float v = 0.f;
        cudaEventElapsedTime(&v, ev[4 * k + j], ev[4 * k + j + 1]);
        t[j] += v;
      }
    for (size_t j = 0; j < 3 && j < ms_len; ++j) ms[j] = t[j] / iterations;
  }
  for (auto & ee : ev) cudaEventDestroy(ee);
  return rc;
}

}  // namespace gb
