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
//      reads a p value another CTA has already overwritten.
//   B  (solution / residual update + r.r)
//        x += alpha p_new;  r -= alpha Ap;  partial += r.r
//
// Each kernel ends by writing one partial sum per CTA, and EVERY CTA of the
// next kernel sums the previous kernel's partials itself, in CTA order:
// B forms p.Ap and alpha = rr / p.Ap; A forms rr from the last B (and the rr
// before it from the B before, kept in a second partial buffer), beta,
// records ||r|| and decides whether to stop (||r|| <= tol, iteration limit,
// NaN; B: breakdown).  All CTAs hold the same numbers because they add the
// same partials in the same order, so no kernel has a serial last-CTA step
// on the critical path.
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
//
// A reads the matrix in the leanest layout it allows, all summing each row's
// products in CSR order (so the iterates never depend on the layout):
//   cg_a_kernel        the CSR arrays, on the matrix's SpMV schedule
//   cg_a_codec_kernel  row schedule, compressed entries (16-bit column
//                      distances; 8-bit value codes or exact floats)
//   cg_a_ell8_kernel   pattern matrices with 8-bit value codes: a pattern byte
//                      and a row of 8 codes per row, no rowptr
//   cg_a_ellv_kernel   other pattern matrices: a pattern byte and a row of 6
//                      or 8 values (doubles, or floats when exact) per row
#include <algorithm>
#include <cmath>
#include <type_traits>
#include <vector>

#include "gb_internal.h"
#include "spmv_tiles.cuh"
#include "cg_common.cuh"

namespace gb {

namespace {

struct CgState {
  double rr;         // r.r of the current residual
  double tol;        // absolute bound on ||r||_2
  double bnorm;      // ||b||_2
  unsigned long long iter;   // iterations done (written by B, read by A)
  unsigned long long niter;  // limit (0 = none)
  unsigned long long kb;     // iteration of the running B (written by A)
  double rrk[2];             // r.r of iteration k in rrk[k & 1] (written by A)
  int done;          // 1: stop
  int status;        // gb_cg_status_t
  unsigned int ticket_i;     // the init kernel's last-CTA ticket
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

// Where A finds the r.r partials: B of iteration j writes buf[j & 1]
// (stride entries apart), the init kernel writes buf[1]; count per buffer.
// `par` = (k + 1) & 1 for the A of iteration k, fixed when the launch is
// enqueued (a graph chunk holds an even number of iterations and every solve
// starts at iteration 0), so that A reads the partials, r.r of the iteration
// before and the solver state in one round of loads.
struct RrPartials {
  const double * buf;
  unsigned count;
  unsigned stride;
  unsigned par;
};

// Start of A for iteration k = st->iter: rr_k from the last B, beta =
// rr_k / rr_{k-1} (0 at k = 0; rr_{k-1} as the previous A recorded it), the
// history entry and the stop test, which the reference makes after each
// update (src/cgd.c:115-119).  CTA 0 records the outcome.  Returns false when
// the solve stops here or has stopped already.  B's partials (every thread)
// and the state (thread 0) are loaded in one round; should `rp.par` not match
// the iteration, the partials of the right buffer are summed again.
__device__ __forceinline__ bool cg_a_begin(CgState * st, RrPartials rp, double * beta) {
  __shared__ double red[32];
  __shared__ double s_rr[2];
  __shared__ unsigned long long s_k;
  __shared__ int s_stop, s_mis;
  int done = 0;
  unsigned long long k = 0, niter = 0, hist_len = 0, hist = 0;
  double rr_prev = 0.0, tol = 0.0;
  double rr = ordered_sum_with(rp.buf + rp.par * rp.stride, rp.count, red, [&] {
    if (threadIdx.x == 0) {
      done = __ldcg(&st->done);
      k = __ldcg(&st->iter);
      rr_prev = __ldcg(&st->rrk[rp.par]);
      tol = __ldcg(&st->tol);
      niter = __ldcg(&st->niter);
      hist = __ldcg(reinterpret_cast<const unsigned long long *>(&st->hist));
      hist_len = __ldcg(&st->hist_len);
    }
  });
  if (threadIdx.x == 0) s_mis = ((k + 1) & 1) != rp.par;
  __syncthreads();
  if (s_mis) {  // parity not as enqueued: sum the other buffer
    const unsigned q = rp.par ^ 1u;
    rr = ordered_sum(rp.buf + q * rp.stride, rp.count, red);
    if (threadIdx.x == 0) rr_prev = __ldcg(&st->rrk[q]);
  }
  if (threadIdx.x == 0) {
    int stop = done ? GB_CG_CONVERGED : -1;
    if (!done) {
      if (k > 0) {
        const double rnorm = sqrt(rr);
        if (!(rnorm == rnorm) || isinf(rnorm)) stop = GB_CG_NONFINITE;
        else if (rnorm <= tol) stop = GB_CG_CONVERGED;
        else if (niter && k >= niter) stop = GB_CG_MAXITER;
        if (blockIdx.x == 0 && hist && k <= hist_len)
          reinterpret_cast<double *>(hist)[k - 1] = rnorm;
      }
      if (blockIdx.x == 0) {
        st->rr = rr;
        st->rrk[k & 1] = rr;
        st->kb = k;
        if (stop >= 0) {
          st->status = stop;
          st->done = 1;
        }
      }
    }
    s_rr[0] = rr;
    s_rr[1] = rr_prev;
    s_k = k;
    s_stop = stop;
  }
  __syncthreads();
  *beta = s_k > 0 ? s_rr[0] / s_rr[1] : 0.0;
  return s_stop < 0;
}

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
    const double s = block_sum(local, red);
    if (threadIdx.x == 0) partial[blockIdx.x] = s;
  }
};

template <int SCHED, bool HINT>
__global__ void __launch_bounds__(kSpmvBlock, MinBlocks<SCHED>::value) cg_a_kernel(const PlanView plan,
    const uint32_t * __restrict__ rowptr, const uint32_t * __restrict__ rowind,
    const double * __restrict__ val, const double * __restrict__ r,
    const double * __restrict__ pold, double * __restrict__ pnew,
    double * __restrict__ ap, double * __restrict__ longdot,
    double * __restrict__ partial, CgState * st, RrPartials rp) {
  pdl_wait_and_release();
  double beta;
  if (!cg_a_begin(st, rp, &beta)) return;
  GatherP g{r, pold, beta};
  // the row schedule finishes long rows through row() like any other row
  OutCgA o{ap, pnew, r, pold, longdot, partial, st, beta,
           SCHED == SCHED_ROW ? 0u : plan.nlong, 0.0};
  spmv_tiles_body<double, double, SCHED, kSpmvBlock, GatherP, OutCgA, false, HINT>(plan, rowptr,
      rowind, val, g, o);
}

// The row-schedule A kernel over compressed entries (RowCodec): the same
// sums, products and epilogue as cg_a_kernel<SCHED_ROW>, fewer bytes.  STAGE
// entries of a row ride in the register pipeline (sized to the longest row
// when that is short: fewer predicated slots per row).
template <class IC, class VC, bool HINT, int STAGE>
__global__ void __launch_bounds__(kSpmvBlock, MinBlocks<SCHED_ROW>::value) cg_a_codec_kernel(
    const PlanView plan, const uint32_t * __restrict__ rowptr, IC ic, VC vc,
    const double * __restrict__ table, uint32_t ntable, const double * __restrict__ r,
    const double * __restrict__ pold, double * __restrict__ pnew, double * __restrict__ ap,
    double * __restrict__ longdot, double * __restrict__ partial, CgState * st, RrPartials rp) {
  __shared__ double s_table[256];
  if constexpr (std::is_same<VC, ValCode8>::value) {
    for (uint32_t i = threadIdx.x; i < ntable; i += kSpmvBlock) s_table[i] = table[i];
    __syncthreads();
    vc.table = s_table;
  }
  pdl_wait_and_release();
  double beta;
  if (!cg_a_begin(st, rp, &beta)) return;
  GatherP g{r, pold, beta};
  OutCgA o{ap, pnew, r, pold, longdot, partial, st, beta, 0u, 0.0};
  spmv_row_loop_c<double, STAGE>(blockIdx.x * kSpmvBlock + threadIdx.x, plan.nrows,
      gridDim.x * kSpmvBlock, plan.ncols, rowptr, ic, vc, g, o, L2Pol<HINT>::stream(),
      L2Pol<HINT>::keep());
  o.finish();
}

#ifndef GB_CG_ELL
#define GB_CG_ELL 1
#endif
// The A kernels on a pattern matrix (every row at most 7 entries, at most 256
// distinct column-offset patterns): a row's column offsets and length come
// from its pattern byte and the shared-memory pattern table, its values from
// a row of 8 slots (zero-padded) that neither waits on rowptr nor on the
// pattern.  Three value rows:
//   EllCodes     8-bit codes into the shared table of distinct values (8 B per
//                row: one 8-byte load),
//   EllVals<T>   the values themselves, T = double (rows of 6 when no row has
//                more than 5 entries, else 8: three or four 16-byte loads) or
//                T = float when every double is exactly a float (rows of 8:
//                two 16-byte loads).
// The products, sums, epilogue and per-CTA partials are cg_a_codec_kernel's
// (same grid, same row order), so the iterates are identical.
__global__ void ell8_codes_kernel(uint32_t n, const uint32_t * __restrict__ rowptr,
    const uint8_t * __restrict__ code8, uint2 * __restrict__ ell8) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint32_t b = __ldg(rowptr + i), e = __ldg(rowptr + i + 1);
    uint32_t w[2] = {0u, 0u};
#pragma unroll
    for (int j = 0; j < 8; ++j)
      if (b + j < e) w[j >> 2] |= static_cast<uint32_t>(__ldg(code8 + b + j)) << (8 * (j & 3));
    ell8[i] = make_uint2(w[0], w[1]);
  }
}

// out[W i + j] = val[rowptr[i] + j] for j < the row's length, else 0.
template <typename T, int W>
__global__ void ell_vals_kernel(uint32_t n, const uint32_t * __restrict__ rowptr,
    const T * __restrict__ val, T * __restrict__ out) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint32_t b = __ldg(rowptr + i), e = __ldg(rowptr + i + 1);
#pragma unroll
    for (int j = 0; j < W; ++j)
      out[static_cast<size_t>(W) * i + j] = b + j < e ? __ldg(val + b + j) : T(0);
  }
}

struct EllCodes {
  const uint2 * rows;
  const double * table;  // shared memory
  using Row = uint2;
  __device__ __forceinline__ Row load(uint32_t i) const { return rows[i]; }
  __device__ __forceinline__ static Row zero() { return make_uint2(0u, 0u); }
  __device__ __forceinline__ double value(const Row & w, int j) const {
    return table[((j < 4 ? w.x : w.y) >> (8 * (j & 3))) & 0xffu];
  }
};

// Row width in elements for a register stage of STAGE entries.
template <typename T, int STAGE>
struct EllWidth {
  static constexpr int value = (sizeof(T) == 8 && STAGE <= 6) ? 6 : 8;
};

template <typename T, int STAGE>
struct EllVals {
  static constexpr int kW = EllWidth<T, STAGE>::value;
  static constexpr int kPer = 16 / static_cast<int>(sizeof(T));  // elements per load
  static constexpr int kVec = (STAGE + kPer - 1) / kPer;          // loads per row
  using V = typename std::conditional<sizeof(T) == 8, double2, float4>::type;
  const T * rows;
  struct Row {
    V v[kVec];
  };
  __device__ __forceinline__ Row load(uint32_t i) const {
    const V * p = reinterpret_cast<const V *>(rows + static_cast<size_t>(kW) * i);
    Row w;
#pragma unroll
    for (int k = 0; k < kVec; ++k) w.v[k] = p[k];
    return w;
  }
  __device__ __forceinline__ static Row zero() { return Row{}; }
  __device__ __forceinline__ static double elem(const double2 & v, int k) {
    return k == 0 ? v.x : v.y;
  }
  __device__ __forceinline__ static double elem(const float4 & v, int k) {
    return static_cast<double>(k == 0 ? v.x : k == 1 ? v.y : k == 2 ? v.z : v.w);
  }
  __device__ __forceinline__ double value(const Row & w, int j) const {
    return elem(w.v[j / kPer], j % kPer);
  }
};

// The row loop shared by the ELL A kernels: the next row's pattern byte,
// value row and own-row operands are loaded one row ahead.
template <int STAGE, class EV, class PM, class PX>
__device__ __forceinline__ void cg_a_ell_rows(uint32_t nrows, const uint8_t * __restrict__ pcode,
    const int32_t * s_pat, const EV & ev, const GatherP & g, OutCgA & o, PM pm, PX px) {
  const uint32_t step = gridDim.x * kSpmvBlock;
  uint32_t i = blockIdx.x * kSpmvBlock + threadIdx.x;
  if (i >= nrows) return;
  uint32_t c_cur = ld_l1_u8(pcode + i, pm);
  typename EV::Row w_cur = ev.load(i);
  OutCgA::Pre q_cur = o.pre(i);
  for (; i < nrows; i += step) {
    const uint32_t i1 = i + step;
    uint32_t c_nx = 0;
    typename EV::Row w_nx = EV::zero();
    OutCgA::Pre q_nx{};
    if (i1 < nrows) {
      c_nx = ld_l1_u8(pcode + i1, pm);
      w_nx = ev.load(i1);
      q_nx = o.pre(i1);
    }
    const int32_t * po = s_pat + c_cur * kPatMax;
    const int len = po[kPatMax - 1];
    double xv[STAGE];
#pragma unroll
    for (int j = 0; j < STAGE; ++j)
      if (j < len) xv[j] = g(i + static_cast<uint32_t>(po[j]), px);
    double sum = 0.0;
#pragma unroll
    for (int j = 0; j < STAGE; ++j)
      if (j < len) sum = add_rn(sum, mul_rn(ev.value(w_cur, j), xv[j]));
    o.row_pre(i, sum, q_cur);
    c_cur = c_nx;
    w_cur = w_nx;
    q_cur = q_nx;
  }
}

template <bool HINT, int STAGE>
__global__ void __launch_bounds__(kSpmvBlock, MinBlocks<SCHED_ROW>::value) cg_a_ell8_kernel(
    uint32_t nrows, const uint8_t * __restrict__ pcode, const int32_t * __restrict__ pat_off,
    uint32_t npat, const uint2 * __restrict__ ell8, const double * __restrict__ table,
    uint32_t ntable, const double * __restrict__ r, const double * __restrict__ pold,
    double * __restrict__ pnew, double * __restrict__ ap, double * __restrict__ partial,
    CgState * st, RrPartials rp) {
  __shared__ double s_table[256];
  __shared__ __align__(16) int32_t s_pat[256 * kPatMax];
  for (uint32_t i = threadIdx.x; i < ntable; i += kSpmvBlock) s_table[i] = table[i];
  for (uint32_t i = threadIdx.x; i < npat * kPatMax; i += kSpmvBlock) s_pat[i] = pat_off[i];
  __syncthreads();
  pdl_wait_and_release();
  double beta;
  if (!cg_a_begin(st, rp, &beta)) return;
  GatherP g{r, pold, beta};
  OutCgA o{ap, pnew, r, pold, nullptr, partial, st, beta, 0u, 0.0};
  cg_a_ell_rows<STAGE>(nrows, pcode, s_pat, EllCodes{ell8, s_table}, g, o,
      L2Pol<HINT>::stream(), L2Pol<HINT>::keep());
  o.finish();
}

template <bool HINT, int STAGE, typename T>
__global__ void __launch_bounds__(kSpmvBlock, MinBlocks<SCHED_ROW>::value) cg_a_ellv_kernel(
    uint32_t nrows, const uint8_t * __restrict__ pcode, const int32_t * __restrict__ pat_off,
    uint32_t npat, const T * __restrict__ vals, const double * __restrict__ r,
    const double * __restrict__ pold, double * __restrict__ pnew, double * __restrict__ ap,
    double * __restrict__ partial, CgState * st, RrPartials rp) {
  __shared__ __align__(16) int32_t s_pat[256 * kPatMax];
  for (uint32_t i = threadIdx.x; i < npat * kPatMax; i += kSpmvBlock) s_pat[i] = pat_off[i];
  __syncthreads();
  pdl_wait_and_release();
  double beta;
  if (!cg_a_begin(st, rp, &beta)) return;
  GatherP g{r, pold, beta};
  OutCgA o{ap, pnew, r, pold, nullptr, partial, st, beta, 0u, 0.0};
  cg_a_ell_rows<STAGE>(nrows, pcode, s_pat, EllVals<T, STAGE>{vals}, g, o,
      L2Pol<HINT>::stream(), L2Pol<HINT>::keep());
  o.finish();
}

// ---- B: x / r update and r.r ----------------------------------------------------

// Every CTA first sums A's p.Ap partials (then the long-row terms) in order
// and forms alpha = rr / p.Ap; CTA 0 records a breakdown (p.Ap <= 0) or NaN.
__global__ void __launch_bounds__(kVecBlock, kSpmvMinBlocks) cg_b_kernel(size_t n,
    double * __restrict__ x, double * __restrict__ r, const double * __restrict__ p,
    const double * __restrict__ ap, const double * __restrict__ partial_a, unsigned na,
    const double * __restrict__ longdot, unsigned nlong, double * __restrict__ partial_b,
    unsigned stride, CgState * st) {
  pdl_wait_and_release();
  __shared__ double red[32];
  __shared__ double s_pap, s_rr;
  __shared__ unsigned long long s_k;
  __shared__ int s_done;
  // A's partials (every thread) and the state (thread 0) in one round of loads
  int done = 0;
  unsigned long long kb = 0;
  double rr_st = 0.0;
  double tot = ordered_sum_with(partial_a, na, red, [&] {
    if (threadIdx.x == 0) {
      done = __ldcg(&st->done);
      kb = __ldcg(&st->kb);
      rr_st = __ldcg(&st->rr);
    }
  });
  if (threadIdx.x == 0) {
    if (!done)
      for (unsigned q = 0; q < nlong; ++q) tot += __ldcg(longdot + q);
    s_pap = tot;
    s_rr = rr_st;
    s_k = kb;
    s_done = done;
  }
  __syncthreads();
  if (s_done) return;
  const unsigned long long k = s_k;
  const double rr_cur = s_rr;
  const double pap = s_pap;
  if (!(pap > 0.0)) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      st->status = (pap == pap && rr_cur == rr_cur) ? GB_CG_BREAKDOWN : GB_CG_NONFINITE;
      st->done = 1;
    }
    return;
  }
  const double alpha = rr_cur / pap;
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
  if (threadIdx.x == 0) partial_b[(k & 1) * stride + blockIdx.x] = s;
  if (blockIdx.x == 0 && threadIdx.x == 0) st->iter = k + 1;
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
    double * ap, double * longdot, double * partial, CgState * st, RrPartials rp, unsigned grid,
    cudaStream_t s, bool pdl) {
  const size_t smem = spmv_smem(SCHED, a.plan.tile_items);
  auto kern = cg_a_kernel<SCHED, HINT>;
  GB_TRY(raise_smem_limit(reinterpret_cast<const void *>(kern), smem));
  GB_CUDA_TRY(launch_k(kern, grid, kSpmvBlock, smem, s, pdl, plan_view(a), a.rowptr,
      a.rowind, a.val64, r, pold, pnew, ap, longdot, partial, st, rp));
  return GOOSEBERRY_SUCCESS;
}

template <bool HINT>
int launch_cg_a_h(const gb_csr & a, int sched, const double * r, const double * pold,
    double * pnew, double * ap, double * longdot, double * partial, CgState * st,
    RrPartials rp, unsigned grid, cudaStream_t s, bool pdl) {
  switch (sched) {
    case GB_SCHED_THREAD:
      return launch_cg_a_t<SCHED_THREAD, HINT>(a, r, pold, pnew, ap, longdot, partial, st, rp, grid,
          s, pdl);
    case GB_SCHED_GROUP4:
      return launch_cg_a_t<SCHED_GROUP4, HINT>(a, r, pold, pnew, ap, longdot, partial, st, rp, grid,
          s, pdl);
    case GB_SCHED_GROUP8:
      return launch_cg_a_t<SCHED_GROUP8, HINT>(a, r, pold, pnew, ap, longdot, partial, st, rp, grid,
          s, pdl);
    case GB_SCHED_WARP:
      return launch_cg_a_t<SCHED_WARP, HINT>(a, r, pold, pnew, ap, longdot, partial, st, rp, grid,
          s, pdl);
    case GB_SCHED_ROW:
      return launch_cg_a_t<SCHED_ROW, HINT>(a, r, pold, pnew, ap, longdot, partial, st, rp, grid,
          s, pdl);
    case GB_SCHED_WTILE:
      return launch_cg_a_t<SCHED_WTILE, HINT>(a, r, pold, pnew, ap, longdot, partial, st, rp, grid,
          s, pdl);
    default:
      return launch_cg_a_t<SCHED_MERGE, HINT>(a, r, pold, pnew, ap, longdot, partial, st, rp, grid,
          s, pdl);
  }
}

// The A kernel with L2-policy loads (hint) or plain loads.
int launch_cg_a(const gb_csr & a, int sched, bool hint, const double * r, const double * pold,
    double * pnew, double * ap, double * longdot, double * partial, CgState * st,
    RrPartials rp, unsigned grid, cudaStream_t s, bool pdl) {
  return hint ? launch_cg_a_h<true>(a, sched, r, pold, pnew, ap, longdot, partial, st, rp, grid,
                                    s, pdl)
              : launch_cg_a_h<false>(a, sched, r, pold, pnew, ap, longdot, partial, st, rp,
                                     grid, s, pdl);
}

template <class IC, class VC, bool HINT>
int launch_cg_a_codec_t(const gb_csr & a, const RowCodec & c, const double * r,
    const double * pold, double * pnew, double * ap, double * longdot, double * partial,
    CgState * st, RrPartials rp, unsigned grid, cudaStream_t s, bool pdl, int * occ) {
  IC ic{};
  VC vc{};
  if constexpr (std::is_same<IC, ColD16>::value) ic.p = c.col16; else ic.p = a.rowind;
  if constexpr (std::is_same<VC, ValCode8>::value) {
    vc.p = c.code8;
    vc.table = nullptr;
  } else if constexpr (std::is_same<VC, ValPlain<float>>::value) {
    vc.p = c.val32;
  } else {
    vc.p = a.val64;
  }
  auto kern = c.stage == 5   ? cg_a_codec_kernel<IC, VC, HINT, 5>
              : c.stage == 7 ? cg_a_codec_kernel<IC, VC, HINT, 7>
                             : cg_a_codec_kernel<IC, VC, HINT, kRowStage>;
  if (occ) {  // occupancy query only
    GB_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(occ, kern, kSpmvBlock, 0));
    return GOOSEBERRY_SUCCESS;
  }
  GB_CUDA_TRY(launch_k(kern, grid, kSpmvBlock, 0, s, pdl, plan_view(a), a.rowptr, ic, vc,
      static_cast<const double *>(c.table), c.ntable, r, pold, pnew, ap, longdot, partial, st,
      rp));
  return GOOSEBERRY_SUCCESS;
}

template <class IC, bool HINT>
int launch_cg_a_codec_v(const gb_csr & a, const RowCodec & c, const double * r,
    const double * pold, double * pnew, double * ap, double * longdot, double * partial,
    CgState * st, RrPartials rp, unsigned grid, cudaStream_t s, bool pdl, int * occ) {
  if (c.code8)
    return launch_cg_a_codec_t<IC, ValCode8, HINT>(a, c, r, pold, pnew, ap, longdot, partial,
        st, rp, grid, s, pdl, occ);
  if (c.val32)
    return launch_cg_a_codec_t<IC, ValPlain<float>, HINT>(a, c, r, pold, pnew, ap, longdot,
        partial, st, rp, grid, s, pdl, occ);
  return launch_cg_a_codec_t<IC, ValPlain<double>, HINT>(a, c, r, pold, pnew, ap, longdot,
      partial, st, rp, grid, s, pdl, occ);
}

// The row-schedule A kernel over the solver's compressed entries (occ != null:
// only its occupancy).
int launch_cg_a_codec(const gb_csr & a, const RowCodec & c, bool hint, const double * r,
    const double * pold, double * pnew, double * ap, double * longdot, double * partial,
    CgState * st, RrPartials rp, unsigned grid, cudaStream_t s, bool pdl,
    int * occ = nullptr) {
  if (c.col16)
    return hint ? launch_cg_a_codec_v<ColD16, true>(a, c, r, pold, pnew, ap, longdot, partial,
                                                     st, rp, grid, s, pdl, occ)
                : launch_cg_a_codec_v<ColD16, false>(a, c, r, pold, pnew, ap, longdot,
                                                      partial, st, rp, grid, s, pdl, occ);
  return hint ? launch_cg_a_codec_v<ColU32, true>(a, c, r, pold, pnew, ap, longdot, partial, st,
                                                   rp, grid, s, pdl, occ)
              : launch_cg_a_codec_v<ColU32, false>(a, c, r, pold, pnew, ap, longdot, partial,
                                                    st, rp, grid, s, pdl, occ);
}

template <int SCHED>
int occupancy_cg_a(size_t smem, int * out) {
  auto kern = cg_a_kernel<SCHED, false>;
  GB_TRY(raise_smem_limit(reinterpret_cast<const void *>(kern), smem));
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
// counter with a limit (2 s unless a test sets one); on time-out the CTA
// raises `abort`, every waiting CTA leaves, and the solve reports
// GB_CG_TIMEOUT with rnorm = NaN.

constexpr unsigned long long kBarrierTimeoutNs = 2000000000ull;
// Values of the abort flag: a barrier timed out, or the host cancelled.
constexpr int kAbortTimeout = 1;
constexpr int kAbortCancel = 2;

// A host-written flag in mapped pinned memory, read past every cache.
__device__ __forceinline__ int ld_host_flag(const int * p) {
  int v;
  asm volatile("ld.volatile.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

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
// A CTA told to skip (`skip`, the failure-path test) does not arrive and
// leaves as if the barrier had been abandoned.
__device__ __forceinline__ bool grid_barrier(unsigned * counter, int * abort_flag,
    unsigned epoch, int * ok_smem, unsigned long long limit_ns, bool skip = false) {
  __syncthreads();
  if (skip) return false;
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
        if (global_ns() - t0 > limit_ns) {
          atomicExch(abort_flag, kAbortTimeout);
          ok = 0;
          break;
        }
      }
    }
    // an abort raised before the last arrival is seen by every CTA here, so
    // all of them leave at the same barrier
    if (ok && *reinterpret_cast<volatile int *>(abort_flag)) ok = 0;
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
  const int * cancel;  // host-mapped cancel request (gb_cg_cancel)
  CgState * st;
  int tol_relative;
  int keep_matrix_in_l2;
  int drop_cta;                       // failure-path test: this CTA skips barrier 1
  unsigned long long barrier_limit_ns;
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
  // CTA 0 reads the host's cancel request one phase before it acts on it, so
  // the read's latency hides behind the phase's work
  int cancel_req = 0;
  if (cta == 0 && tid == 0) cancel_req = ld_host_flag(a.cancel);
  unsigned epoch = 0;
  int status = GB_CG_MAXITER;
  unsigned long long it = 0;
  double rr = 0.0, bnorm = 0.0, tol = tol_in, beta = 0.0;
  bool aborted = false;
  const unsigned long long lim = a.barrier_limit_ns;
  if (!grid_barrier(a.sync, a.abort_flag, ++epoch, &ok_smem, lim,
                    static_cast<int>(cta) == a.drop_cta)) {
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
      // a cancel stops the solve before x moves, so x matches `it`
      if (cta == 0 && tid == 0 && cancel_req) atomicExch(a.abort_flag, kAbortCancel);
      if (!grid_barrier(a.sync, a.abort_flag, ++epoch, &ok_smem, lim)) { aborted = true; break; }
      if (cta == 0 && tid == 0) cancel_req = ld_host_flag(a.cancel);
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
      if (!grid_barrier(a.sync, a.abort_flag, ++epoch, &ok_smem, lim)) { aborted = true; break; }
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
    const bool cancelled =
        aborted && *reinterpret_cast<volatile int *>(a.abort_flag) == kAbortCancel;
    st->iter = it;
    st->rr = aborted && !cancelled ? __longlong_as_double(0x7ff8000000000000ll) : rr;
    st->bnorm = bnorm;
    st->tol = tol;
    // an abort that is not a cancel is a barrier that timed out (CTA 0 may be
    // the CTA that left without arriving: it reports the same)
    st->status = cancelled ? GB_CG_CANCELLED : (aborted ? GB_CG_TIMEOUT : status);
    st->done = 1;
  }
}

template <int SCHED>
int persistent_setup_t(size_t smem, int * occ, const void ** fn) {
  auto kern = cg_persistent_kernel<SCHED>;
  *fn = reinterpret_cast<const void *>(kern);
  GB_TRY(raise_smem_limit(*fn, smem));
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
  double * partial_b = nullptr;  // two buffers of pstride (B of even / odd iterations)
  unsigned pstride = 0;
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
  int * cancel_h = nullptr;   // pinned, mapped: set by gb_cg_cancel
  int * cancel_d = nullptr;   // its device address
  int drop_cta = -1;          // gb_cg_set_barrier_fault
  unsigned long long barrier_limit_ns = gb::kBarrierTimeoutNs;
  int keep_l2 = 0;
  bool l2_hint = false;  // A kernel with L2-policy loads (working set fits in L2)
  bool use_codec = false;  // row schedule over compressed entries
  gb::RowCodec codec;
  gb::RowPatterns pat;     // pattern matrices with coded values: rows of 8 codes
  uint2 * ell8 = nullptr;  // [n] 8 value codes per row (cg_a_ell8_kernel)
  void * ellv = nullptr;   // [n * width] values per row (cg_a_ellv_kernel)
  bool ellv_f32 = false;   // ellv holds floats (every value exactly a float)
  gb::MixedCg * mixed = nullptr;  // GB_CG_MIXED solver (owns its workspace)
};

namespace gb {
namespace {

void destroy_cg(gb_cg * s) {
  if (!s) return;
  cudaDeviceSynchronize();  // its memory goes back to the pool below
  mixed_destroy(s->mixed);
  free_row_codec(s->codec);
  free_row_patterns(s->pat);
  dev_free(s->ell8);
  dev_free(s->ellv);
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
  dev_free(s->longdot);
  dev_free(s->st);
  dev_free(s->cta_tiles);
  dev_free(s->sync);
  pinned_slot_free(s->host_status);
  pinned_slot_free(s->cancel_h);
  delete s;
}

// Stored matrix bytes per row outside the entries: rowptr, or a pattern byte
// and a row of values or codes.
size_t cg_row_bytes(const gb_cg * s) {
  if (s->ell8) return 1 + 8;
  if (s->ellv)
    return 1 + (s->ellv_f32 ? 8 * sizeof(float) : (s->codec.stage == 5 ? 6 : 8) * sizeof(double));
  return 4;
}

// The partials the A of iteration k reads (B of iteration k - 1 wrote them).
RrPartials rr_partials(const gb_cg * s, size_t k) {
  return RrPartials{s->partial_b, s->grid_b, s->pstride, static_cast<unsigned>((k + 1) & 1)};
}

// The A of iteration k (only its parity matters).
int launch_a(gb_cg * s, size_t k, const double * pold, double * pnew, cudaStream_t cs,
    bool pdl) {
  if (s->ell8) {  // same grid as the codec kernel: the same partials
    auto kern = s->codec.stage == 5
                    ? (s->l2_hint ? cg_a_ell8_kernel<true, 5> : cg_a_ell8_kernel<false, 5>)
                    : (s->l2_hint ? cg_a_ell8_kernel<true, 7> : cg_a_ell8_kernel<false, 7>);
    GB_CUDA_TRY(launch_k(kern, s->grid_a, kSpmvBlock, 0, cs, pdl,
        static_cast<uint32_t>(s->n), static_cast<const uint8_t *>(s->pat.code8),
        static_cast<const int32_t *>(s->pat.off), s->pat.npat,
        static_cast<const uint2 *>(s->ell8), static_cast<const double *>(s->codec.table),
        s->codec.ntable, static_cast<const double *>(s->r), pold, pnew, s->ap, s->partial_a,
        s->st, rr_partials(s, k)));
    return GOOSEBERRY_SUCCESS;
  }
  if (s->ellv) {  // same grid as the codec kernel: the same partials
    const auto common = [&](auto kern, const auto * vals) {
      return launch_k(kern, s->grid_a, kSpmvBlock, 0, cs, pdl, static_cast<uint32_t>(s->n),
          static_cast<const uint8_t *>(s->pat.code8), static_cast<const int32_t *>(s->pat.off),
          s->pat.npat, vals, static_cast<const double *>(s->r), pold, pnew, s->ap,
          s->partial_a, s->st, rr_partials(s, k));
    };
    const bool s5 = s->codec.stage == 5, h = s->l2_hint;
    if (s->ellv_f32) {
      const float * v = static_cast<const float *>(s->ellv);
      GB_CUDA_TRY(s5 ? (h ? common(cg_a_ellv_kernel<true, 5, float>, v)
                          : common(cg_a_ellv_kernel<false, 5, float>, v))
                     : (h ? common(cg_a_ellv_kernel<true, 7, float>, v)
                          : common(cg_a_ellv_kernel<false, 7, float>, v)));
    } else {
      const double * v = static_cast<const double *>(s->ellv);
      GB_CUDA_TRY(s5 ? (h ? common(cg_a_ellv_kernel<true, 5, double>, v)
                          : common(cg_a_ellv_kernel<false, 5, double>, v))
                     : (h ? common(cg_a_ellv_kernel<true, 7, double>, v)
                          : common(cg_a_ellv_kernel<false, 7, double>, v)));
    }
    return GOOSEBERRY_SUCCESS;
  }
  return s->use_codec
             ? launch_cg_a_codec(*s->a, s->codec, s->l2_hint, s->r, pold, pnew, s->ap,
                   s->longdot, s->partial_a, s->st, rr_partials(s, k), s->grid_a, cs, pdl)
             : launch_cg_a(*s->a, s->sched, s->l2_hint, s->r, pold, pnew, s->ap, s->longdot,
                   s->partial_a, s->st, rr_partials(s, k), s->grid_a, cs, pdl);
}

int launch_b(gb_cg * s, const double * pnew, cudaStream_t cs, bool pdl) {
  // the row schedule sums long rows like any other row: no long-row terms
  const unsigned nlong = s->sched == GB_SCHED_ROW ? 0u
                         : static_cast<unsigned>(s->a->plan.longrows.size());
  GB_CUDA_TRY(launch_k(cg_b_kernel, s->grid_b, kVecBlock, 0, cs, pdl, s->n, s->x, s->r, pnew,
      static_cast<const double *>(s->ap), static_cast<const double *>(s->partial_a), s->grid_a,
      static_cast<const double *>(s->longdot), nlong, s->partial_b, s->pstride, s->st));
  return GOOSEBERRY_SUCCESS;
}

// One chunk of iterations (A, B per iteration) and the status mirror into
// host_status[slot], on the capture stream cs.
int enqueue_chunk(gb_cg * s, int slot, cudaStream_t cs) {
  int rc = GOOSEBERRY_SUCCESS;
  for (int k = 0; k < s->chunk && rc == GOOSEBERRY_SUCCESS; ++k) {
    const double * pold = s->p[k & 1];
    double * pnew = s->p[(k + 1) & 1];
    rc = launch_a(s, static_cast<size_t>(k), pold, pnew, cs, k > 0);
    if (rc != GOOSEBERRY_SUCCESS) break;
    rc = launch_b(s, pnew, cs, true);
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
  args.cancel = s->cancel_d;
  args.st = s->st;
  args.tol_relative = tol_relative;
  args.keep_matrix_in_l2 = s->keep_l2;
  args.drop_cta = s->drop_cta;
  args.barrier_limit_ns = s->barrier_limit_ns;
  void * kargs[] = {&args};
  GB_CUDA_TRY(cudaLaunchCooperativeKernel(s->fn_p, dim3(s->grid_p), dim3(kSpmvBlock), kargs,
      s->smem_p, stream));
  return GOOSEBERRY_SUCCESS;
}

int create_cg(const gb_csr * a, int mode, gb_cg * s) {
  GB_CHECK_INPUT(a->nrows == a->ncols, "CG needs a square matrix, got %ux%u", a->nrows,
      a->ncols);
  const bool want_persistent = (mode & GB_CG_PERSISTENT) != 0;
  const bool plain_entries = (mode & GB_CG_PLAIN_ENTRIES) != 0;
  mode &= ~(GB_CG_PERSISTENT | GB_CG_PLAIN_ENTRIES);
  GB_CHECK_INPUT(mode == GB_CG_F64 || mode == GB_CG_MIXED, "unknown CG mode %d", mode);
  GB_TRY(pinned_slot_alloc(sizeof(int), reinterpret_cast<void **>(&s->cancel_h),
      reinterpret_cast<void **>(&s->cancel_d)));
  if (mode == GB_CG_MIXED) {
    s->a = a;
    s->mode = mode;
    s->n = a->nrows;
    return mixed_create(a, plain_entries, &s->mixed);
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
  // the row schedule reads compressed entries when the matrix allows it
  // (banded columns, few distinct or float-exact values)
  size_t entry_bytes = 12;
  if (s->sched == GB_SCHED_ROW && !want_persistent && !plain_entries) {
    GB_TRY(build_row_codec(*a, &s->codec, nullptr));
    s->use_codec = s->codec.col16 || s->codec.code8 || s->codec.val32;
    entry_bytes = s->codec.entry_bytes();
    // a pattern matrix: its values (or their codes) in rows of 8, no rowptr
    if (GB_CG_ELL && a->nnz > 0 && (s->codec.stage == 5 || s->codec.stage == 7)) {
      GB_TRY(build_row_patterns(*a, &s->pat, nullptr));
      if (s->pat.code8) {
        const size_t rows = std::max<size_t>(s->n, 1);
        const unsigned g = static_cast<unsigned>(std::max<size_t>(1, std::min<size_t>(
            (s->n + 255) / 256, static_cast<size_t>(a->sm_count) * 8)));
        const uint32_t nr = static_cast<uint32_t>(s->n);
        if (s->codec.code8) {
          GB_TRY(dev_alloc(&s->ell8, rows * sizeof(uint2)));
          ell8_codes_kernel<<<g, 256>>>(nr, a->rowptr, s->codec.code8, s->ell8);
        } else if (s->codec.val32) {
          GB_TRY(dev_alloc(&s->ellv, rows * 8 * sizeof(float)));
          ell_vals_kernel<float, 8><<<g, 256>>>(nr, a->rowptr, s->codec.val32,
              static_cast<float *>(s->ellv));
          s->ellv_f32 = true;
        } else if (s->codec.stage == 5) {
          GB_TRY(dev_alloc(&s->ellv, rows * 6 * sizeof(double)));
          ell_vals_kernel<double, 6><<<g, 256>>>(nr, a->rowptr, a->val64,
              static_cast<double *>(s->ellv));
        } else {
          GB_TRY(dev_alloc(&s->ellv, rows * 8 * sizeof(double)));
          ell_vals_kernel<double, 8><<<g, 256>>>(nr, a->rowptr, a->val64,
              static_cast<double *>(s->ellv));
        }
        GB_CUDA_TRY(cudaGetLastError());
        GB_CUDA_TRY(cudaDeviceSynchronize());
        entry_bytes = 0;
      }
    }
  }
  // evict-first/evict-last hints keep an L2-sized working set (matrix, rowptr,
  // r, both p, Ap, x) resident across iterations; beyond L2 the plain loads win
  GB_TRY(l2_fits(cg_row_bytes(s) * (s->n + 1) + entry_bytes * a->nnz + 40ull * s->n,
      &s->l2_hint));
  const size_t smem = spmv_smem(s->sched, a->plan.tile_items);
  int occ = 0;
  if (s->use_codec)
    GB_TRY(launch_cg_a_codec(*a, s->codec, false, nullptr, nullptr, nullptr, nullptr, nullptr,
        nullptr, nullptr, RrPartials{}, 0, nullptr, false, &occ));
  else
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
  GB_TRY(dev_alloc(&s->partial_b, 2 * static_cast<size_t>(gmax) * sizeof(double)));
  s->pstride = gmax;
  GB_TRY(dev_alloc(&s->longdot,
      std::max<size_t>(a->plan.longrows.size(), 1) * sizeof(double)));
  GB_TRY(dev_alloc(&s->st, sizeof(CgState)));
  GB_CUDA_TRY(cudaMemset(s->st, 0, sizeof(CgState)));
  GB_TRY(pinned_slot_alloc(2 * sizeof(CgStatus), reinterpret_cast<void **>(&s->host_status),
      nullptr));
  if (want_persistent) GB_TRY(setup_persistent(a, s));
  if (!s->persistent) {
    GB_CUDA_TRY(cudaStreamCreateWithFlags(&s->cap_stream, cudaStreamNonBlocking));
    GB_TRY(capture_chunk(s, 0));
    GB_TRY(capture_chunk(s, 1));
  }
  return GOOSEBERRY_SUCCESS;
}

bool cancel_requested(const gb_cg * s) {
  return __atomic_load_n(s->cancel_h, __ATOMIC_ACQUIRE) != 0;
}
void clear_cancel(gb_cg * s) { __atomic_store_n(s->cancel_h, 0, __ATOMIC_RELEASE); }

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
  // its r.r partials land where A of iteration 0 looks (the odd B buffer)
  cg_init_kernel<<<s->grid_b, kVecBlock, 0, stream>>>(s->n, b, s->x, s->r, s->p[0],
      s->partial_b + s->pstride, s->st, tol_relative);
  GB_CUDA_TRY(cudaGetLastError());
  return GOOSEBERRY_SUCCESS;
}

int solve_cg(gb_cg * s, const double * b, double * x, double tol, int tol_relative,
    size_t niter, double * history, size_t history_len, gb_cg_result_t * res,
    cudaStream_t stream) {
  if (s->mixed) {
    const int rc = mixed_solve(s->mixed, b, x, tol, tol_relative, niter, history, history_len,
        res, stream, s->cancel_h);
    if (rc == GOOSEBERRY_SUCCESS && res && res->status == GB_CG_CANCELLED) clear_cancel(s);
    return rc;
  }
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
  bool cancelled = false;
  while (rc == GOOSEBERRY_SUCCESS && !s->persistent) {
    cudaError_t e = cudaEventSynchronize(ev[slot]);
    if (e != cudaSuccess) {
      set_error("CG solve failed: %s", cudaGetErrorString(e));
      rc = GOOSEBERRY_ERROR_UNKNOWN;
      break;
    }
    if (s->host_status[slot].done) break;
    if (cancel_requested(s)) {  // the graph in flight finishes; no new one starts
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
    if (flags[1] == kAbortCancel || (cancelled && !fin.done)) {
      fin.status = GB_CG_CANCELLED;
      clear_cancel(s);
    }
    if (e != cudaSuccess) {
      set_error("CG result copy failed: %s", cudaGetErrorString(e));
      rc = GOOSEBERRY_ERROR_UNKNOWN;
    } else {
      if (flags[1] == kAbortTimeout || fin.status == GB_CG_TIMEOUT) {
        // the device is fine (every wait has a limit); the solve is not
        set_error("CG solve abandoned: a grid barrier timed out");
        rc = GOOSEBERRY_ERROR_UNKNOWN;
        fin.status = GB_CG_TIMEOUT;
      }
      if (res) {
        res->iterations = fin.iter;
        res->refinements = 0;
        res->rnorm = std::sqrt(fin.rr);
        res->bnorm = fin.bnorm;
        res->status = fin.status;
        res->kernel_launches = launches;
      }
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
    rc = launch_a(s, k, pold, pnew, stream, false);
    cudaEventRecord(ev[3 * k + 1], stream);
    if (rc == GOOSEBERRY_SUCCESS) rc = launch_b(s, pnew, stream, false);
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

int gb_cg_cancel(gb_cg_t * s) {
  GB_CHECK_INPUT(s != nullptr, "solver is NULL");
  __atomic_store_n(s->cancel_h, 1, __ATOMIC_RELEASE);
  return GOOSEBERRY_SUCCESS;
}

int gb_cg_set_barrier_fault(gb_cg_t * s, int drop_cta, unsigned limit_ms) {
  GB_CHECK_INPUT(s != nullptr, "solver is NULL");
  GB_CHECK_INPUT(drop_cta < 0 || s->persistent,
      "the barrier fault applies to GB_CG_PERSISTENT solvers only");
  GB_CHECK_INPUT(drop_cta < 0 || static_cast<unsigned>(drop_cta) < s->grid_p,
      "drop_cta %d is not a CTA of the %u-CTA solve", drop_cta, s->grid_p);
  s->drop_cta = drop_cta < 0 ? -1 : drop_cta;
  s->barrier_limit_ns = limit_ms ? static_cast<unsigned long long>(limit_ms) * 1000000ull
                                 : gb::kBarrierTimeoutNs;
  return GOOSEBERRY_SUCCESS;
}

int gb_cg_entry_bytes(const gb_cg_t * s, size_t * bytes) {
  GB_CHECK_INPUT(s != nullptr && bytes != nullptr, "NULL argument");
  *bytes = s->mixed ? mixed_entry_bytes(s->mixed)
                     : ((s->ell8 || s->ellv) ? 0 : (s->use_codec ? s->codec.entry_bytes() : 12));
  return GOOSEBERRY_SUCCESS;
}

int gb_cg_row_bytes(const gb_cg_t * s, size_t * bytes) {
  GB_CHECK_INPUT(s != nullptr && bytes != nullptr, "NULL argument");
  *bytes = s->mixed ? mixed_row_bytes(s->mixed) : gb::cg_row_bytes(s);
  return GOOSEBERRY_SUCCESS;
}

int gb_cg_profile(gb_cg_t * s, const double * b, size_t iterations, double * ms,
    size_t ms_len, size_t * nkernels, gb_stream_t stream) {
  GB_CHECK_INPUT(s != nullptr, "solver is NULL");
  return gb::profile_cg(s, b, iterations, ms, ms_len, nkernels,
      static_cast<cudaStream_t>(stream));
}

}  // extern "C"
