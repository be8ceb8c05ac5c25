// lmb_solver.cuh -- conjugate gradient on D^+D with device-resident scalars.
//
// Algorithm: cg! of the reference (cg.jl:73-137): stop when
// |r| <= max(atol, rtol |b|), report converged / maximum_iterations /
// nonpositive_curvature / numerical_breakdown.  One iteration is three
// kernels, all scalars (alpha, beta, |r|^2) stay on the GPU:
//   K1  tmp = D p                       and  pAp = |tmp|^2 = <p, D^+D p>
//   K2  Ap  = D^+ tmp (never stored):   x += alpha p,  r -= alpha Ap,  rr = |r|^2
//   K3  p   = r + beta p
// The last block of each reducing kernel computes the next scalar.  When a
// finishing condition is met the state leaves RUNNING and every later kernel
// returns at entry, so the host may enqueue several iterations between
// checks without changing the arithmetic.
//
// Mixed precision (Clark et al., "Solving lattice QCD systems of equations
// using mixed precision solvers on GPUs", CPC 181 (2010) 1517): K1-K3 run on
// FP32 or int16 fields, x_low accumulates in FP32; when |r_low| < delta *
// max|r| since the last update (or |r_low| reaches the tolerance), the state
// pauses with RELIABLE and the host performs a reliable update in FP64:
// x += x_low, x_low = 0, r = b - D^+D x, r_low = r, rr = |r|^2.  Only the
// FP64 true residual decides convergence.
#pragma once
#include "lmb_staggered.cuh"
#include "lmb_wilson.cuh"

namespace lmb {

enum CGStatus {
  ST_RUNNING = 0,
  ST_RELIABLE = 1,
  ST_CONVERGED = 2,
  ST_MAXITER = 3,
  ST_NONPOSITIVE = 4,
  ST_BREAKDOWN = 5
};

struct CGState {
  double rr;        // |r|^2 of the iterated residual
  double pAp, alpha, beta;
  double tol2;      // max(atol, rtol |b|)^2
  double maxrr;     // max |r|^2 since the last reliable update
  double delta2;    // delta^2 (0 = plain CG, no reliable updates)
  double rr_true;   // last FP64 true residual |b - D^+D x|^2
  double rr_pending;
  double bb;
  double xx;        // |x0|^2 of the initial guess
  int iter;
  int maxiter;
  int status;
  int reliable_updates;
};

LMB_D void finalize_pAp(CGState *st, double pAp) {
  st->pAp = pAp;
  if (!isfinite(pAp)) st->status = ST_BREAKDOWN;
  else if (pAp <= 0.0) st->status = ST_NONPOSITIVE;
  else st->alpha = st->rr / pAp;
}

LMB_D void finalize_rr(CGState *st, double rr_new) {
  if (!isfinite(rr_new) || rr_new < 0.0) {
    st->iter++;
    st->status = ST_BREAKDOWN;
    return;
  }
  if (st->delta2 > 0.0) {
    if (rr_new <= st->tol2 || rr_new < st->delta2 * st->maxrr) {
      st->rr_pending = rr_new;
      st->status = ST_RELIABLE;
      return;
    }
    st->maxrr = fmax(st->maxrr, rr_new);
  }
  st->iter++;
  if (st->delta2 == 0.0 && rr_new <= st->tol2) {
    st->rr = rr_new;
    st->status = ST_CONVERGED;
    return;
  }
  st->beta = rr_new / st->rr;
  st->rr = rr_new;
  if (st->iter >= st->maxiter) st->status = ST_MAXITER;
}

// mode 0: initial residual, 1: reliable update, 2: report only
LMB_D void finalize_true(CGState *st, double rr_true, int mode) {
  st->rr_true = rr_true;
  if (mode == 2) return;
  if (!isfinite(rr_true) || rr_true < 0.0) {
    st->status = ST_BREAKDOWN;
    return;
  }
  if (mode == 1) {
    st->iter++;
    st->reliable_updates++;
  }
  if (rr_true <= st->tol2) {
    st->rr = rr_true;
    st->status = ST_CONVERGED;
    return;
  }
  if (mode == 1) st->beta = rr_true / st->rr;
  st->rr = rr_true;
  st->maxrr = rr_true;
  st->status = (st->iter >= st->maxiter) ? ST_MAXITER : ST_RUNNING;
}

template <typename R>
LMB_D double sum_norm2(const Cx<R> *v, int n) {
  double s = 0;
#pragma unroll
  for (int k = 0; k < 12; k++)
    if (k < n) s += (double)norm2(v[k]);
  return s;
}

// ---------------------------------------------------------------------------
// epilogues
// ---------------------------------------------------------------------------
template <int PS, int NC = 12>
struct EpiStore {
  Field<PS, NC> out;
  const int *status;  // optional: skip when != RUNNING
  LMB_D bool skip() const { return status && *(volatile const int *)status != ST_RUNNING; }
  template <typename R> LMB_D void operator()(int s, bool active, const Cx<R> *v) const {
    if (active) out.store(s, v);
  }
  LMB_D void pair(int s0, int s1, bool active, const Cx2 *v) const {
    if (active) store2(out, s0, s1, v);
  }
  // s0 even, s1 = s0 + 1
  LMB_D void pair_adj(int s0, bool active, const Cx2 *v) const {
    if (active) store_adj(out, s0, v);
  }
  // the site-by-site interface of the FP64 pair stencils (no reduction)
  template <typename R> LMB_D void site_acc(int s, bool active, const Cx<R> *v, double (&)[1]) const {
    if (active) out.store(s, v);
  }
  LMB_D void finish(double (&)[1]) const {}
};

template <int PS, int NC = 12>
struct EpiStoreNorm {  // K1
  Field<PS, NC> out;
  CGState *st;
  double *partials;
  unsigned *counter;
  // set by the sharded operators: the grid's sum goes to *local (summed
  // over the ranks and passed to finalize() afterwards) instead of finalize
  double *local = nullptr;
  LMB_D bool skip() const { return ((volatile CGState *)st)->status != ST_RUNNING; }
  LMB_D void finalize(double total) const { finalize_pAp(st, total); }
  template <typename R> LMB_D void operator()(int s, bool active, const Cx<R> *v) const {
    double n2[1] = {0.0}, tot[1];
    if (active) {
      out.store(s, v);
      n2[0] = sum_norm2(v, NC);
    }
    if (grid_reduce<kDslashThreads, 1>(n2, partials, counter, tot) && threadIdx.x == 0) {
      if (local) *local = tot[0];
      else finalize_pAp(st, tot[0]);
    }
  }
  LMB_D void pair_adj(int s0, bool active, const Cx2 *v) const {
    double n2[1] = {0.0};
    pair_adj_acc(s0, active, v, n2);
    finish(n2);
  }
  // persistent kernels: store and add |v|^2 to red; finish() once per block
  template <typename R> LMB_D void site_acc(int s, bool active, const Cx<R> *v, double (&red)[1]) const {
    if (active) {
      out.store(s, v);
      red[0] += sum_norm2(v, NC);
    }
  }
  LMB_D void pair_adj_acc(int s0, bool active, const Cx2 *v, double (&red)[1]) const {
    if (active) {
      store_adj(out, s0, v);
      float2 q = f2(0.f);
#pragma unroll
      for (int k = 0; k < NC; k++) q = norm2_acc(v[k], q);
      red[0] += (double)q.x + (double)q.y;
    }
  }
  LMB_D void finish(double (&red)[1]) const {
    double tot[1];
    if (grid_reduce<kDslashThreads, 1>(red, partials, counter, tot) && threadIdx.x == 0) {
      if (local) *local = tot[0];
      else finalize_pAp(st, tot[0]);
    }
  }
  LMB_D void pair(int s0, int s1, bool active, const Cx2 *v) const {
    double n2[1] = {0.0}, tot[1];
    if (active) {
      store2(out, s0, s1, v);
      float2 q = f2(0.f);
#pragma unroll
      for (int k = 0; k < NC; k++) q = norm2_acc(v[k], q);
      n2[0] = (double)q.x + (double)q.y;
    }
    if (grid_reduce<kDslashThreads, 1>(n2, partials, counter, tot) && threadIdx.x == 0) {
      if (local) *local = tot[0];
      else finalize_pAp(st, tot[0]);
    }
  }
};

template <int PS, int PX, int NC = 12>
struct EpiCGUpdate {  // K2
  Field<PS, NC> p, r;
  Field<PX, NC> x;
  CGState *st;
  double *partials;
  unsigned *counter;
  double *local = nullptr;  // as EpiStoreNorm::local
  LMB_D bool skip() const { return ((volatile CGState *)st)->status != ST_RUNNING; }
  LMB_D void finalize(double total) const { finalize_rr(st, total); }
  template <typename R> LMB_D void operator()(int s, bool active, const Cx<R> *v) const {
    double n2[1] = {0.0}, tot[1];
    if (active) {
      const R alpha = (R)st->alpha;
      Cx<R> pv[NC], rv[NC], xv[NC];
      p.load(s, pv);
      r.load(s, rv);
      x.load(s, xv);
#pragma unroll
      for (int k = 0; k < NC; k++) {
        rv[k] = rv[k] - alpha * v[k];
        xv[k] = xv[k] + alpha * pv[k];
      }
      r.store(s, rv);
      x.store(s, xv);
      n2[0] = sum_norm2(rv, NC);
    }
    if (grid_reduce<kDslashThreads, 1>(n2, partials, counter, tot) && threadIdx.x == 0) {
      if (local) *local = tot[0];
      else finalize_rr(st, tot[0]);
    }
  }
  LMB_D void pair_adj(int s0, bool active, const Cx2 *v) const {
    double n2[1] = {0.0};
    pair_adj_acc(s0, active, v, n2);
    finish(n2);
  }
  // one site: update and add |r|^2 to red (the FP64 pair stencils)
  template <typename R> LMB_D void site_acc(int s, bool active, const Cx<R> *v, double (&red)[1]) const {
    if (active) {
      const R alpha = (R)st->alpha;
      Cx<R> pv[NC], rv[NC], xv[NC];
      p.load(s, pv);
      r.load(s, rv);
      x.load(s, xv);
#pragma unroll
      for (int k = 0; k < NC; k++) {
        rv[k] = rv[k] - alpha * v[k];
        xv[k] = xv[k] + alpha * pv[k];
      }
      r.store(s, rv);
      x.store(s, xv);
      red[0] += sum_norm2(rv, NC);
    }
  }
  // persistent kernels: update and add |r|^2 to red; finish() once per block
  LMB_D void pair_adj_acc(int s0, bool active, const Cx2 *v, double (&red)[1]) const {
    if (active) {
      const float a = (float)st->alpha;
      const float2 pa = f2(a), na = f2(-a);
      Cx2 pv[NC], rv[NC], xv[NC];
      load_adj_rw(p, s0, pv);
      load_adj_rw(r, s0, rv);
      load_adj_rw(x, s0, xv);
      float2 q = f2(0.f);
#pragma unroll
      for (int k = 0; k < NC; k++) {
        rv[k] = Cx2(fma2(na, v[k].re, rv[k].re), fma2(na, v[k].im, rv[k].im));
        xv[k] = Cx2(fma2(pa, pv[k].re, xv[k].re), fma2(pa, pv[k].im, xv[k].im));
        q = norm2_acc(rv[k], q);
      }
      store_adj(r, s0, rv);
      store_adj(x, s0, xv);
      red[0] += (double)q.x + (double)q.y;
    }
  }
  LMB_D void finish(double (&red)[1]) const {
    double tot[1];
    if (grid_reduce<kDslashThreads, 1>(red, partials, counter, tot) && threadIdx.x == 0) {
      if (local) *local = tot[0];
      else finalize_rr(st, tot[0]);
    }
  }
  LMB_D void pair(int s0, int s1, bool active, const Cx2 *v) const {
    double n2[1] = {0.0}, tot[1];
    if (active) {
      const float a = (float)st->alpha;
      const float2 pa = f2(a), na = f2(-a);
      Cx2 pv[NC], rv[NC], xv[NC];
      load2(p, s0, s1, pv);
      load2(r, s0, s1, rv);
      load2(x, s0, s1, xv);
      float2 q = f2(0.f);
#pragma unroll
      for (int k = 0; k < NC; k++) {
        rv[k] = Cx2(fma2(na, v[k].re, rv[k].re), fma2(na, v[k].im, rv[k].im));
        xv[k] = Cx2(fma2(pa, pv[k].re, xv[k].re), fma2(pa, pv[k].im, xv[k].im));
        q = norm2_acc(rv[k], q);
      }
      store2(r, s0, s1, rv);
      store2(x, s0, s1, xv);
      n2[0] = (double)q.x + (double)q.y;
    }
    if (grid_reduce<kDslashThreads, 1>(n2, partials, counter, tot) && threadIdx.x == 0) {
      if (local) *local = tot[0];
      else finalize_rr(st, tot[0]);
    }
  }
};

// epilogues that the persistent two-site kernels drive (pair_adj_acc +
// finish: the reduction carried in registers across tiles).  K2's update
// has pair_adj_acc too, but its longer tiles measured faster one block per
// tile (32^3x64 int16: 0.269 against 0.272 ms; K1 0.213 against 0.221 ms).
template <class Epi> struct PersistentEpi { static constexpr bool value = false; };
template <int PS, int NC> struct PersistentEpi<EpiStoreNorm<PS, NC>> { static constexpr bool value = true; };

// the first pass of a two-pass operator: a plain store that skips whenever
// the epilogue of the second pass does (a paused CG skips every pass)
template <int PS, class Follow>
struct EpiStoreFollow {
  Field<PS, 12> out;
  Follow follow;
  LMB_D bool skip() const { return follow.skip(); }
  template <typename R> LMB_D void operator()(int s, bool active, const Cx<R> *v) const {
    if (active) out.store(s, v);
  }
};

// |b - v|^2 summed over the grid into *out (no CG state)
template <int NC = 12>
struct EpiResidualNorm {
  Field<PREC_DOUBLE, NC> b;
  double *partials;
  unsigned *counter;
  double *out;
  double *local = nullptr;  // as EpiStoreNorm::local
  LMB_D bool skip() const { return false; }
  LMB_D void finalize(double total) const { *out = total; }
  template <typename R> LMB_D void operator()(int s, bool active, const Cx<R> *v) const {
    double n2[1] = {0.0}, tot[1];
    if (active) {
      Cx<double> bv[NC];
      b.load(s, bv);
#pragma unroll
      for (int k = 0; k < NC; k++) {
        const double dr = bv[k].re - (double)v[k].re, di = bv[k].im - (double)v[k].im;
        n2[0] += dr * dr + di * di;
      }
    }
    if (grid_reduce<kDslashThreads, 1>(n2, partials, counter, tot) && threadIdx.x == 0) {
      if (local) *local = tot[0];
      else *out = tot[0];
    }
  }
};

// r = b - v (FP64), r_low = r (optional), |r|^2 -> finalize_true(mode)
template <int PS, int NC = 12>
struct EpiTrueResidual {
  Field<PREC_DOUBLE, NC> b, r;
  Field<PS, NC> r_low;
  int write_low;
  int mode;
  CGState *st;
  double *partials;
  unsigned *counter;
  double *local = nullptr;  // as EpiStoreNorm::local
  LMB_D bool skip() const { return false; }
  LMB_D void finalize(double total) const { finalize_true(st, total, mode); }
  template <typename R> LMB_D void operator()(int s, bool active, const Cx<R> *v) const {
    double n2[1] = {0.0}, tot[1];
    if (active) {
      Cx<double> bv[NC], rv[NC];
      b.load(s, bv);
#pragma unroll
      for (int k = 0; k < NC; k++) rv[k] = Cx<double>(bv[k].re - (double)v[k].re, bv[k].im - (double)v[k].im);
      r.store(s, rv);
      if (write_low) r_low.store(s, rv);
      n2[0] = sum_norm2(rv, NC);
    }
    if (grid_reduce<kDslashThreads, 1>(n2, partials, counter, tot) && threadIdx.x == 0) {
      if (local) *local = tot[0];
      else finalize_true(st, tot[0], mode);
    }
  }
};

// epilogues whose kernels end in a grid reduction (a `local` slot and
// finalize(total)); the sharded operators sum the slot over the ranks
template <class Epi> struct ReducingEpi { static constexpr bool value = false; };
template <int PS, int NC> struct ReducingEpi<EpiStoreNorm<PS, NC>> { static constexpr bool value = true; };
template <int PS, int PX, int NC> struct ReducingEpi<EpiCGUpdate<PS, PX, NC>> { static constexpr bool value = true; };
template <int NC> struct ReducingEpi<EpiResidualNorm<NC>> { static constexpr bool value = true; };
template <int PS, int NC> struct ReducingEpi<EpiTrueResidual<PS, NC>> { static constexpr bool value = true; };

// ---------------------------------------------------------------------------
// vector kernels
// ---------------------------------------------------------------------------
constexpr int kBlasThreads = 256;

// K3: p = r + beta p
template <int PS, int NC>
__global__ void __launch_bounds__(kBlasThreads)
    cg_p_update_kernel(Field<PS, NC> p, const Field<PS, NC> r, const CGState *st, int64_t V) {
  if (((volatile const CGState *)st)->status != ST_RUNNING) return;
  const int64_t s = (int64_t)blockIdx.x * kBlasThreads + threadIdx.x;
  if (s >= V) return;
  typedef typename Real<PS>::type R;
  const R beta = (R)st->beta;
  Cx<R> pv[NC], rv[NC];
  p.load(s, pv);
  r.load(s, rv);
#pragma unroll
  for (int k = 0; k < NC; k++) pv[k] = rv[k] + beta * pv[k];
  p.store(s, pv);
}

// K3 on x-adjacent site pairs (V even; FP32 or int16 storage, NC = 12):
// packed FP32 and 256-bit loads / stores, V/2 threads
template <int PS>
__global__ void __launch_bounds__(kBlasThreads)
    cg_p_update_adj_kernel(Field<PS, 12> p, const Field<PS, 12> r, const CGState *st, int64_t V) {
  if (((volatile const CGState *)st)->status != ST_RUNNING) return;
  const int64_t s = 2 * ((int64_t)blockIdx.x * kBlasThreads + threadIdx.x);
  if (s >= V) return;
  const float2 beta = f2((float)st->beta);
  Cx2 pv[12], rv[12];
  load_adj_rw(p, s, pv);
  load_adj_rw(r, s, rv);
#pragma unroll
  for (int k = 0; k < 12; k++) pv[k] = Cx2(fma2(beta, pv[k].re, rv[k].re), fma2(beta, pv[k].im, rv[k].im));
  store_adj(p, s, pv);
}

// dst = src (precision conversion)
template <int PD, int PSRC, int NC>
__global__ void __launch_bounds__(kBlasThreads)
    convert_kernel(Field<PD, NC> dst, const Field<PSRC, NC> src, int64_t V) {
  const int64_t s = (int64_t)blockIdx.x * kBlasThreads + threadIdx.x;
  if (s >= V) return;
  typedef typename Real<PD>::type RD;
  typedef typename Real<PSRC>::type RS;
  Cx<RS> a[NC];
  Cx<RD> b[NC];
  src.load(s, a);
#pragma unroll
  for (int k = 0; k < NC; k++) b[k] = Cx<RD>((RD)a[k].re, (RD)a[k].im);
  dst.store(s, b);
}

// x64 += x_low; x_low = 0
template <int PX, int NC>
__global__ void __launch_bounds__(kBlasThreads)
    fold_kernel(Field<PREC_DOUBLE, NC> x, Field<PX, NC> xl, int64_t V) {
  const int64_t s = (int64_t)blockIdx.x * kBlasThreads + threadIdx.x;
  if (s >= V) return;
  typedef typename Real<PX>::type RX;
  Cx<double> a[NC];
  Cx<RX> b[NC], z[NC];
  x.load(s, a);
  xl.load(s, b);
#pragma unroll
  for (int k = 0; k < NC; k++) {
    a[k] = Cx<double>(a[k].re + (double)b[k].re, a[k].im + (double)b[k].im);
    z[k] = Cx<RX>(0, 0);
  }
  x.store(s, a);
  xl.store(s, z);
}

// |b|^2 into st->bb and the tolerance, |x0|^2 into st->xx
template <int NC>
__global__ void __launch_bounds__(kBlasThreads)
    norm_bx_kernel(const Field<PREC_DOUBLE, NC> b, const Field<PREC_DOUBLE, NC> x, CGState *st, int64_t V,
                   double rtol, double atol, double *partials, unsigned *counter, double *local2 = nullptr) {
  const int64_t s = (int64_t)blockIdx.x * kBlasThreads + threadIdx.x;
  double n2[2] = {0.0, 0.0}, tot[2];
  if (s < V) {
    Cx<double> v[NC];
    b.load(s, v);
#pragma unroll
    for (int k = 0; k < NC; k++) n2[0] += norm2(v[k]);
    x.load(s, v);
#pragma unroll
    for (int k = 0; k < NC; k++) n2[1] += norm2(v[k]);
  }
  if (grid_reduce<kBlasThreads, 2>(n2, partials, counter, tot) && threadIdx.x == 0) {
    if (local2) {  // a block of a process grid: summed over the ranks first
      local2[0] = tot[0];
      local2[1] = tot[1];
      return;
    }
    st->bb = tot[0];
    st->xx = tot[1];
    const double bn = sqrt(tot[0]);
    const double tol = fmax(atol, rtol * bn);
    st->tol2 = tol * tol;
  }
}

// |b|^2, |x0|^2 and the tolerance from the sums over the ranks
template <int = 0>
__global__ void set_norms_kernel(CGState *st, const double *sums, double rtol, double atol) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  st->bb = sums[0];
  st->xx = sums[1];
  const double tol = fmax(atol, rtol * sqrt(sums[0]));
  st->tol2 = tol * tol;
}

// the initial residual of a zero guess: r = b, r_low = r (optional),
// |r|^2 -> finalize_true(mode); blocks of kDslashThreads sites, the partition
// of the stencil epilogue it replaces (same reduction order)
template <int PS, int NC>
__global__ void __launch_bounds__(kDslashThreads)
    residual_of_zero_kernel(const Field<PREC_DOUBLE, NC> b, Field<PREC_DOUBLE, NC> r, Field<PS, NC> r_low,
                            int write_low, int mode, CGState *st, int64_t V, double *partials, unsigned *counter) {
  const int64_t s = (int64_t)blockIdx.x * kDslashThreads + threadIdx.x;
  double n2[1] = {0.0}, tot[1];
  if (s < V) {
    Cx<double> v[NC];
    b.load(s, v);
    r.store(s, v);
    if (write_low) r_low.store(s, v);
    n2[0] = sum_norm2(v, NC);
  }
  if (grid_reduce<kDslashThreads, 1>(n2, partials, counter, tot) && threadIdx.x == 0) finalize_true(st, tot[0], mode);
}

// |a|^2 into st->bb and the tolerance
template <int NC>
__global__ void __launch_bounds__(kBlasThreads)
    norm_b_kernel(const Field<PREC_DOUBLE, NC> a, CGState *st, int64_t V, double rtol, double atol,
                  double *partials, unsigned *counter) {
  const int64_t s = (int64_t)blockIdx.x * kBlasThreads + threadIdx.x;
  double n2[1] = {0.0}, tot[1];
  if (s < V) {
    Cx<double> v[NC];
    a.load(s, v);
#pragma unroll
    for (int k = 0; k < NC; k++) n2[0] += norm2(v[k]);
  }
  if (grid_reduce<kBlasThreads, 1>(n2, partials, counter, tot) && threadIdx.x == 0) {
    st->bb = tot[0];
    const double bn = sqrt(tot[0]);
    const double tol = fmax(atol, rtol * bn);
    st->tol2 = tol * tol;
  }
}

}  // namespace lmb
