// lmb_staggered.cuh -- staggered and HISQ stencils on CUDA cores.
//
//   D psi = m psi + fc sum_mu eta_mu(x) [X_mu(x) psi(x+mu) - X_mu(x-mu)^+ psi(x-mu)]
//                 + lc sum_mu eta_mu(x) [L_mu(x) psi(x+3mu) - L_mu(x-3mu)^+ psi(x-3mu)]
// with fc = 1/2, lc = -(1+eps)/48 for D and both negated for D^+
// (StaggeredDiracOperator.jl:1-17, 129-198; HISQDiracOperator.jl:55-72,
// 269-357).  Plain staggered is the case without the Naik term.
// eta_mu(x) = (-1)^(sum_{nu<mu} x_nu) with zero-based GLOBAL coordinates
// (LinearAlgebras/staggered.jl:43-57): the rank offset is Geom::eta_off.
// Fermion boundary phases: a wrap forward multiplies by phase, backward by
// 1/phase, per wrap (a Naik hop on an extent below 3 may wrap twice).
#pragma once
#include "lmb_common.cuh"
#include "lmb_wilson.cuh"

namespace lmb {

constexpr int kStagThreads = kDslashThreads;  // the epilogue reductions assume it
// minimum resident blocks per SM requested for the one-site stencil and its
// persistent form
#ifndef LMB_STAG_MINB
#define LMB_STAG_MINB 0
#endif
#ifndef LMB_STAG_PMINB
#define LMB_STAG_PMINB 4
#endif
#ifndef LMB_STAG_K2MINB
#define LMB_STAG_K2MINB 4
#endif

// neighbour at signed distance d along mu with the number of edge crossings
// (the loops run at most once on extents >= 3; measured faster on B200 than
// an unrolled branch-free form)
LMB_D int shift_site_any(const Geom &g, int s, const int *c, int mu, int d, int *wraps) {
  const int L = g.L[mu];
  int raw = c[mu] + d;
  int w = 0;
  while (raw >= L) {
    raw -= L;
    w++;
  }
  while (raw < 0) {
    raw += L;
    w--;
  }
  *wraps = w;
  return s + (raw - c[mu]) * g.stride[mu];
}

template <typename R>
LMB_D void apply_wraps(const Geom &g, int mu, int wraps, Cx<R> *v) {
  if (!wraps || !((g.phase_mask >> mu) & 1)) return;
  const double *ph = wraps > 0 ? g.ph_fwd[mu] : g.ph_bwd[mu];
  const Cx<R> f((R)ph[0], (R)ph[1]);
  const int n = wraps > 0 ? wraps : -wraps;
  for (int k = 0; k < n; k++)
#pragma unroll
    for (int i = 0; i < 3; i++) v[i] = v[i] * f;
}

template <typename R>
LMB_D void su3_mul_vec(const Cx<R> *u, const Cx<R> *v, Cx<R> *o) {
#pragma unroll
  for (int r = 0; r < 3; r++) {
    Cx<R> t = u[r] * v[0];
    t = cfma(u[r + 3], v[1], t);
    o[r] = cfma(u[r + 6], v[2], t);
  }
}
template <typename R>
LMB_D void su3_adj_mul_vec(const Cx<R> *u, const Cx<R> *v, Cx<R> *o) {
#pragma unroll
  for (int r = 0; r < 3; r++) {
    Cx<R> t = conj(u[3 * r]) * v[0];
    t = cfma_conj(u[3 * r + 1], v[1], t);
    o[r] = cfma_conj(u[3 * r + 2], v[2], t);
  }
}

// neighbour at +d / -d (d <= 3) on an extent >= d: at most one crossing,
// selected without a branch (the form of fwd_site / bwd_site)
LMB_D int shift_site_sel(const Geom &g, int s, const int *c, int mu, int d, int *wraps) {
  const int L = g.L[mu];
  if (d > 0) {
    const int up = c[mu] + d >= L;
    *wraps = up;
    return s + (up ? d - L : d) * g.stride[mu];
  }
  const int dn = c[mu] + d < 0;
  *wraps = -dn;
  return s + (dn ? d + L : d) * g.stride[mu];
}

// PH_T (only the t phase may differ from 1, T >= 3 so that a hop crosses
// the edge at most once): multiply every t hop by the selected factor
template <typename R>
LMB_D void apply_wrap_sel(const Geom &g, int wraps, Cx<R> *v) {
  const double *ph = wraps > 0 ? g.ph_fwd[3] : g.ph_bwd[3];
  const Cx<R> f(wraps ? (R)ph[0] : (R)1, wraps ? (R)ph[1] : (R)0);
#pragma unroll
  for (int i = 0; i < 3; i++) v[i] = v[i] * f;
}

// forward minus backward hop of one direction at distance D, into acc
template <typename R, int MU, int D, int PHM, class SF, class G>
LMB_D void stag_hop(const Geom &g, int s, const int *c, const SF &in, const G &U, R eta, Cx<R> *acc) {
  Cx<R> v[3], u[9], o[3];
  int w;
  // PH_T launches only on extents >= 3: at most one crossing per hop
  const int sp = (D == 1)          ? fwd_site(g, s, c, MU, 1, &w)
                 : (PHM == PH_ANY) ? shift_site_any(g, s, c, MU, D, &w)
                                   : shift_site_sel(g, s, c, MU, D, &w);
  in.load(sp, v);
  if constexpr (PHM == PH_ANY) apply_wraps(g, MU, w, v);
  else if constexpr (MU == 3) apply_wrap_sel(g, w, v);
  U.load(MU, s, u);
  su3_mul_vec(u, v, o);
#pragma unroll
  for (int i = 0; i < 3; i++) acc[i] = acc[i] + eta * o[i];
  int wb;
  const int sm = (D == 1)          ? bwd_site(g, s, c, MU, 1, &wb)
                 : (PHM == PH_ANY) ? shift_site_any(g, s, c, MU, -D, &wb)
                                   : shift_site_sel(g, s, c, MU, -D, &wb);
  if (D == 1 && wb) wb = -1;
  in.load(sm, v);
  if constexpr (PHM == PH_ANY) apply_wraps(g, MU, wb, v);
  else if constexpr (MU == 3) apply_wrap_sel(g, wb, v);
  U.load(MU, sm, u);
  su3_adj_mul_vec(u, v, o);
#pragma unroll
  for (int i = 0; i < 3; i++) acc[i] = acc[i] - eta * o[i];
}

struct NoLinks {
  int64_t V;
  template <typename R> LMB_D void load(int, int64_t, Cx<R> *) const {}
};

// D psi at site s (3 components)
template <typename R, bool NAIK, int PHM, class SF, class GF, class GL>
LMB_D void stag_site(const Geom &g, int s, const SF &in, const GF &X, const GL &Lk, R mass, R fc, R lc,
                     Cx<R> *out) {
  int c[4];
  site_coords(g, s, c);
  const int p0 = c[0] + g.eta_off[0], p1 = p0 + c[1] + g.eta_off[1], p2 = p1 + c[2] + g.eta_off[2];
  const R eta[4] = {(R)1, (p0 & 1) ? (R)-1 : (R)1, (p1 & 1) ? (R)-1 : (R)1, (p2 & 1) ? (R)-1 : (R)1};
  Cx<R> fat[3] = {Cx<R>(0, 0), Cx<R>(0, 0), Cx<R>(0, 0)};
  stag_hop<R, 0, 1, PHM>(g, s, c, in, X, eta[0], fat);
  stag_hop<R, 1, 1, PHM>(g, s, c, in, X, eta[1], fat);
  stag_hop<R, 2, 1, PHM>(g, s, c, in, X, eta[2], fat);
  stag_hop<R, 3, 1, PHM>(g, s, c, in, X, eta[3], fat);
  Cx<R> psi[3];
  in.load(s, psi);
  if constexpr (NAIK) {
    Cx<R> lng[3] = {Cx<R>(0, 0), Cx<R>(0, 0), Cx<R>(0, 0)};
    stag_hop<R, 0, 3, PHM>(g, s, c, in, Lk, eta[0], lng);
    stag_hop<R, 1, 3, PHM>(g, s, c, in, Lk, eta[1], lng);
    stag_hop<R, 2, 3, PHM>(g, s, c, in, Lk, eta[2], lng);
    stag_hop<R, 3, 3, PHM>(g, s, c, in, Lk, eta[3], lng);
#pragma unroll
    for (int i = 0; i < 3; i++) out[i] = mass * psi[i] + fc * fat[i] + lc * lng[i];
  } else {
#pragma unroll
    for (int i = 0; i < 3; i++) out[i] = mass * psi[i] + fc * fat[i];
  }
}

template <int PS, int NC> struct EpiStore;  // lmb_solver.cuh
template <int PS, int NC> struct EpiStoreNorm;
template <int PS, int PX, int NC> struct EpiCGUpdate;

// resident blocks per SM requested from the register allocator: the plain
// FP64 store (mul!, the Dslash rate) is latency bound at 104 registers and
// runs ~11 % faster with five 128-thread blocks per SM (96 registers); the
// CG epilogues spill at that bound and keep the default, except the
// persistent K1 and the K2 update, whose four blocks per SM (128
// registers, a few words spilled) measured faster than three (48^3x96 FP64
// HISQ: K1 3.42 against 3.60 ms, K2 3.87 against 4.34 ms)
template <typename R, class Epi> struct StagMinBlocks { static constexpr int value = LMB_STAG_MINB; };
template <int NC> struct StagMinBlocks<double, EpiStore<PREC_DOUBLE, NC>> { static constexpr int value = 5; };
template <int NC> struct StagMinBlocks<double, EpiCGUpdate<PREC_DOUBLE, PREC_DOUBLE, NC>> {
  static constexpr int value = LMB_STAG_K2MINB;
};

// Epi as for the Wilson kernel, on 3-component fields
template <typename R, bool NAIK, int PHM, class SF, class GF, class GL, class Epi>
__global__ void __launch_bounds__(kStagThreads, (StagMinBlocks<R, Epi>::value))
    staggered_dslash_kernel(const Geom g, const SF in, const GF X, const GL Lk, const R mass, const R fc,
                            const R lc, Epi epi, const SiteRange rg) {
  if (epi.skip()) return;
  const int s = rg.lo + blockIdx.x * kStagThreads + threadIdx.x;
  const bool active = s < rg.hi;
  Cx<R> out[3];
  if (active) stag_site<R, NAIK, PHM>(g, s, in, X, Lk, mass, fc, lc, out);
  epi(s, active, out);
}

// Persistent form for the reducing CG epilogues (see
// wilson_half_adj_persistent_kernel): the resident blocks walk the tiles in a
// fixed order, the reduction is carried in registers and done once per block
template <typename R, bool NAIK, int PHM, class SF, class GF, class GL, class Epi>
__global__ void __launch_bounds__(kStagThreads, LMB_STAG_PMINB)
    staggered_persistent_kernel(const Geom g, const SF in, const GF X, const GL Lk, const R mass, const R fc,
                                const R lc, Epi epi, int ntiles, const SiteRange rg) {
  if (epi.skip()) return;
  double red[1] = {0.0};
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int s = rg.lo + tile * kStagThreads + threadIdx.x;
    const bool active = s < rg.hi;
    Cx<R> out[3];
    if (active) stag_site<R, NAIK, PHM>(g, s, in, X, Lk, mass, fc, lc, out);
    epi.site_acc(s, active, out, red);
  }
  epi.finish(red);
}

// ---------------------------------------------------------------------------
// FP32 / int16-storage HISQ and staggered stencil on x-adjacent site pairs
// (s0 = 2i, s1 = s0 + 1) with packed FP32 arithmetic and 256-bit loads
// (lmb_pair.cuh).  Conditions
// of the PH_T mode (only the t phase, every extent >= 3) and an even x
// extent; 18-real FP32 links.  eta_mu for mu >= 1 is opposite on the two
// lanes (x and x + 1).
// ---------------------------------------------------------------------------
LMB_D void su3_mul_vec2(const Cx2 *u, const Cx2 *v, Cx2 *o) {
#pragma unroll
  for (int r = 0; r < 3; r++) o[r] = cfma(u[r + 6], v[2], cfma(u[r + 3], v[1], u[r] * v[0]));
}
LMB_D void su3_adj_mul_vec2(const Cx2 *u, const Cx2 *v, Cx2 *o) {
#pragma unroll
  for (int r = 0; r < 3; r++) {
    const Cx2 a = u[3 * r], b = v[0];
    const Cx2 t(fma2(a.im, b.im, a.re * b.re), fma2(-a.im, b.re, a.re * b.im));
    o[r] = cfma_conj(u[3 * r + 2], v[2], cfma_conj(u[3 * r + 1], v[1], t));
  }
}
LMB_D void phase_t_sel(const Geom &g, int wraps, Cx2 *v) {
  const double *ph = wraps > 0 ? g.ph_fwd[3] : g.ph_bwd[3];
  const float pr = wraps ? (float)ph[0] : 1.f, pi = wraps ? (float)ph[1] : 0.f;
  const Cx2 f(f2(pr), f2(pi));
#pragma unroll
  for (int i = 0; i < 3; i++) v[i] = v[i] * f;
}

// acc += eta [U(x) psi(x + D mu) - U(x - D mu)^+ psi(x - D mu)]; fields and
// 18-real links stored as FP32 (PS = PREC_SINGLE) or int16 (PREC_HALF)
template <int MU, int D, int PS>
LMB_D void stag_hop_adj(const Geom &g, int s0, const int *c0, const int *c1, const Field<PS, 3> &in,
                        const Gauge<PS> &U, float2 eta, Cx2 *acc) {
  Cx2 v[3], u[9], o[3];
  int w0, w1;
  if constexpr (MU == 0) {
    const int n0 = shift_site_sel(g, s0, c0, 0, D, &w0), n1 = shift_site_sel(g, s0 + 1, c1, 0, D, &w1);
    load2(in, n0, n1, v);
  } else {
    const int n = (D == 1) ? fwd_site(g, s0, c0, MU, 1, &w0) : shift_site_sel(g, s0, c0, MU, D, &w0);
    load_adj(in, n, v);
    if constexpr (MU == 3) phase_t_sel(g, w0, v);
  }
  load_adj(U, MU, s0, u);
  su3_mul_vec2(u, v, o);
#pragma unroll
  for (int i = 0; i < 3; i++) acc[i] = Cx2(fma2(eta, o[i].re, acc[i].re), fma2(eta, o[i].im, acc[i].im));
  if constexpr (MU == 0) {
    const int n0 = shift_site_sel(g, s0, c0, 0, -D, &w0), n1 = shift_site_sel(g, s0 + 1, c1, 0, -D, &w1);
    load2(in, n0, n1, v);
    load2(U, 0, n0, n1, u);
  } else {
    const int n = (D == 1) ? bwd_site(g, s0, c0, MU, 1, &w0) : shift_site_sel(g, s0, c0, MU, -D, &w0);
    if (D == 1 && w0) w0 = -1;
    load_adj(in, n, v);
    if constexpr (MU == 3) phase_t_sel(g, w0, v);
    load_adj(U, MU, n, u);
  }
  su3_adj_mul_vec2(u, v, o);
#pragma unroll
  for (int i = 0; i < 3; i++) acc[i] = Cx2(fma2(-eta, o[i].re, acc[i].re), fma2(-eta, o[i].im, acc[i].im));
}

// D psi at the x-adjacent sites s0 (x even) and s0 + 1
template <bool NAIK, int PS>
LMB_D void stag_adj_sites(const Geom &g, int s0, const Field<PS, 3> &in, const Gauge<PS> &X, const Gauge<PS> &Lk,
                          float mass, float fc, float lc, Cx2 *out) {
  int c0[4], c1[4];
  site_coords(g, s0, c0);
  c1[0] = c0[0] + 1;
  c1[1] = c0[1];
  c1[2] = c0[2];
  c1[3] = c0[3];
  const int p0 = c0[0] + g.eta_off[0], p1 = p0 + c0[1] + g.eta_off[1], p2 = p1 + c0[2] + g.eta_off[2];
  const float e1 = (p0 & 1) ? -1.f : 1.f, e2 = (p1 & 1) ? -1.f : 1.f, e3 = (p2 & 1) ? -1.f : 1.f;
  const float2 eta0 = f2(1.f), eta1 = f2(e1, -e1), eta2 = f2(e2, -e2), eta3 = f2(e3, -e3);
  Cx2 fat[3] = {cx2_zero(), cx2_zero(), cx2_zero()};
  stag_hop_adj<0, 1, PS>(g, s0, c0, c1, in, X, eta0, fat);
  stag_hop_adj<1, 1, PS>(g, s0, c0, c1, in, X, eta1, fat);
  stag_hop_adj<2, 1, PS>(g, s0, c0, c1, in, X, eta2, fat);
  stag_hop_adj<3, 1, PS>(g, s0, c0, c1, in, X, eta3, fat);
  Cx2 psi[3];
  load_adj(in, s0, psi);
  const float2 m2 = f2(mass), f2c = f2(fc);
  if constexpr (NAIK) {
    Cx2 lng[3] = {cx2_zero(), cx2_zero(), cx2_zero()};
    stag_hop_adj<0, 3, PS>(g, s0, c0, c1, in, Lk, eta0, lng);
    stag_hop_adj<1, 3, PS>(g, s0, c0, c1, in, Lk, eta1, lng);
    stag_hop_adj<2, 3, PS>(g, s0, c0, c1, in, Lk, eta2, lng);
    stag_hop_adj<3, 3, PS>(g, s0, c0, c1, in, Lk, eta3, lng);
    const float2 l2 = f2(lc);
#pragma unroll
    for (int k = 0; k < 3; k++)
      out[k] = Cx2(fma2(l2, lng[k].re, fma2(f2c, fat[k].re, m2 * psi[k].re)),
                   fma2(l2, lng[k].im, fma2(f2c, fat[k].im, m2 * psi[k].im)));
  } else {
#pragma unroll
    for (int k = 0; k < 3; k++)
      out[k] = Cx2(fma2(f2c, fat[k].re, m2 * psi[k].re), fma2(f2c, fat[k].im, m2 * psi[k].im));
  }
}

// one thread per pair of the range (rg.lo, rg.hi even).  Epi must provide
// skip() and pair_adj(s0, active, out[3]).
template <bool NAIK, int PS, class Epi>
__global__ void __launch_bounds__(kStagThreads, LMB_PAIR_MINB)
    staggered_adj_kernel(const Geom g, const Field<PS, 3> in, const Gauge<PS> X, const Gauge<PS> Lk,
                         const float mass, const float fc, const float lc, Epi epi, const SiteRange rg) {
  if (epi.skip()) return;
  const int i = blockIdx.x * kStagThreads + threadIdx.x;
  const bool active = i < ((rg.hi - rg.lo) >> 1);
  const int s0 = rg.lo + 2 * i;
  Cx2 out[3];
  if (active) stag_adj_sites<NAIK, PS>(g, s0, in, X, Lk, mass, fc, lc, out);
  epi.pair_adj(s0, active, out);
}

// persistent form for the reducing CG epilogues (as the Wilson pair kernel)
template <bool NAIK, int PS, class Epi>
__global__ void __launch_bounds__(kStagThreads, LMB_PAIR_MINB)
    staggered_adj_persistent_kernel(const Geom g, const Field<PS, 3> in, const Gauge<PS> X, const Gauge<PS> Lk,
                                    const float mass, const float fc, const float lc, Epi epi, int ntiles,
                                    const SiteRange rg) {
  if (epi.skip()) return;
  double red[1] = {0.0};
  const int npairs = (rg.hi - rg.lo) >> 1;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int i = tile * kStagThreads + threadIdx.x;
    const bool active = i < npairs;
    const int s0 = rg.lo + 2 * i;
    Cx2 out[3];
    if (active) stag_adj_sites<NAIK, PS>(g, s0, in, X, Lk, mass, fc, lc, out);
    epi.pair_adj_acc(s0, active, out, red);
  }
  epi.finish(red);
}

// ---------------------------------------------------------------------------
// FP64 HISQ / staggered stencil on x-adjacent site pairs.  FP64 has no packed
// arithmetic: the point is the loads.  The one-site FP64 stencil is bound by
// the latency of its 16 gathers of 12 loads each (long-scoreboard stalls,
// FP64 pipe ~15 % busy); here one 256-bit load per plane serves both sites
// of every y, z, t hop and of the site's own links, so each load instruction
// carries twice the bytes.  Same conditions as the FP32 pair stencil (PH_T,
// even x extent, 18-real links).
// ---------------------------------------------------------------------------
LMB_D void phase_t_sel_d(const Geom &g, int wraps, Cd2 *v) {
  const double *ph = wraps > 0 ? g.ph_fwd[3] : g.ph_bwd[3];
  const Cd2 f(d2(wraps ? ph[0] : 1.0), d2(wraps ? ph[1] : 0.0));
#pragma unroll
  for (int i = 0; i < 3; i++) v[i] = v[i] * f;
}

template <int MU, int D>
LMB_D void stag_hop_adj_d(const Geom &g, int s0, const int *c0, const int *c1, const Field<PREC_DOUBLE, 3> &in,
                          const Gauge<PREC_DOUBLE> &U, double2 eta, Cd2 *acc) {
  Cd2 v[3], u[9], o[3];
  int w0, w1;
  if constexpr (MU == 0) {
    const int n0 = shift_site_sel(g, s0, c0, 0, D, &w0), n1 = shift_site_sel(g, s0 + 1, c1, 0, D, &w1);
    load2(in, n0, n1, v);
  } else {
    const int n = (D == 1) ? fwd_site(g, s0, c0, MU, 1, &w0) : shift_site_sel(g, s0, c0, MU, D, &w0);
    load_adj(in, n, v);
    if constexpr (MU == 3) phase_t_sel_d(g, w0, v);
  }
  load_adj(U, MU, s0, u);
  su3_mul_vec(u, v, o);
#pragma unroll
  for (int i = 0; i < 3; i++) acc[i] = Cd2(fmad2(eta, o[i].re, acc[i].re), fmad2(eta, o[i].im, acc[i].im));
  if constexpr (MU == 0) {
    const int n0 = shift_site_sel(g, s0, c0, 0, -D, &w0), n1 = shift_site_sel(g, s0 + 1, c1, 0, -D, &w1);
    load2(in, n0, n1, v);
    load2(U, 0, n0, n1, u);
  } else {
    const int n = (D == 1) ? bwd_site(g, s0, c0, MU, 1, &w0) : shift_site_sel(g, s0, c0, MU, -D, &w0);
    if (D == 1 && w0) w0 = -1;
    load_adj(in, n, v);
    if constexpr (MU == 3) phase_t_sel_d(g, w0, v);
    load_adj(U, MU, n, u);
  }
  su3_adj_mul_vec(u, v, o);
#pragma unroll
  for (int i = 0; i < 3; i++) acc[i] = Cd2(fmad2(-eta, o[i].re, acc[i].re), fmad2(-eta, o[i].im, acc[i].im));
}

template <bool NAIK>
LMB_D void stag_adj_sites_d(const Geom &g, int s0, const Field<PREC_DOUBLE, 3> &in, const Gauge<PREC_DOUBLE> &X,
                            const Gauge<PREC_DOUBLE> &Lk, double mass, double fc, double lc, Cd2 *out) {
  int c0[4], c1[4];
  site_coords(g, s0, c0);
  c1[0] = c0[0] + 1;
  c1[1] = c0[1];
  c1[2] = c0[2];
  c1[3] = c0[3];
  const int p0 = c0[0] + g.eta_off[0], p1 = p0 + c0[1] + g.eta_off[1], p2 = p1 + c0[2] + g.eta_off[2];
  const double e1 = (p0 & 1) ? -1.0 : 1.0, e2 = (p1 & 1) ? -1.0 : 1.0, e3 = (p2 & 1) ? -1.0 : 1.0;
  const double2 eta0 = d2(1.0), eta1 = d2(e1, -e1), eta2 = d2(e2, -e2), eta3 = d2(e3, -e3);
  Cd2 fat[3] = {cd2_zero(), cd2_zero(), cd2_zero()};
  stag_hop_adj_d<0, 1>(g, s0, c0, c1, in, X, eta0, fat);
  stag_hop_adj_d<1, 1>(g, s0, c0, c1, in, X, eta1, fat);
  stag_hop_adj_d<2, 1>(g, s0, c0, c1, in, X, eta2, fat);
  stag_hop_adj_d<3, 1>(g, s0, c0, c1, in, X, eta3, fat);
  const double2 m2 = d2(mass), fc2 = d2(fc);
  Cd2 psi[3];
  if constexpr (NAIK) {
    // fat * fc and the Naik sum share one accumulator; psi comes last
#pragma unroll
    for (int k = 0; k < 3; k++) fat[k] = Cd2(fc2 * fat[k].re, fc2 * fat[k].im);
    const double2 lc2 = d2(lc);
    const double2 el0 = lc2 * eta0, el1 = lc2 * eta1, el2 = lc2 * eta2, el3 = lc2 * eta3;
    stag_hop_adj_d<0, 3>(g, s0, c0, c1, in, Lk, el0, fat);
    stag_hop_adj_d<1, 3>(g, s0, c0, c1, in, Lk, el1, fat);
    stag_hop_adj_d<2, 3>(g, s0, c0, c1, in, Lk, el2, fat);
    stag_hop_adj_d<3, 3>(g, s0, c0, c1, in, Lk, el3, fat);
    load_adj(in, s0, psi);
#pragma unroll
    for (int k = 0; k < 3; k++) out[k] = Cd2(fmad2(m2, psi[k].re, fat[k].re), fmad2(m2, psi[k].im, fat[k].im));
  } else {
    load_adj(in, s0, psi);
#pragma unroll
    for (int k = 0; k < 3; k++)
      out[k] = Cd2(fmad2(fc2, fat[k].re, m2 * psi[k].re), fmad2(fc2, fat[k].im, m2 * psi[k].im));
  }
}

// resident 128-thread blocks per SM requested for the FP64 pair stencil:
// three (168 registers, a few spilled words) for the plain apply and K2,
// two (255 registers, no spill) for the persistent K1 (48^3x96 HISQ CG:
// K1 2.79 against 3.27 ms at three; K2 3.39 against 3.55 ms at two)
template <class Epi> struct StagD2MinBlocks { static constexpr int value = 3; };
template <> struct StagD2MinBlocks<EpiStoreNorm<PREC_DOUBLE, 3>> { static constexpr int value = 2; };
// gridDim.x blocks walk the ntiles tiles of kStagThreads pairs (one tile
// per block when gridDim.x = ntiles; the resident blocks for the persistent
// K1), the reduction carried in registers and done once per block
template <bool NAIK, class Epi>
__global__ void __launch_bounds__(kStagThreads, StagD2MinBlocks<Epi>::value)
    staggered_adj_d_kernel(const Geom g, const Field<PREC_DOUBLE, 3> in, const Gauge<PREC_DOUBLE> X,
                           const Gauge<PREC_DOUBLE> Lk, const double mass, const double fc, const double lc, Epi epi,
                           int ntiles, const SiteRange rg) {
  if (epi.skip()) return;
  double red[1] = {0.0};
  const int npairs = (rg.hi - rg.lo) >> 1;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int i = tile * kStagThreads + threadIdx.x;
    const bool active = i < npairs;
    const int s0 = rg.lo + 2 * i;
    Cd2 out[3];
    if (active) stag_adj_sites_d<NAIK>(g, s0, in, X, Lk, mass, fc, lc, out);
    Cx<double> o0[3], o1[3];
#pragma unroll
    for (int k = 0; k < 3; k++) {
      o0[k] = Cx<double>(out[k].re.x, out[k].im.x);
      o1[k] = Cx<double>(out[k].re.y, out[k].im.y);
    }
    epi.site_acc(s0, active, o0, red);
    epi.site_acc(s0 + 1, active, o1, red);
  }
  epi.finish(red);
}

}  // namespace lmb
