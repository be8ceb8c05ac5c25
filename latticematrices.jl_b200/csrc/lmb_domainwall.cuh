// lmb_domainwall.cuh -- generalised / Mobius domain-wall operator
// (DiracOperators_5D.jl:48-115, 226-268, 731-857):
//   D5 psi   = A [psi - F psi + D_W (B psi + C F psi)]
//   D5^+ psi = q - F^+ q + B D_W^+ q + F^+ (C D_W^+ q),   q = A psi
// A, B, C: coefficients a_s, b_s, c_s of the fifth coordinate; D_W the 4D
// Wilson kernel (4 + M) - 1/2 sum_mu [U(1 - g)psi(x+mu) + U^+(1 + g)psi(x-mu)]
// on every s-slice with the shared 4D links; F takes spins 1, 2 from s - 1
// and spins 3, 4 from s + 1, with -mass across the walls (F^+ the reverse).
// Mobius(b, c) is a = 1, b_s = (b + c)/2, c_s = (b - c)/2.
//
// Fields: V4 * L5 sites, site = x4 + V4 * s (slices contiguous), the planes
// of Field<P, 12>.  Two passes per application:
//   D5:   Y = B psi + C F psi (local);  out = a (psi - F psi + (4+M) Y - 1/2 H Y)
//   D5^+: Z = a D_W^+ psi (stencil);    out = a psi - F^+(A psi) + b Z + F^+(C Z)
// (A is constant on a slice, so D_W^+ (A psi) = a D_W^+ psi.)
#pragma once
#include "lmb_solver.cuh"

namespace lmb {

struct DWParams {
  int L5;
  double mass, M;
  const double *a, *b, *c;  // L5 each, device memory
};

// fifth-coordinate neighbours of slice s: F (adj = 0) or F^+ (adj = 1) takes
// the lower spins (components 0..5) from slice lo with factor flo and the
// upper spins (6..11) from slice hi with factor fhi
LMB_D void dw_F_sources(const DWParams &d, int s, int adj, int &lo, int &hi, double &flo, double &fhi) {
  const int L5 = d.L5;
  const int sm = s == 0 ? L5 - 1 : s - 1, sp = s == L5 - 1 ? 0 : s + 1;
  if (!adj) {
    lo = sm;
    hi = sp;
    flo = s == 0 ? -d.mass : 1.0;
    fhi = s == L5 - 1 ? -d.mass : 1.0;
  } else {
    lo = sp;
    hi = sm;
    flo = s == L5 - 1 ? -d.mass : 1.0;
    fhi = s == 0 ? -d.mass : 1.0;
  }
}

// out = (F psi)(x4, s) or (F^+ psi), each source slice weighted by w[slice]
// (w = nullptr: 1)
template <class SF, typename R>
LMB_D void dw_F_site(const SF &f, int64_t s4, int s, int64_t V4, const DWParams &d, int adj, const double *w,
                     Cx<R> *out) {
  int lo, hi;
  double flo, fhi;
  dw_F_sources(d, s, adj, lo, hi, flo, fhi);
  if (w) {
    flo *= w[lo];
    fhi *= w[hi];
  }
  Cx<R> t[12];
  f.load(s4 + (int64_t)lo * V4, t);
#pragma unroll
  for (int k = 0; k < 6; k++) out[k] = (R)flo * t[k];
  f.load(s4 + (int64_t)hi * V4, t);
#pragma unroll
  for (int k = 6; k < 12; k++) out[k] = (R)fhi * t[k];
}

// Wilson hop of direction MU on slice `off` (field index = 4D index + off,
// links indexed by the 4D site)
template <typename R, int DAG, int MU, class SF, class G>
LMB_D void dw_hop(const Geom &g, int s4, const int *c, int64_t off, const SF &in, const G &U, Cx<R> *acc) {
  constexpr int FPM = DAG ? +1 : -1;
  constexpr int BPM = -FPM;
  Cx<R> p[12], h[6], uh[6], u[9];
  int wrap;
  {
    const int sp = fwd_site(g, s4, c, MU, 1, &wrap);
    in.load(sp + off, p);
    project<FPM, MU>(p, h);
    if (wrap && ((g.phase_mask >> MU) & 1)) scale_phase(h, 6, g.ph_fwd[MU]);
    U.load(MU, s4, u);
    su3_mul_half(u, h, uh);
    reconstruct<FPM, MU>(acc, uh);
  }
  {
    const int sm = bwd_site(g, s4, c, MU, 1, &wrap);
    in.load(sm + off, p);
    project<BPM, MU>(p, h);
    if (wrap && ((g.phase_mask >> MU) & 1)) scale_phase(h, 6, g.ph_bwd[MU]);
    U.load(MU, sm, u);
    su3_adj_mul_half(u, h, uh);
    reconstruct<BPM, MU>(acc, uh);
  }
}

// a store that skips with another epilogue (a paused CG skips every pass)
template <int PS, class Follow>
struct EpiStoreFollow {
  Field<PS, 12> out;
  Follow follow;
  LMB_D bool skip() const { return follow.skip(); }
  template <typename R> LMB_D void operator()(int s, bool active, const Cx<R> *v) const {
    if (active) out.store(s, v);
  }
};

// D5 pass 1: Y = b psi + c F psi
template <int P, class Epi>
__global__ void __launch_bounds__(kDslashThreads)
    dw_fifth_kernel(Field<P, 12> Y, const Field<P, 12> psi, const int64_t V4, const DWParams d, Epi epi) {
  typedef typename Real<P>::type R;
  if (epi.skip()) return;
  const int64_t s = (int64_t)blockIdx.x * kDslashThreads + threadIdx.x;
  if (s >= V4 * d.L5) return;
  const int s5 = (int)(s / V4);
  const int64_t s4 = s - (int64_t)s5 * V4;
  Cx<R> p[12], f[12];
  psi.load(s, p);
  dw_F_site(psi, s4, s5, V4, d, 0, nullptr, f);
  const R b = (R)d.b[s5], c = (R)d.c[s5];
#pragma unroll
  for (int k = 0; k < 12; k++) p[k] = b * p[k] + c * f[k];
  Y.store(s, p);
}

// stencil pass: out = a_s [(4 + M) Y - 1/2 H Y] (+ a_s (psi - F psi) if LOCAL)
template <typename R, int DAG, int LOCAL, class SF, class G, class Epi>
__global__ void __launch_bounds__(kDslashThreads)
    dw_stencil_kernel(const Geom g, const SF Y, const SF psi, const G U, const DWParams d, Epi epi) {
  if (epi.skip()) return;
  const int64_t V4 = g.V;
  const int64_t s = (int64_t)blockIdx.x * kDslashThreads + threadIdx.x;
  const bool active = s < V4 * d.L5;
  Cx<R> out[12];
  if (active) {
    const int s5 = (int)(s / V4);
    const int s4 = (int)(s - (int64_t)s5 * V4);
    const int64_t off = (int64_t)s5 * V4;
    int c[4];
    site_coords(g, s4, c);
    Cx<R> acc[12];
#pragma unroll
    for (int k = 0; k < 12; k++) acc[k] = Cx<R>(0, 0);
    dw_hop<R, DAG, 0>(g, s4, c, off, Y, U, acc);
    dw_hop<R, DAG, 1>(g, s4, c, off, Y, U, acc);
    dw_hop<R, DAG, 2>(g, s4, c, off, Y, U, acc);
    dw_hop<R, DAG, 3>(g, s4, c, off, Y, U, acc);
    Cx<R> y[12];
    Y.load(s, y);
    const R a = (R)d.a[s5], diag = (R)(4.0 + d.M);
#pragma unroll
    for (int k = 0; k < 12; k++) out[k] = a * (diag * y[k] - (R)0.5 * acc[k]);
    if constexpr (LOCAL) {
      Cx<R> p[12], f[12];
      psi.load(s, p);
      dw_F_site(psi, (int64_t)s4, s5, V4, d, 0, nullptr, f);
#pragma unroll
      for (int k = 0; k < 12; k++) out[k] = out[k] + a * (p[k] - f[k]);
    }
  }
  epi((int)s, active, out);
}

// D5^+ pass 2: out = a psi - F^+(A psi) + b Z + F^+(C Z)
template <typename R, class SF, class Epi>
__global__ void __launch_bounds__(kDslashThreads)
    dw_adjoint_local_kernel(const SF psi, const SF Z, const int64_t V4, const DWParams d, Epi epi) {
  if (epi.skip()) return;
  const int64_t s = (int64_t)blockIdx.x * kDslashThreads + threadIdx.x;
  const bool active = s < V4 * d.L5;
  Cx<R> out[12];
  if (active) {
    const int s5 = (int)(s / V4);
    const int64_t s4 = s - (int64_t)s5 * V4;
    Cx<R> p[12], z[12], fa[12], fc[12];
    psi.load(s, p);
    Z.load(s, z);
    dw_F_site(psi, s4, s5, V4, d, 1, d.a, fa);
    dw_F_site(Z, s4, s5, V4, d, 1, d.c, fc);
    const R a = (R)d.a[s5], b = (R)d.b[s5];
#pragma unroll
    for (int k = 0; k < 12; k++) out[k] = a * p[k] - fa[k] + b * z[k] + fc[k];
  }
  epi((int)s, active, out);
}

// pack / unpack of 5D padded fields (NC1, NC2, X+2nw, .., T+2nw, L5+2nw)
template <typename TIN, int PS, int NC>
__global__ void __launch_bounds__(256)
    pack_field5_kernel(Field<PS, NC> dst, const TIN *src, const Geom g, const Padded pd, int L5) {
  const int64_t s = (int64_t)blockIdx.x * 256 + threadIdx.x;
  if (s >= g.V * L5) return;
  const int s5 = (int)(s / g.V);
  const int s4 = (int)(s - (int64_t)s5 * g.V);
  int c[4];
  site_coords(g, s4, c);
  const int64_t p4 = (int64_t)pd.P[0] * pd.P[1] * pd.P[2] * pd.P[3];
  const TIN *q = src + (padded_site(pd, c) + (int64_t)(s5 + pd.nw) * p4) * NC;
  typedef typename Real<PS>::type R;
  Cx<R> v[NC];
#pragma unroll
  for (int k = 0; k < NC; k++) v[k] = Cx<R>((R)q[k].x, (R)q[k].y);
  dst.store(s, v);
}
template <typename TOUT, int PS, int NC>
__global__ void __launch_bounds__(256)
    unpack_field5_kernel(TOUT *dst, const Field<PS, NC> src, const Geom g, const Padded pd, int L5) {
  const int64_t s = (int64_t)blockIdx.x * 256 + threadIdx.x;
  if (s >= g.V * L5) return;
  const int s5 = (int)(s / g.V);
  const int s4 = (int)(s - (int64_t)s5 * g.V);
  int c[4];
  site_coords(g, s4, c);
  const int64_t p4 = (int64_t)pd.P[0] * pd.P[1] * pd.P[2] * pd.P[3];
  TOUT *q = dst + (padded_site(pd, c) + (int64_t)(s5 + pd.nw) * p4) * NC;
  typedef typename Real<PS>::type R;
  Cx<R> v[NC];
  src.load(s, v);
#pragma unroll
  for (int k = 0; k < NC; k++) {
    q[k].x = v[k].re;
    q[k].y = v[k].im;
  }
}

}  // namespace lmb
