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
// Fields: V4 * L5 sites, site = s + L5 * x4 (the fifth coordinate fastest),
// the planes of Field<P, 12>.  The L5 sites of one 4D point are adjacent, so
// the loads of psi at s - 1 and s + 1 hit the lines the neighbouring lanes
// fetch, and the L5 lanes of one 4D point read the same link (one
// transaction).
//
// One pass per application (L5 <= kDslashThreads):
//   D5:   out = a (psi - F psi + (4+M) Y - 1/2 H Y) with Y = B psi + C F psi
//         rebuilt at each of the 8 neighbours from psi at s, s - 1, s + 1;
//   D5^+: Z = a D_W^+ psi per site (A is constant on a slice, so
//         D_W^+ (A psi) = a D_W^+ psi), exchanged between the L5 sites of a
//         4D point through shared memory; out = a psi - F^+(A psi) + b Z +
//         F^+(C Z).  Blocks hold floor(kDslashThreads / L5) whole 4D points.
// Longer fifth dimensions take two passes (a local pass and a stencil pass).
#pragma once
#include "lmb_pack.cuh"
#include "lmb_solver.cuh"

namespace lmb {

struct DWParams {
  int L5;
  double mass, M;
  const double *a, *b, *c;  // L5 each, device memory
};

LMB_D int64_t dw_idx(int64_t x4, int s, int L5) { return (int64_t)s + (int64_t)L5 * x4; }

// fifth-coordinate neighbours of slice s: F (adj = 0) or F^+ (adj = 1) takes
// spins 1, 2 (components 0..5) from slice lo with factor flo and spins 3, 4
// (components 6..11) from slice hi with factor fhi
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

// components [K0, K1) of site i (the planes that hold them)
template <int K0, int K1, typename R>
LMB_D void load_part(const Field<PREC_DOUBLE, 12> &f, int64_t i, Cx<R> *v) {
#pragma unroll
  for (int k = K0; k < K1; k++) {
    const double2 t = __ldg(f.data + k * f.V + i);
    v[k] = Cx<R>((R)t.x, (R)t.y);
  }
}
template <int K0, int K1, typename R>
LMB_D void load_part(const Field<PREC_SINGLE, 12> &f, int64_t i, Cx<R> *v) {
  static_assert(K0 % 2 == 0 && K1 % 2 == 0, "float4 planes hold component pairs");
#pragma unroll
  for (int p = K0 / 2; p < K1 / 2; p++) {
    const float4 t = __ldg(f.data + p * f.V + i);
    v[2 * p] = Cx<R>((R)t.x, (R)t.y);
    v[2 * p + 1] = Cx<R>((R)t.z, (R)t.w);
  }
}
template <int K0, int K1, typename R>
LMB_D void load_part(const Field<PREC_HALF, 12> &f, int64_t i, Cx<R> *v) {
  const Dec16 d = dec16_of_base(__ldg(f.norm + i));
#pragma unroll
  for (int p = K0 / 4; p < (K1 + 3) / 4; p++) {
    const int4 t = __ldg(f.data + p * f.V + i);
    const int w[4] = {t.x, t.y, t.z, t.w};
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const int k = 4 * p + j;
      if (k >= K0 && k < K1) {
        const float2 q = dec_pair(w[j], d);
        v[k] = Cx<R>((R)q.x, (R)q.y);
      }
    }
  }
}

// (F psi)(x4, s) or (F^+ psi), each source slice weighted by w[slice]
// (w = nullptr: 1)
template <class SF, typename R>
LMB_D void dw_F_site(const SF &f, int64_t x4, int s, const DWParams &d, int adj, const double *w, Cx<R> *out) {
  int lo, hi;
  double flo, fhi;
  dw_F_sources(d, s, adj, lo, hi, flo, fhi);
  if (w) {
    flo *= w[lo];
    fhi *= w[hi];
  }
  load_part<0, 6>(f, dw_idx(x4, lo, d.L5), out);
  load_part<6, 12>(f, dw_idx(x4, hi, d.L5), out);
#pragma unroll
  for (int k = 0; k < 6; k++) out[k] = (R)flo * out[k];
#pragma unroll
  for (int k = 6; k < 12; k++) out[k] = (R)fhi * out[k];
}

// the spins-3,4 part of the (1 -+ gamma_MU) projection (the spins-1,2 part
// of every projection is the identity: h = x_{0..5} + lower(x_{6..11}))
template <int PM, int MU, typename R>
LMB_D void project_lower(const Cx<R> *p, Cx<R> *h) {
#pragma unroll
  for (int c = 0; c < 3; c++) {
    const Cx<R> s3 = p[c + 6], s4 = p[c + 9];
    if (MU == 0) {
      h[c] = PM > 0 ? -mul_i(s4) : mul_i(s4);
      h[c + 3] = PM > 0 ? -mul_i(s3) : mul_i(s3);
    } else if (MU == 1) {
      h[c] = PM > 0 ? -s4 : s4;
      h[c + 3] = PM > 0 ? s3 : -s3;
    } else if (MU == 2) {
      h[c] = PM > 0 ? -mul_i(s3) : mul_i(s3);
      h[c + 3] = PM > 0 ? mul_i(s4) : -mul_i(s4);
    } else {
      h[c] = PM > 0 ? -s3 : s3;
      h[c + 3] = PM > 0 ? -s4 : s4;
    }
  }
}

// the projected half spinor of Y(y4, s) built term by term (only six
// components live): b P psi(s) + cl psi_{0..5}(lo) + ch lower(psi_{6..11}(hi))
template <int PM, int MU, typename R, class SF>
LMB_D void dw_Y_proj(const SF &psi, int64_t y4, int s, int lo, int hi, int L5, R b, R cl, R ch, Cx<R> *h) {
  Cx<R> q[12], t[6];
  psi.load(dw_idx(y4, s, L5), q);
  project<PM, MU>(q, h);
#pragma unroll
  for (int k = 0; k < 6; k++) h[k] = b * h[k];
  load_part<0, 6>(psi, dw_idx(y4, lo, L5), q);
#pragma unroll
  for (int k = 0; k < 6; k++) h[k] = h[k] + cl * q[k];
  load_part<6, 12>(psi, dw_idx(y4, hi, L5), q);
  project_lower<PM, MU>(q, t);
#pragma unroll
  for (int k = 0; k < 6; k++) h[k] = h[k] + ch * t[k];
}

// Wilson hop of direction MU of slice s.  FUSED: the hopped field is Y
// rebuilt from psi (dw_Y_proj); else the field `in` itself.
template <typename R, int DAG, int MU, bool FUSED, class SF, class G>
LMB_D void dw_hop(const Geom &g, int x4, const int *c, int s, int lo, int hi, int L5, R b, R cl, R ch,
                  const SF &in, const G &U, Cx<R> *acc) {
  constexpr int FPM = DAG ? +1 : -1;
  constexpr int BPM = -FPM;
  Cx<R> p[12], h[6], uh[6], u[9];
  int wrap;
  {
    const int sp = fwd_site(g, x4, c, MU, 1, &wrap);
    if constexpr (FUSED) {
      dw_Y_proj<FPM, MU>(in, sp, s, lo, hi, L5, b, cl, ch, h);
    } else {
      in.load(dw_idx(sp, s, L5), p);
      project<FPM, MU>(p, h);
    }
    if (wrap && ((g.phase_mask >> MU) & 1)) scale_phase(h, 6, g.ph_fwd[MU]);
    U.load(MU, x4, u);
    su3_mul_half(u, h, uh);
    reconstruct<FPM, MU>(acc, uh);
  }
  {
    const int sm = bwd_site(g, x4, c, MU, 1, &wrap);
    if constexpr (FUSED) {
      dw_Y_proj<BPM, MU>(in, sm, s, lo, hi, L5, b, cl, ch, h);
    } else {
      in.load(dw_idx(sm, s, L5), p);
      project<BPM, MU>(p, h);
    }
    if (wrap && ((g.phase_mask >> MU) & 1)) scale_phase(h, 6, g.ph_bwd[MU]);
    U.load(MU, sm, u);
    su3_adj_mul_half(u, h, uh);
    reconstruct<BPM, MU>(acc, uh);
  }
}

template <typename R, int DAG, bool FUSED, class SF, class G>
LMB_D void dw_hops(const Geom &g, int x4, int s, int lo, int hi, int L5, R b, R cl, R ch, const SF &in,
                   const G &U, Cx<R> *acc) {
  int c[4];
  site_coords(g, x4, c);
#pragma unroll
  for (int k = 0; k < 12; k++) acc[k] = Cx<R>(0, 0);
  dw_hop<R, DAG, 0, FUSED>(g, x4, c, s, lo, hi, L5, b, cl, ch, in, U, acc);
  dw_hop<R, DAG, 1, FUSED>(g, x4, c, s, lo, hi, L5, b, cl, ch, in, U, acc);
  dw_hop<R, DAG, 2, FUSED>(g, x4, c, s, lo, hi, L5, b, cl, ch, in, U, acc);
  dw_hop<R, DAG, 3, FUSED>(g, x4, c, s, lo, hi, L5, b, cl, ch, in, U, acc);
}

// ---------------------------------------------------------------------------
// one-pass kernels
// ---------------------------------------------------------------------------
// resident blocks per SM the one-pass kernels are compiled for, which caps
// their registers (128 threads x B blocks: 65536 / (128 B) registers)
#ifndef LMB_DW_MINB
#define LMB_DW_MINB 4
#endif
#ifndef LMB_DW_MINB_D
#define LMB_DW_MINB_D 3
#endif
template <typename R> struct DWMinBlocks { static constexpr int value = LMB_DW_MINB; };
template <> struct DWMinBlocks<double> { static constexpr int value = LMB_DW_MINB_D; };

// D5: one thread per 5D site, site = blockIdx.x * kDslashThreads + threadIdx.x
template <typename R, class SF, class G, class Epi>
__global__ void __launch_bounds__(kDslashThreads, DWMinBlocks<R>::value)
    dw_forward_kernel(const Geom g, const SF psi, const G U, const DWParams d, Epi epi) {
  if (epi.skip()) return;
  const int L5 = d.L5;
  const int64_t i = (int64_t)blockIdx.x * kDslashThreads + threadIdx.x;
  const bool active = i < g.V * L5;
  Cx<R> out[12];
  if (active) {
    const int x4 = (int)(i / L5);
    const int s = (int)(i - (int64_t)x4 * L5);
    int lo, hi;
    double flo, fhi;
    dw_F_sources(d, s, 0, lo, hi, flo, fhi);
    const R b = (R)d.b[s], c = (R)d.c[s];
    const R cl = c * (R)flo, ch = c * (R)fhi;
    Cx<R> acc[12];
    dw_hops<R, 0, true>(g, x4, s, lo, hi, L5, b, cl, ch, psi, U, acc);
    Cx<R> p[12], f[12];
    psi.load(i, p);
    load_part<0, 6>(psi, dw_idx(x4, lo, L5), f);
    load_part<6, 12>(psi, dw_idx(x4, hi, L5), f);
    const R a = (R)d.a[s], diag = (R)(4.0 + d.M);
#pragma unroll
    for (int k = 0; k < 12; k++) {
      const Cx<R> fk = (k < 6 ? (R)flo : (R)fhi) * f[k];
      const Cx<R> y = b * p[k] + c * fk;
      out[k] = a * (diag * y - (R)0.5 * acc[k] + p[k] - fk);
    }
  }
  epi((int)(active ? i : 0), active, out);
}

// D5^+: blocks of kDslashThreads threads holding `npts` whole 4D points
// (npts * L5 <= kDslashThreads; the remaining threads only take part in
// the barriers and the epilogue's reduction)
template <typename R, class SF, class G, class Epi>
__global__ void __launch_bounds__(kDslashThreads, DWMinBlocks<R>::value)
    dw_adjoint_kernel(const Geom g, const SF psi, const G U, const DWParams d, int npts, Epi epi) {
  __shared__ R zs[24 * kDslashThreads];
  if (epi.skip()) return;
  const int L5 = d.L5;
  const int t = threadIdx.x;
  const int gx = t / L5;
  const int s = t - gx * L5;
  const int64_t x4 = (int64_t)blockIdx.x * npts + gx;
  const bool active = gx < npts && x4 < g.V;
  const int64_t i = x4 * L5 + s;
  if (active) {
    Cx<R> acc[12], p[12];
    dw_hops<R, 1, false>(g, (int)x4, s, 0, 0, L5, (R)0, (R)0, (R)0, psi, U, acc);
    psi.load(i, p);
    const R a = (R)d.a[s], diag = (R)(4.0 + d.M);
#pragma unroll
    for (int k = 0; k < 12; k++) {
      const Cx<R> z = a * (diag * p[k] - (R)0.5 * acc[k]);
      zs[(2 * k) * kDslashThreads + t] = z.re;
      zs[(2 * k + 1) * kDslashThreads + t] = z.im;
    }
  }
  __syncthreads();
  Cx<R> out[12];
  if (active) {
    int lo, hi;
    double flo, fhi;
    dw_F_sources(d, s, 1, lo, hi, flo, fhi);
    const int tlo = gx * L5 + lo, thi = gx * L5 + hi;
    const R zl = (R)(flo * d.c[lo]), zh = (R)(fhi * d.c[hi]);
    const R pl = (R)(flo * d.a[lo]), ph = (R)(fhi * d.a[hi]);
    const R a = (R)d.a[s], b = (R)d.b[s];
    Cx<R> p[12], f[12];
    psi.load(i, p);
    load_part<0, 6>(psi, dw_idx(x4, lo, L5), f);
    load_part<6, 12>(psi, dw_idx(x4, hi, L5), f);
#pragma unroll
    for (int k = 0; k < 12; k++) {
      const int tt = k < 6 ? tlo : thi;
      const Cx<R> zn(zs[(2 * k) * kDslashThreads + tt], zs[(2 * k + 1) * kDslashThreads + tt]);
      const Cx<R> z(zs[(2 * k) * kDslashThreads + t], zs[(2 * k + 1) * kDslashThreads + t]);
      out[k] = a * p[k] - (k < 6 ? pl : ph) * f[k] + b * z + (k < 6 ? zl : zh) * zn;
    }
  }
  epi((int)(active ? i : 0), active, out);
}

// ---------------------------------------------------------------------------
// two-pass kernels (any L5)
// ---------------------------------------------------------------------------
// D5 pass 1: Y = b psi + c F psi
template <int P, class Epi>
__global__ void __launch_bounds__(kDslashThreads)
    dw_fifth_kernel(Field<P, 12> Y, const Field<P, 12> psi, const int64_t V4, const DWParams d, Epi epi) {
  typedef typename Real<P>::type R;
  if (epi.skip()) return;
  const int64_t i = (int64_t)blockIdx.x * kDslashThreads + threadIdx.x;
  if (i >= V4 * d.L5) return;
  const int64_t x4 = i / d.L5;
  const int s = (int)(i - x4 * d.L5);
  Cx<R> p[12], f[12];
  psi.load(i, p);
  dw_F_site(psi, x4, s, d, 0, nullptr, f);
  const R b = (R)d.b[s], c = (R)d.c[s];
#pragma unroll
  for (int k = 0; k < 12; k++) p[k] = b * p[k] + c * f[k];
  Y.store(i, p);
}

// stencil pass: out = a_s [(4 + M) Y - 1/2 H Y] (+ a_s (psi - F psi) if LOCAL)
template <typename R, int DAG, int LOCAL, class SF, class G, class Epi>
__global__ void __launch_bounds__(kDslashThreads)
    dw_stencil_kernel(const Geom g, const SF Y, const SF psi, const G U, const DWParams d, Epi epi) {
  if (epi.skip()) return;
  const int L5 = d.L5;
  const int64_t i = (int64_t)blockIdx.x * kDslashThreads + threadIdx.x;
  const bool active = i < g.V * L5;
  Cx<R> out[12];
  if (active) {
    const int x4 = (int)(i / L5);
    const int s = (int)(i - (int64_t)x4 * L5);
    Cx<R> acc[12];
    dw_hops<R, DAG, false>(g, x4, s, 0, 0, L5, (R)0, (R)0, (R)0, Y, U, acc);
    Cx<R> y[12];
    Y.load(i, y);
    const R a = (R)d.a[s], diag = (R)(4.0 + d.M);
#pragma unroll
    for (int k = 0; k < 12; k++) out[k] = a * (diag * y[k] - (R)0.5 * acc[k]);
    if constexpr (LOCAL) {
      Cx<R> p[12], f[12];
      psi.load(i, p);
      dw_F_site(psi, (int64_t)x4, s, d, 0, nullptr, f);
#pragma unroll
      for (int k = 0; k < 12; k++) out[k] = out[k] + a * (p[k] - f[k]);
    }
  }
  epi((int)(active ? i : 0), active, out);
}

// D5^+ pass 2: out = a psi - F^+(A psi) + b Z + F^+(C Z)
template <typename R, class SF, class Epi>
__global__ void __launch_bounds__(kDslashThreads)
    dw_adjoint_local_kernel(const SF psi, const SF Z, const int64_t V4, const DWParams d, Epi epi) {
  if (epi.skip()) return;
  const int64_t i = (int64_t)blockIdx.x * kDslashThreads + threadIdx.x;
  const bool active = i < V4 * d.L5;
  Cx<R> out[12];
  if (active) {
    const int64_t x4 = i / d.L5;
    const int s = (int)(i - x4 * d.L5);
    Cx<R> p[12], z[12], fa[12], fc[12];
    psi.load(i, p);
    Z.load(i, z);
    dw_F_site(psi, x4, s, d, 1, d.a, fa);
    dw_F_site(Z, x4, s, d, 1, d.c, fc);
    const R a = (R)d.a[s], b = (R)d.b[s];
#pragma unroll
    for (int k = 0; k < 12; k++) out[k] = a * p[k] - fa[k] + b * z[k] + fc[k];
  }
  epi((int)(active ? i : 0), active, out);
}

// ---------------------------------------------------------------------------
// pack / unpack of 5D padded fields (NC1, NC2, X+2nw, .., T+2nw, L5+2nw)
// ---------------------------------------------------------------------------
template <typename TIN, int PS, int NC>
__global__ void __launch_bounds__(256)
    pack_field5_kernel(Field<PS, NC> dst, const TIN *src, const Geom g, const Padded pd, int L5) {
  const int64_t i = (int64_t)blockIdx.x * 256 + threadIdx.x;
  if (i >= g.V * L5) return;
  const int x4 = (int)(i / L5);
  const int s = (int)(i - (int64_t)x4 * L5);
  int c[4];
  site_coords(g, x4, c);
  const int64_t p4 = (int64_t)pd.P[0] * pd.P[1] * pd.P[2] * pd.P[3];
  const TIN *q = src + (padded_site(pd, c) + (int64_t)(s + pd.nw) * p4) * NC;
  typedef typename Real<PS>::type R;
  Cx<R> v[NC];
#pragma unroll
  for (int k = 0; k < NC; k++) v[k] = Cx<R>((R)q[k].x, (R)q[k].y);
  dst.store(i, v);
}
template <typename TOUT, int PS, int NC>
__global__ void __launch_bounds__(256)
    unpack_field5_kernel(TOUT *dst, const Field<PS, NC> src, const Geom g, const Padded pd, int L5) {
  const int64_t i = (int64_t)blockIdx.x * 256 + threadIdx.x;
  if (i >= g.V * L5) return;
  const int x4 = (int)(i / L5);
  const int s = (int)(i - (int64_t)x4 * L5);
  int c[4];
  site_coords(g, x4, c);
  const int64_t p4 = (int64_t)pd.P[0] * pd.P[1] * pd.P[2] * pd.P[3];
  TOUT *q = dst + (padded_site(pd, c) + (int64_t)(s + pd.nw) * p4) * NC;
  typedef typename Real<PS>::type R;
  Cx<R> v[NC];
  src.load(i, v);
#pragma unroll
  for (int k = 0; k < NC; k++) {
    q[k].x = v[k].re;
    q[k].y = v[k].im;
  }
}

}  // namespace lmb
