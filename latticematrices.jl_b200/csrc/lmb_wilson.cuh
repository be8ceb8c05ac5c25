// lmb_wilson.cuh -- Wilson and Wilson-clover stencil on CUDA cores.
//
// One thread owns one lattice site.  Per direction it loads the neighbouring
// 12-component spinor, projects it to a half spinor with (1 -/+ gamma_mu),
// multiplies the two colour vectors by U_mu(x) (forward) or U_mu(x-mu)^+
// (backward) and reconstructs into the 12-component accumulator.  The
// projector/reconstruction table is the chiral-basis one of the reference
// (WilsonDiracOperator.jl:157-263, Operators.jl:44-66):
//   D psi = A(x) psi(x) - kappa sum_mu [U_mu(x)(1 - g_mu)psi(x+mu)
//                                       + U_mu(x-mu)^+ (1 + g_mu) psi(x-mu)]
// where A = 1 for plain Wilson and A = 1 - kappa cSW sum_{mu<nu} g_mu g_nu F_mu_nu
// for Wilson-clover (WilsonDiracCloverOperator.jl:481-559).  D^+ swaps the
// projector signs and keeps A (A is Hermitian).
//
// The kernel is templated on the storage precision of the input spinor, the
// links and the clover blocks, and on an epilogue that consumes the 12 output
// components (plain store, store + |out|^2, or a fused CG update).
#pragma once
#include "lmb_common.cuh"
#include "lmb_pair.cuh"

namespace lmb {

// threads per block and the minimum resident blocks per SM requested from
// the register allocator (0 = no request); set at compile time
#ifndef LMB_DSLASH_THREADS
#define LMB_DSLASH_THREADS 128
#endif
#ifndef LMB_DSLASH_MINB
#define LMB_DSLASH_MINB 0
#endif
// two-site kernels: 3 resident blocks of 128 threads per SM (<= 168
// registers) measured fastest on B200
#ifndef LMB_PAIR_MINB
#define LMB_PAIR_MINB 3
#endif
constexpr int kDslashThreads = LMB_DSLASH_THREADS;

// half-spin projection rows of (1 + PM g_mu) psi (WilsonDiracOperator.jl:157-175)
template <int PM, int MU, typename R>
LMB_D void project(const Cx<R> *p, Cx<R> *h) {
#pragma unroll
  for (int c = 0; c < 3; c++) {
    const Cx<R> s1 = p[c], s2 = p[c + 3], s3 = p[c + 6], s4 = p[c + 9];
    if (MU == 0) {
      h[c] = PM > 0 ? s1 - mul_i(s4) : s1 + mul_i(s4);
      h[c + 3] = PM > 0 ? s2 - mul_i(s3) : s2 + mul_i(s3);
    } else if (MU == 1) {
      h[c] = PM > 0 ? s1 - s4 : s1 + s4;
      h[c + 3] = PM > 0 ? s2 + s3 : s2 - s3;
    } else if (MU == 2) {
      h[c] = PM > 0 ? s1 - mul_i(s3) : s1 + mul_i(s3);
      h[c + 3] = PM > 0 ? s2 + mul_i(s4) : s2 - mul_i(s4);
    } else {
      h[c] = PM > 0 ? s1 - s3 : s1 + s3;
      h[c + 3] = PM > 0 ? s2 - s4 : s2 + s4;
    }
  }
}

// accumulate the full spinor rebuilt from a half spinor
// (WilsonDiracOperator.jl:225-263)
template <int PM, int MU, typename R>
LMB_D void reconstruct(Cx<R> *acc, const Cx<R> *h) {
#pragma unroll
  for (int c = 0; c < 3; c++) {
    const Cx<R> h0 = h[c], h1 = h[c + 3];
    acc[c] = acc[c] + h0;
    acc[c + 3] = acc[c + 3] + h1;
    if (MU == 0) {
      acc[c + 6] = PM > 0 ? acc[c + 6] + mul_i(h1) : acc[c + 6] - mul_i(h1);
      acc[c + 9] = PM > 0 ? acc[c + 9] + mul_i(h0) : acc[c + 9] - mul_i(h0);
    } else if (MU == 1) {
      acc[c + 6] = PM > 0 ? acc[c + 6] + h1 : acc[c + 6] - h1;
      acc[c + 9] = PM > 0 ? acc[c + 9] - h0 : acc[c + 9] + h0;
    } else if (MU == 2) {
      acc[c + 6] = PM > 0 ? acc[c + 6] + mul_i(h0) : acc[c + 6] - mul_i(h0);
      acc[c + 9] = PM > 0 ? acc[c + 9] - mul_i(h1) : acc[c + 9] + mul_i(h1);
    } else {
      acc[c + 6] = PM > 0 ? acc[c + 6] - h0 : acc[c + 6] + h0;
      acc[c + 9] = PM > 0 ? acc[c + 9] - h1 : acc[c + 9] + h1;
    }
  }
}

// out[r + 3*half] = sum_k U(r,k) h[k + 3*half], U column-major (u[r + 3k])
template <typename R>
LMB_D void su3_mul_half(const Cx<R> *u, const Cx<R> *h, Cx<R> *o) {
#pragma unroll
  for (int half = 0; half < 2; half++)
#pragma unroll
    for (int r = 0; r < 3; r++) {
      Cx<R> v = u[r] * h[3 * half];
      v = cfma(u[r + 3], h[3 * half + 1], v);
      v = cfma(u[r + 6], h[3 * half + 2], v);
      o[r + 3 * half] = v;
    }
}
// U^+ : (U^+)(r,k) = conj(U(k,r)) = conj(u[k + 3r])
template <typename R>
LMB_D void su3_adj_mul_half(const Cx<R> *u, const Cx<R> *h, Cx<R> *o) {
#pragma unroll
  for (int half = 0; half < 2; half++)
#pragma unroll
    for (int r = 0; r < 3; r++) {
      Cx<R> v = conj(u[3 * r]) * h[3 * half];
      v = cfma_conj(u[3 * r + 1], h[3 * half + 1], v);
      v = cfma_conj(u[3 * r + 2], h[3 * half + 2], v);
      o[r + 3 * half] = v;
    }
}

template <typename R>
LMB_D void scale_phase(Cx<R> *h, int n, const double *ph) {
  const Cx<R> f((R)ph[0], (R)ph[1]);
#pragma unroll
  for (int k = 0; k < 6; k++)
    if (k < n) h[k] = h[k] * f;
}

// Boundary-phase code of the stencils.  PH_T: only the t phase may differ
// from 1 (the usual antiperiodic fermions), applied to every t hop as a
// multiplication by a selected factor (1 off the edge): no branch, so the
// compiler is free to issue the next hop's loads early.  PH_ANY: any
// direction, applied only when the hop crossed the edge.
enum PhaseMode { PH_T = 0, PH_ANY = 1 };

LMB_HD int phase_mode_of(int phase_mask) { return (phase_mask & ~8) ? PH_ANY : PH_T; }

template <typename R>
LMB_D void scale_phase_sel(Cx<R> *h, const double *ph, int wrap) {
  const Cx<R> f(wrap ? (R)ph[0] : (R)1, wrap ? (R)ph[1] : (R)0);
#pragma unroll
  for (int k = 0; k < 6; k++) h[k] = h[k] * f;
}

// Hermitian 6x6 (packed: 6 real diagonal, 15 complex lower triangle in row
// order) times a 6-vector
template <typename R>
LMB_D void herm6_mul(const R *a, const Cx<R> *v, Cx<R> *o) {
#pragma unroll
  for (int i = 0; i < 6; i++) o[i] = a[i] * v[i];
  int k = 6;
#pragma unroll
  for (int i = 1; i < 6; i++)
#pragma unroll
    for (int j = 0; j < i; j++) {
      const Cx<R> aij(a[k], a[k + 1]);  // A[i][j]; A[j][i] = conj
      o[i] = cfma(aij, v[j], o[i]);
      o[j] = cfma_conj(aij, v[i], o[j]);
      k += 2;
    }
}

// hopping term of one direction, forward and backward, accumulated into acc
template <typename R, int DAG, int MU, int PHM = PH_ANY, class SF, class G>
LMB_D void hop_dir(const Geom &g, int s, const int *c, const SF &in, const G &U,
                   Cx<R> *acc) {
  // D: forward (1 - g), backward (1 + g);  D^+: swapped
  constexpr int FPM = DAG ? +1 : -1;
  constexpr int BPM = -FPM;
  Cx<R> p[12], h[6], uh[6], u[9];
  int wrap;
  {
    const int sp = fwd_site(g, s, c, MU, 1, &wrap);
    in.load(sp, p);
    project<FPM, MU>(p, h);
    if constexpr (PHM == PH_ANY) {
      if (wrap && ((g.phase_mask >> MU) & 1)) scale_phase(h, 6, g.ph_fwd[MU]);
    } else if constexpr (MU == 3) {
      scale_phase_sel(h, g.ph_fwd[3], wrap);
    }
    U.load(MU, s, u);
    su3_mul_half(u, h, uh);
    reconstruct<FPM, MU>(acc, uh);
  }
  {
    const int sm = bwd_site(g, s, c, MU, 1, &wrap);
    in.load(sm, p);
    project<BPM, MU>(p, h);
    if constexpr (PHM == PH_ANY) {
      if (wrap && ((g.phase_mask >> MU) & 1)) scale_phase(h, 6, g.ph_bwd[MU]);
    } else if constexpr (MU == 3) {
      scale_phase_sel(h, g.ph_bwd[3], wrap);
    }
    U.load(MU, sm, u);
    su3_adj_mul_half(u, h, uh);
    reconstruct<BPM, MU>(acc, uh);
  }
}

// no-op clover for plain Wilson
struct NoClover {
  int64_t V;
};

// D psi at site s (plain Wilson: A = 1)
template <typename R, int DAG, class SF, class G>
LMB_D void wilson_site(const Geom &g, int s, const SF &in, const G &U, R kappa, Cx<R> *out) {
  int c[4];
  site_coords(g, s, c);
  Cx<R> acc[12];
#pragma unroll
  for (int k = 0; k < 12; k++) acc[k] = Cx<R>(0, 0);
  hop_dir<R, DAG, 0>(g, s, c, in, U, acc);
  hop_dir<R, DAG, 1>(g, s, c, in, U, acc);
  hop_dir<R, DAG, 2>(g, s, c, in, U, acc);
  hop_dir<R, DAG, 3>(g, s, c, in, U, acc);
  Cx<R> p[12];
  in.load(s, p);
#pragma unroll
  for (int k = 0; k < 12; k++) out[k] = p[k] - kappa * acc[k];
}

// out = A psi(s) - kappa acc (A = 1 without the clover term)
template <typename R, bool CLOVER, class SF, class CL>
LMB_D void wilson_site_finish(int s, const SF &in, const CL &A, R kappa, const Cx<R> *acc, Cx<R> *out) {
  Cx<R> p[12];
  in.load(s, p);
  if constexpr (CLOVER) {
    R a[36];
    Cx<R> v[6], o[6];
#pragma unroll
    for (int blk = 0; blk < 2; blk++) {
      A.load(blk, s, a);
#pragma unroll
      for (int k = 0; k < 6; k++) v[k] = p[6 * blk + k];
      herm6_mul(a, v, o);
#pragma unroll
      for (int k = 0; k < 6; k++) out[6 * blk + k] = o[k] - kappa * acc[6 * blk + k];
    }
  } else {
#pragma unroll
    for (int k = 0; k < 12; k++) out[k] = p[k] - kappa * acc[k];
  }
}

// D psi (or D^+ psi) at site s with coordinates c (one site per thread)
template <typename R, int DAG, bool CLOVER, int PHM, class SF, class G, class CL>
LMB_D void wilson_site_out(const Geom &g, int s, const int *c, const SF &in, const G &U, const CL &A, R kappa,
                           Cx<R> *out) {
  Cx<R> acc[12];
#pragma unroll
  for (int k = 0; k < 12; k++) acc[k] = Cx<R>(0, 0);
  hop_dir<R, DAG, 0, PHM>(g, s, c, in, U, acc);
  hop_dir<R, DAG, 1, PHM>(g, s, c, in, U, acc);
  hop_dir<R, DAG, 2, PHM>(g, s, c, in, U, acc);
  hop_dir<R, DAG, 3, PHM>(g, s, c, in, U, acc);
  wilson_site_finish<R, CLOVER>(s, in, A, kappa, acc, out);
}

// The Wilson(-clover) kernel.  Epi must provide:
//   bool skip() const                      -- whole grid exits (paused solve)
//   void operator()(s, active, out[12])    -- consume the result
template <typename R, int DAG, bool CLOVER, int PHM, class SF, class G, class CL, class Epi>
__global__ void __launch_bounds__(kDslashThreads, LMB_DSLASH_MINB)
    wilson_dslash_kernel(const Geom g, const SF in, const G U, const CL A,
                         const R kappa, Epi epi, const SiteRange rg) {
  if (epi.skip()) return;
  const int s = rg.lo + blockIdx.x * kDslashThreads + threadIdx.x;
  const bool active = s < rg.hi;
  Cx<R> out[12];
  if (active) {
    int c[4];
    site_coords(g, s, c);
    wilson_site_out<R, DAG, CLOVER, PHM>(g, s, c, in, U, A, kappa, out);
  }
  epi(s, active, out);
}


// ---------------------------------------------------------------------------
// two sites per thread (FP32 arithmetic; see lmb_pair.cuh): lane x = site
// s0 = (x, y, z, t), lane y = site s1 = s0 + V/2 = (x, y, z, t + T/2), T even.
// Along x, y, z both lanes step identically (same wrap); along t each lane
// has its own neighbour and wrap.
// ---------------------------------------------------------------------------
// h *= phase on the lanes whose hop crossed the edge
LMB_D void phase2(Cx2 *h, const double *ph, int w0, int w1) {
  const float pr = (float)ph[0], pi = (float)ph[1];
  const Cx2 f(f2(w0 ? pr : 1.f, w1 ? pr : 1.f), f2(w0 ? pi : 0.f, w1 ? pi : 0.f));
#pragma unroll
  for (int k = 0; k < 6; k++) h[k] = h[k] * f;
}

template <int DAG, int MU, int PHM, class SF, class G>
LMB_D void hop_dir2(const Geom &g, int s0, const int *c0, int s1, const int *c1, const SF &in, const G &U,
                    Cx2 *acc) {
  constexpr int FPM = DAG ? +1 : -1;
  constexpr int BPM = -FPM;
  const bool ph = (g.phase_mask >> MU) & 1;
  Cx2 p[12], h[6], uh[6], u[9];
  {
    int w0, w1;
    const int sp0 = fwd_site(g, s0, c0, MU, 1, &w0);
    int sp1;
    if (MU < 3) {
      sp1 = sp0 + (s1 - s0);
      w1 = w0;
    } else {
      sp1 = fwd_site(g, s1, c1, MU, 1, &w1);
    }
    load2(in, sp0, sp1, p);
    project<FPM, MU>(p, h);
    if constexpr (PHM == PH_ANY) {
      if (ph && (w0 | w1)) phase2(h, g.ph_fwd[MU], w0, w1);
    } else if constexpr (MU == 3) {
      phase2(h, g.ph_fwd[3], w0, w1);
    }
    load2(U, MU, s0, s1, u);
    su3_mul_half(u, h, uh);
    reconstruct<FPM, MU>(acc, uh);
  }
  {
    int w0, w1;
    const int sm0 = bwd_site(g, s0, c0, MU, 1, &w0);
    int sm1;
    if (MU < 3) {
      sm1 = sm0 + (s1 - s0);
      w1 = w0;
    } else {
      sm1 = bwd_site(g, s1, c1, MU, 1, &w1);
    }
    load2(in, sm0, sm1, p);
    project<BPM, MU>(p, h);
    if constexpr (PHM == PH_ANY) {
      if (ph && (w0 | w1)) phase2(h, g.ph_bwd[MU], w0, w1);
    } else if constexpr (MU == 3) {
      phase2(h, g.ph_bwd[3], w0, w1);
    }
    load2(U, MU, sm0, sm1, u);
    su3_adj_mul_half(u, h, uh);
    reconstruct<BPM, MU>(acc, uh);
  }
}

// The two-site Wilson(-clover) kernel: V/2 threads.  Epi must provide
// skip() and pair(s0, s1, active, out[12]) with out[k] holding both sites.
template <int DAG, bool CLOVER, int PHM, class SF, class G, class CL, class Epi>
__global__ void __launch_bounds__(kDslashThreads, LMB_PAIR_MINB)
    wilson_dslash_pair_kernel(const Geom g, const SF in, const G U, const CL A, const float kappa, Epi epi) {
  if (epi.skip()) return;
  const int vh = (int)(g.V >> 1);
  const int s0 = blockIdx.x * kDslashThreads + threadIdx.x;
  const bool active = s0 < vh;
  const int s1 = s0 + vh;
  Cx2 out[12];
  if (active) {
    int c0[4], c1[4];
    site_coords(g, s0, c0);
    c1[0] = c0[0];
    c1[1] = c0[1];
    c1[2] = c0[2];
    c1[3] = c0[3] + (g.L[3] >> 1);
    Cx2 acc[12];
#pragma unroll
    for (int k = 0; k < 12; k++) acc[k] = cx2_zero();
    hop_dir2<DAG, 0, PHM>(g, s0, c0, s1, c1, in, U, acc);
    hop_dir2<DAG, 1, PHM>(g, s0, c0, s1, c1, in, U, acc);
    hop_dir2<DAG, 2, PHM>(g, s0, c0, s1, c1, in, U, acc);
    hop_dir2<DAG, 3, PHM>(g, s0, c0, s1, c1, in, U, acc);
    Cx2 p[12];
    load2(in, s0, s1, p);
    const float2 k2 = f2(kappa);
    if constexpr (CLOVER) {
      float2 a[36];
      Cx2 o[6];
#pragma unroll
      for (int blk = 0; blk < 2; blk++) {
        load2(A, blk, s0, s1, a);
        herm6_mul(a, p + 6 * blk, o);
#pragma unroll
        for (int k = 0; k < 6; k++) out[6 * blk + k] = cfms_real(k2, acc[6 * blk + k], o[k]);
      }
    } else {
#pragma unroll
      for (int k = 0; k < 12; k++) out[k] = cfms_real(k2, acc[k], p[k]);
    }
  }
  epi.pair(s0, s1, active, out);
}

// ---------------------------------------------------------------------------
// (1 + PM g_mu) psi straight from the raw int16 words of psi: a raw float is
// psi + c with c = base (1 + 2^-8) of its site (lmb_pair.cuh), so a
// difference of two raw values is psi_a - psi_b and a sum is
// (raw_a - 2c) + raw_b.  Every step is exact: operands and results are
// integers times the site's quantum 2^(e-15) below 2^24 in magnitude, so h
// equals project() of the decoded spinor bit for bit, with 2 or 3 FADD2 per
// complex entry of h instead of 6.  nc2 = -2c per lane.
// ---------------------------------------------------------------------------
template <int SIG>
LMB_D float2 raw_comb(float2 a, float2 b, float2 nc2) {
  if constexpr (SIG > 0) return (a + nc2) + b;
  else return a - b;
}
// a + SIG * b (IM = false) or a + SIG * i b (IM = true), a and b raw
template <int SIG, bool IM>
LMB_D Cx2 raw_term(const Cx2 &a, const Cx2 &b, float2 nc2) {
  if constexpr (IM) return Cx2(raw_comb<-SIG>(a.re, b.im, nc2), raw_comb<SIG>(a.im, b.re, nc2));
  else return Cx2(raw_comb<SIG>(a.re, b.re, nc2), raw_comb<SIG>(a.im, b.im, nc2));
}
// the rows of project<PM, MU> on raw words
template <int PM, int MU>
LMB_D void project_raw(const Cx2 *p, float2 nc2, Cx2 *h) {
  constexpr int S = PM > 0 ? 1 : -1;
#pragma unroll
  for (int c = 0; c < 3; c++) {
    if constexpr (MU == 0) {
      h[c] = raw_term<-S, true>(p[c], p[c + 9], nc2);
      h[c + 3] = raw_term<-S, true>(p[c + 3], p[c + 6], nc2);
    } else if constexpr (MU == 1) {
      h[c] = raw_term<-S, false>(p[c], p[c + 9], nc2);
      h[c + 3] = raw_term<S, false>(p[c + 3], p[c + 6], nc2);
    } else if constexpr (MU == 2) {
      h[c] = raw_term<-S, true>(p[c], p[c + 6], nc2);
      h[c + 3] = raw_term<S, true>(p[c + 3], p[c + 9], nc2);
    } else {
      h[c] = raw_term<-S, false>(p[c], p[c + 6], nc2);
      h[c + 3] = raw_term<-S, false>(p[c + 3], p[c + 9], nc2);
    }
  }
}

// ---------------------------------------------------------------------------
// int16 storage, reconstruct-12 links: lanes are x-adjacent sites s0 = 2i
// (x even) and s1 = s0 + 1 (lmb_pair.cuh: one 256-bit load per plane serves
// both).  y, z, t hops and the site's own links, spinor and clover use those
// loads; x hops, whose neighbours differ per lane, load each lane.
// ---------------------------------------------------------------------------
template <int DAG, int MU, int PHM>
LMB_D void hop_adj(const Geom &g, int s0, const int *c0, const int *c1, const Field<PREC_HALF, 12> &in,
                   const Gauge12<PREC_HALF> &U, Cx2 *acc) {
  constexpr int FPM = DAG ? +1 : -1;
  constexpr int BPM = -FPM;
  const bool ph = (g.phase_mask >> MU) & 1;
  Cx2 p[12], h[6], uh[6], u[9];
  float2 nc2;
  {
    int w0, w1;
    if constexpr (MU == 0) {
      w0 = 0;  // x + 1 of an even x never crosses the edge
      const int n1 = fwd_site(g, s0 + 1, c1, 0, 1, &w1);
      load2_raw(in, s0 + 1, n1, p, nc2);
    } else {
      load_adj_raw(in, fwd_site(g, s0, c0, MU, 1, &w0), p, nc2);
      w1 = w0;
    }
    project_raw<FPM, MU>(p, nc2, h);
    if constexpr (PHM == PH_ANY) {
      if (ph && (w0 | w1)) phase2(h, g.ph_fwd[MU], w0, w1);
    } else if constexpr (MU == 3) {
      phase2(h, g.ph_fwd[3], w0, w1);
    }
    load_adj(U, MU, s0, u);
    su3_mul_half(u, h, uh);
    reconstruct<FPM, MU>(acc, uh);
  }
  {
    int w0, w1;
    if constexpr (MU == 0) {
      const int n0 = bwd_site(g, s0, c0, 0, 1, &w0);
      w1 = 0;  // x - 1 of an odd x never crosses the edge
      load2_raw(in, n0, s0, p, nc2);
      project_raw<BPM, MU>(p, nc2, h);
      if constexpr (PHM == PH_ANY) {
        if (ph && (w0 | w1)) phase2(h, g.ph_bwd[MU], w0, w1);
      }
      load2(U, 0, n0, s0, u);
    } else {
      const int n0 = bwd_site(g, s0, c0, MU, 1, &w0);
      w1 = w0;
      load_adj_raw(in, n0, p, nc2);
      project_raw<BPM, MU>(p, nc2, h);
      if constexpr (PHM == PH_ANY) {
        if (ph && (w0 | w1)) phase2(h, g.ph_bwd[MU], w0, w1);
      } else if constexpr (MU == 3) {
        phase2(h, g.ph_bwd[3], w0, w1);
      }
      load_adj(U, MU, n0, u);
    }
    su3_adj_mul_half(u, h, uh);
    reconstruct<BPM, MU>(acc, uh);
  }
}

// D psi (or D^+ psi) at the x-adjacent sites s0 (x even) and s0 + 1
template <int DAG, bool CLOVER, int PHM, class CL>
LMB_D void half_adj_sites(const Geom &g, int s0, const Field<PREC_HALF, 12> &in, const Gauge12<PREC_HALF> &U,
                          const CL &A, float kappa, Cx2 *out) {
  int c0[4], c1[4];
  site_coords(g, s0, c0);
  c1[0] = c0[0] + 1;
  c1[1] = c0[1];
  c1[2] = c0[2];
  c1[3] = c0[3];
  // out = -kappa * hopping sum, then A psi accumulated into it (no separate
  // A psi array is live)
#pragma unroll
  for (int k = 0; k < 12; k++) out[k] = cx2_zero();
  hop_adj<DAG, 0, PHM>(g, s0, c0, c1, in, U, out);
  hop_adj<DAG, 1, PHM>(g, s0, c0, c1, in, U, out);
  hop_adj<DAG, 2, PHM>(g, s0, c0, c1, in, U, out);
  hop_adj<DAG, 3, PHM>(g, s0, c0, c1, in, U, out);
  Cx2 p[12];
  load_adj(in, s0, p);
  const float2 nk2 = f2(-kappa);
  if constexpr (CLOVER) {
#pragma unroll
    for (int k = 0; k < 12; k++) out[k] = Cx2(nk2 * out[k].re, nk2 * out[k].im);
    float2 a[36];
#pragma unroll
    for (int blk = 0; blk < 2; blk++) {
      load_adj(A, blk, s0, a);
      herm6_mul_acc(a, p + 6 * blk, out + 6 * blk);
    }
  } else {
#pragma unroll
    for (int k = 0; k < 12; k++) out[k] = Cx2(fma2(nk2, out[k].re, p[k].re), fma2(nk2, out[k].im, p[k].im));
  }
}

// one thread per pair of the range (rg.lo, rg.hi even); needs x even.  Epi
// must provide skip() and pair_adj(s0, active, out[12]) (sites s0, s0 + 1).
template <int DAG, bool CLOVER, int PHM, class CL, class Epi>
__global__ void __launch_bounds__(kDslashThreads, LMB_PAIR_MINB)
    wilson_half_adj_kernel(const Geom g, const Field<PREC_HALF, 12> in, const Gauge12<PREC_HALF> U, const CL A,
                           const float kappa, Epi epi, const SiteRange rg) {
  if (epi.skip()) return;
  const int i = blockIdx.x * kDslashThreads + threadIdx.x;
  const bool active = i < ((rg.hi - rg.lo) >> 1);
  const int s0 = rg.lo + 2 * i;
  Cx2 out[12];
  if (active) half_adj_sites<DAG, CLOVER, PHM>(g, s0, in, U, A, kappa, out);
  epi.pair_adj(s0, active, out);
}

// Persistent form for the reducing CG epilogues: gridDim.x blocks (the
// device's resident blocks) walk the tiles of kDslashThreads pairs
// t = blockIdx.x, blockIdx.x + gridDim.x, ... in a fixed order.  The
// epilogue carries its reduction in registers across the tiles
// (pair_adj_acc) and reduces once per block at the end (finish), so no block
// waits at a barrier or on the grid counter between tiles, and the result
// does not depend on timing.
template <int DAG, bool CLOVER, int PHM, class CL, class Epi>
__global__ void __launch_bounds__(kDslashThreads, LMB_PAIR_MINB)
    wilson_half_adj_persistent_kernel(const Geom g, const Field<PREC_HALF, 12> in, const Gauge12<PREC_HALF> U,
                                      const CL A, const float kappa, Epi epi, int ntiles, const SiteRange rg) {
  if (epi.skip()) return;
  double red[1] = {0.0};
  const int npairs = (rg.hi - rg.lo) >> 1;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int i = tile * kDslashThreads + threadIdx.x;
    const bool active = i < npairs;
    const int s0 = rg.lo + 2 * i;
    Cx2 out[12];
    if (active) half_adj_sites<DAG, CLOVER, PHM>(g, s0, in, U, A, kappa, out);
    epi.pair_adj_acc(s0, active, out, red);
  }
  epi.finish(red);
}

}  // namespace lmb
