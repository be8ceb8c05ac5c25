// lmb_evenodd.cuh -- even/odd (Schur) preconditioned Wilson / Wilson-clover
// solve of D x = b.
//
// D = A - kappa H with A = 1 (Wilson) or 1 + clover term (two Hermitian 6x6
// blocks per site, WilsonDiracCloverOperator.jl:481-525) and H the hopping
// term.  H only couples sites of opposite parity, so on (even, odd) blocks
//   D = [[A_ee, -k H_eo], [-k H_oe, A_oo]],
// and with the Schur complement  Dh = A_ee - k^2 H_eo A_oo^-1 H_oe:
//   bh_e = b_e + k H_eo A_oo^-1 b_o,   Dh x_e = bh_e,
//   x_o  = A_oo^-1 (b_o + k H_oe x_e).
// The odd equations then hold exactly and the even residual is
// bh_e - Dh x_e, so the full residual |b - D x| is the Schur system's.
// Dh is solved by CG on Dh Dh^+ y = bh_e, x_e = Dh^+ y (CGNE: its residual
// is bh_e - Dh x_e itself), with Dh^+ = A_ee - k^2 H^+_eo A_oo^-1 H^+_oe.
//
// Links and clover blocks are read from parity-ordered copies (site s at
// parity(s) V/2 + s/2, every plane permuted alike), so the sites of one
// parity are contiguous and no sector carries the other parity's data.
//
// Parity: a site is even when its global coordinate sum is
// (_global_site_is_even, LatticeMatrices.jl:357-363; the even/odd kernels
// of linearalgebra_D.jl:2815-2930 use the same rule).  Half fields hold the
// V/2 sites of one parity at checkerboard index lex / 2, which needs an even
// x extent; periodic parity needs every extent even.
#pragma once
#include "lmb_pack.cuh"
#include "lmb_solver.cuh"

namespace lmb {

LMB_D int coord_parity(const Geom &g, const int c[4]) {
  return (c[0] + c[1] + c[2] + c[3] + g.eta_off[0] + g.eta_off[1] + g.eta_off[2] + g.eta_off[3]) & 1;
}

// checkerboard index cb of parity p: lexicographic site and its coordinates
LMB_D int cb_site(const Geom &g, int cb, int p, int c[4]) {
  const int lex0 = 2 * cb;
  site_coords(g, lex0, c);  // c[0] even
  const int fix = (coord_parity(g, c) + p) & 1;
  c[0] += fix;
  return lex0 + fix;
}

// site s at parity(s) V/2 + s/2 in each of `nplanes` planes of V elements
template <typename T>
__global__ void __launch_bounds__(256)
    eo_permute_kernel(T *dst, const T *src, int nplanes, const Geom g) {
  const int64_t s = (int64_t)blockIdx.x * 256 + threadIdx.x;
  if (s >= g.V) return;
  int c[4];
  site_coords(g, (int)s, c);
  const int64_t e = (int64_t)coord_parity(g, c) * (g.V / 2) + (s >> 1);
  for (int k = 0; k < nplanes; k++) dst[k * g.V + e] = src[k * g.V + s];
}

// ---------------------------------------------------------------------------
// clover block inverse: each Hermitian 6x6 block (6 real diagonal entries,
// then the 15 complex entries below the diagonal row by row) is inverted by
// Gauss-Jordan elimination with partial pivoting in FP64; the inverse is
// Hermitian and is stored in the same packed form.  A pivot below 1e-12 of
// the block's largest entry counts the block as singular in *bad.
// ---------------------------------------------------------------------------
template <int = 0>
__global__ void __launch_bounds__(128) clover_invert_kernel(double2 *dst, const double2 *src, int64_t V,
                                                            unsigned *bad) {
  const int64_t t = (int64_t)blockIdx.x * 128 + threadIdx.x;
  if (t >= 2 * V) return;
  const int blk = (int)(t / V);
  const int64_t s = t - (int64_t)blk * V;
  double a[36];
#pragma unroll
  for (int k = 0; k < 18; k++) {
    const double2 q = src[(blk * 18 + k) * V + s];
    a[2 * k] = q.x;
    a[2 * k + 1] = q.y;
  }
  double mr[6][12], mi[6][12];  // [A | I]
  double amax = 0.0;
#pragma unroll
  for (int i = 0; i < 6; i++)
#pragma unroll
    for (int j = 0; j < 12; j++) {
      mr[i][j] = (j == i + 6) ? 1.0 : 0.0;
      mi[i][j] = 0.0;
    }
#pragma unroll
  for (int i = 0; i < 6; i++) {
    mr[i][i] = a[i];
    amax = fmax(amax, fabs(a[i]));
  }
  {
    int k = 6;
#pragma unroll
    for (int i = 1; i < 6; i++)
#pragma unroll
      for (int j = 0; j < i; j++) {
        mr[i][j] = a[k];
        mi[i][j] = a[k + 1];
        mr[j][i] = a[k];
        mi[j][i] = -a[k + 1];
        amax = fmax(amax, fabs(a[k]) + fabs(a[k + 1]));
        k += 2;
      }
  }
  bool singular = !(amax > 0.0);
  for (int col = 0; col < 6; col++) {
    int piv = col;
    double best = mr[col][col] * mr[col][col] + mi[col][col] * mi[col][col];
    for (int r = col + 1; r < 6; r++) {
      const double m2 = mr[r][col] * mr[r][col] + mi[r][col] * mi[r][col];
      if (m2 > best) {
        best = m2;
        piv = r;
      }
    }
    if (!(best > 1e-24 * amax * amax)) {
      singular = true;
      break;
    }
    if (piv != col)
      for (int j = 0; j < 12; j++) {
        double tr = mr[col][j], ti = mi[col][j];
        mr[col][j] = mr[piv][j];
        mi[col][j] = mi[piv][j];
        mr[piv][j] = tr;
        mi[piv][j] = ti;
      }
    // row col /= pivot
    const double pr = mr[col][col], pi = mi[col][col];
    const double inv = 1.0 / (pr * pr + pi * pi);
    const double qr = pr * inv, qi = -pi * inv;  // 1 / pivot
    for (int j = 0; j < 12; j++) {
      const double xr = mr[col][j], xi = mi[col][j];
      mr[col][j] = xr * qr - xi * qi;
      mi[col][j] = xr * qi + xi * qr;
    }
    for (int r = 0; r < 6; r++) {
      if (r == col) continue;
      const double fr = mr[r][col], fi = mi[r][col];
      for (int j = 0; j < 12; j++) {
        const double xr = mr[col][j], xi = mi[col][j];
        mr[r][j] -= fr * xr - fi * xi;
        mi[r][j] -= fr * xi + fi * xr;
      }
    }
  }
  if (singular) {
    atomicAdd(bad, 1u);
    return;
  }
  double o[36];
#pragma unroll
  for (int i = 0; i < 6; i++) o[i] = mr[i][i + 6];
  {
    int k = 6;
#pragma unroll
    for (int i = 1; i < 6; i++)
#pragma unroll
      for (int j = 0; j < i; j++) {
        o[k] = mr[i][j + 6];
        o[k + 1] = mi[i][j + 6];
        k += 2;
      }
  }
#pragma unroll
  for (int k = 0; k < 18; k++) dst[(blk * 18 + k) * V + s] = make_double2(o[2 * k], o[2 * k + 1]);
}

// ---------------------------------------------------------------------------
// half-field kernels
// ---------------------------------------------------------------------------
// hop of direction MU into site s (lexicographic, parity p, parity-ordered
// index es) from the opposite-parity half field `in` (neighbour n at
// checkerboard index n / 2); U parity-ordered
template <typename R, int DAG, int MU, class SF, class G>
LMB_D void eo_hop(const Geom &g, int s, int64_t es, int p, const int *c, const SF &in, const G &U, Cx<R> *acc) {
  constexpr int FPM = DAG ? +1 : -1;
  constexpr int BPM = -FPM;
  Cx<R> q[12], h[6], uh[6], u[9];
  int wrap;
  {
    const int sp = fwd_site(g, s, c, MU, 1, &wrap);
    in.load(sp >> 1, q);
    project<FPM, MU>(q, h);
    if (wrap && ((g.phase_mask >> MU) & 1)) scale_phase(h, 6, g.ph_fwd[MU]);
    U.load(MU, es, u);
    su3_mul_half(u, h, uh);
    reconstruct<FPM, MU>(acc, uh);
  }
  {
    const int sm = bwd_site(g, s, c, MU, 1, &wrap);
    in.load(sm >> 1, q);
    project<BPM, MU>(q, h);
    if (wrap && ((g.phase_mask >> MU) & 1)) scale_phase(h, 6, g.ph_bwd[MU]);
    U.load(MU, (int64_t)(1 - p) * (g.V / 2) + (sm >> 1), u);
    su3_adj_mul_half(u, h, uh);
    reconstruct<BPM, MU>(acc, uh);
  }
}

template <typename R, class C>
LMB_D void clover_apply(const C &A, int64_t s, Cx<R> *v) {
#pragma unroll
  for (int blk = 0; blk < 2; blk++) {
    R a[36];
    Cx<R> o[6];
    A.load(blk, s, a);
    herm6_mul(a, v + 6 * blk, o);
#pragma unroll
    for (int k = 0; k < 6; k++) v[6 * blk + k] = o[k];
  }
}

// Sites of parity p (one thread per checkerboard index; links and clover
// blocks parity-ordered):
//   v = c1 W(x) [WMODE 1]  or  c1 A(x) W(x) [WMODE 2]  (W: parity p)
//     + c2 (H in)(x)        (H^+ when DAG; in: parity 1 - p)
//   out = A^-1(x) v when AINV, else v.     CL = false: A = 1.
template <typename R, int DAG, int WMODE, bool AINV, bool CL, class SF, class G, class C, class Epi>
__global__ void __launch_bounds__(kDslashThreads)
    eo_hop_kernel(const Geom g, const int p, const SF in, const SF W, const G U, const C A, const C Ainv,
                  const R c1, const R c2, Epi epi) {
  if (epi.skip()) return;
  const int64_t cb = (int64_t)blockIdx.x * kDslashThreads + threadIdx.x;
  const bool active = cb < g.V / 2;
  Cx<R> v[12];
  if (active) {
    int c[4];
    const int s = cb_site(g, (int)cb, p, c);
    const int64_t es = (int64_t)p * (g.V / 2) + cb;
    Cx<R> acc[12];
#pragma unroll
    for (int k = 0; k < 12; k++) acc[k] = Cx<R>(0, 0);
    eo_hop<R, DAG, 0>(g, s, es, p, c, in, U, acc);
    eo_hop<R, DAG, 1>(g, s, es, p, c, in, U, acc);
    eo_hop<R, DAG, 2>(g, s, es, p, c, in, U, acc);
    eo_hop<R, DAG, 3>(g, s, es, p, c, in, U, acc);
#pragma unroll
    for (int k = 0; k < 12; k++) v[k] = c2 * acc[k];
    if constexpr (WMODE != 0) {
      Cx<R> w[12];
      W.load(cb, w);
      if constexpr (WMODE == 2 && CL) clover_apply<R>(A, es, w);
#pragma unroll
      for (int k = 0; k < 12; k++) v[k] = v[k] + c1 * w[k];
    }
    if constexpr (AINV && CL) clover_apply<R>(Ainv, es, v);
  }
  epi((int)(active ? cb : 0), active, v);
}

// out = A^-1 in on the sites of parity p (CL = false: a copy; Ainv
// parity-ordered)
template <bool CL, class C>
__global__ void __launch_bounds__(256)
    eo_local_kernel(Field<PREC_DOUBLE, 12> out, const Field<PREC_DOUBLE, 12> in, const Geom g, const int p,
                    const C Ainv) {
  const int64_t cb = (int64_t)blockIdx.x * 256 + threadIdx.x;
  if (cb >= g.V / 2) return;
  Cx<double> v[12];
  in.load(cb, v);
  if constexpr (CL) clover_apply<double>(Ainv, (int64_t)p * (g.V / 2) + cb, v);
  out.store(cb, v);
}

// padded reference layout <-> even and odd half fields (FP64)
template <typename T>
__global__ void __launch_bounds__(256)
    eo_pack_kernel(Field<PREC_DOUBLE, 12> e, Field<PREC_DOUBLE, 12> o, const T *src, const Geom g,
                   const Padded pd) {
  const int64_t s = (int64_t)blockIdx.x * 256 + threadIdx.x;
  if (s >= g.V) return;
  int c[4];
  site_coords(g, (int)s, c);
  const T *q = src + padded_site(pd, c) * 12;
  Cx<double> v[12];
#pragma unroll
  for (int k = 0; k < 12; k++) v[k] = Cx<double>((double)q[k].x, (double)q[k].y);
  (coord_parity(g, c) ? o : e).store(s >> 1, v);
}
template <typename T>
__global__ void __launch_bounds__(256)
    eo_unpack_kernel(T *dst, const Field<PREC_DOUBLE, 12> e, const Field<PREC_DOUBLE, 12> o, const Geom g,
                     const Padded pd) {
  const int64_t s = (int64_t)blockIdx.x * 256 + threadIdx.x;
  if (s >= g.V) return;
  int c[4];
  site_coords(g, (int)s, c);
  T *q = dst + padded_site(pd, c) * 12;
  Cx<double> v[12];
  (coord_parity(g, c) ? o : e).load(s >> 1, v);
#pragma unroll
  for (int k = 0; k < 12; k++) {
    q[k].x = v[k].re;
    q[k].y = v[k].im;
  }
}

// |e|^2 + |o|^2 into *out
template <int = 0>
__global__ void __launch_bounds__(256)
    eo_norm2_kernel(const Field<PREC_DOUBLE, 12> e, const Field<PREC_DOUBLE, 12> o, int64_t Vh, double *partials,
                    unsigned *counter, double *out) {
  const int64_t cb = (int64_t)blockIdx.x * 256 + threadIdx.x;
  double n2[1] = {0.0}, tot[1];
  if (cb < Vh) {
    Cx<double> v[12];
    e.load(cb, v);
    n2[0] += sum_norm2(v, 12);
    o.load(cb, v);
    n2[0] += sum_norm2(v, 12);
  }
  if (grid_reduce<256, 1>(n2, partials, counter, tot) && threadIdx.x == 0) *out = tot[0];
}

}  // namespace lmb
