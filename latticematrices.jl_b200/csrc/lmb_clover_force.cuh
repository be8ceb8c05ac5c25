// lmb_clover_force.cuh -- hand-written adjoint of the Wilson-clover operator
// (FP64): gradient of f = coef Re<dr, D(U) psi> with respect to the links
// (wilson_clover_link_pullback!, WilsonCloverPullback.jl:342-403),
//   D psi = psi - kappa sum_mu [U_mu(x)(1 - g_mu)psi(x+mu) + U_mu(x-mu)^+(1 + g_mu)psi(x-mu)]
//           - kappa cSW sum_{mu<nu} G_mu_nu F_mu_nu psi,
//   F_mu_nu = (Q - Q^+)/8,  Q = the four plaquette leaves at x.
// Convention as lmb_hisq_force.cuh: df = Re sum conj(G_ij) dU_ij.
// Three stages, each gathering at the site it owns (no atomics):
//   1. hopping term: dU_mu(x) += c [dr(x) ((1-g)psi(x+mu))^+ + ((1+g)psi(x)) dr(x+mu)^+]
//      (WilsonDiracOperator.jl:382-411), fermion phases on wrapped hops;
//   2. cotangent of each F_mu_nu: dF(x) = c' sum_spin dr(x) (G psi(x))^+
//      (WilsonCloverPullback.jl:99-159);
//   3. through F = (Q - Q^+)/8 onto the links of the leaves: dQ = (dF - dF^+)/8,
//      and for a leaf P = M1 M2 M3 M4 the factor M_K = U gets left^+ dQ right^+,
//      M_K = U^+ gets right dQ^+ left (WilsonCloverPullback.jl:161-292).
#pragma once
#include "lmb_hisq_smear.cuh"
#include "lmb_wilson.cuh"

namespace lmb {

// (1 + PM g_mu) psi as a full 12-component spinor (k = colour + 3 spin)
template <int PM, int MU>
LMB_D void spin_project_full(const Cx<double> *psi, Cx<double> *out) {
  Cx<double> h[6];
  project<PM, MU>(psi, h);
#pragma unroll
  for (int k = 0; k < 12; k++) out[k] = Cx<double>(0, 0);
  reconstruct<PM, MU>(out, h);
}

// G[a + 3b] += c sum_spin x[a + 3s] conj(y[b + 3s])
LMB_D void outer_spin_add(const Cx<double> *x, const Cx<double> *y, double c, Cx<double> *G) {
#pragma unroll
  for (int a = 0; a < 3; a++)
#pragma unroll
    for (int b = 0; b < 3; b++) {
      Cx<double> v(0, 0);
#pragma unroll
      for (int s = 0; s < 4; s++) v = cfma_conj(y[b + 3 * s], x[a + 3 * s], v);
      G[a + 3 * b] = G[a + 3 * b] + c * v;
    }
}

template <int MU>
LMB_D void hop_outer(const Geom &g, int s, const int *c, const Field<PREC_DOUBLE, 12> &dr,
                     const Field<PREC_DOUBLE, 12> &psi, const Cx<double> *dr_x, const Cx<double> *psi_x,
                     double coef, double2 *dU) {
  int w;
  const int sp = fwd_site(g, s, c, MU, 1, &w);
  const bool ph = w && ((g.phase_mask >> MU) & 1);
  Cx<double> v[12], t[12], G[9];
  load9(dU + (size_t)MU * 9 * g.V, g.V, s, G);
  // U_mu(x) (1 - g) psi(x+mu) in (D psi)(x)
  psi.load(sp, t);
  if (ph) {
    const Cx<double> f(g.ph_fwd[MU][0], g.ph_fwd[MU][1]);
#pragma unroll
    for (int k = 0; k < 12; k++) t[k] = t[k] * f;
  }
  spin_project_full<-1, MU>(t, v);
  outer_spin_add(dr_x, v, coef, G);
  // U_mu(x)^+ (1 + g) psi(x) in (D psi)(x+mu), 1/phase when that hop wraps
  spin_project_full<+1, MU>(psi_x, v);
  if (ph) {
    const Cx<double> f(g.ph_bwd[MU][0], g.ph_bwd[MU][1]);
#pragma unroll
    for (int k = 0; k < 12; k++) v[k] = v[k] * f;
  }
  dr.load(sp, t);
  outer_spin_add(v, t, coef, G);
  store9(dU + (size_t)MU * 9 * g.V, g.V, s, G);
}

// stage 1: dU (36 planes, mu*9 + r + 3c) += coef * hopping-term gradient
template <int = 0>
__global__ void __launch_bounds__(128)
    wilson_outer_product_kernel(double2 *dU, const Field<PREC_DOUBLE, 12> dr, const Field<PREC_DOUBLE, 12> psi,
                                const Geom g, double coef) {
  const int s = blockIdx.x * 128 + threadIdx.x;
  if (s >= g.V) return;
  int c[4];
  site_coords(g, s, c);
  Cx<double> d[12], p[12];
  dr.load(s, d);
  psi.load(s, p);
  hop_outer<0>(g, s, c, dr, psi, d, p, coef, dU);
  hop_outer<1>(g, s, c, dr, psi, d, p, coef, dU);
  hop_outer<2>(g, s, c, dr, psi, d, p, coef, dU);
  hop_outer<3>(g, s, c, dr, psi, d, p, coef, dU);
}

// spin matrices of the clover term per plane (12, 13, 14, 23, 24, 34), as
// the block form of kernel_add_clover_term! (WilsonDiracCloverOperator.jl:
// 481-525): (G psi)_s for each colour
template <int PLANE>
LMB_D void clover_gamma_apply(const Cx<double> *p, Cx<double> *o) {
  const Cx<double> I(0, 1);
#pragma unroll
  for (int c = 0; c < 3; c++) {
    const Cx<double> p1 = p[c], p2 = p[c + 3], p3 = p[c + 6], p4 = p[c + 9];
    Cx<double> o1, o2, o3, o4;
    if (PLANE == 0) {  // 12: diag(i, -i, i, -i)
      o1 = I * p1; o2 = -(I * p2); o3 = I * p3; o4 = -(I * p4);
    } else if (PLANE == 1) {  // 13
      o1 = -p2; o2 = p1; o3 = -p4; o4 = p3;
    } else if (PLANE == 2) {  // 14
      o1 = I * p2; o2 = I * p1; o3 = -(I * p4); o4 = -(I * p3);
    } else if (PLANE == 3) {  // 23
      o1 = I * p2; o2 = I * p1; o3 = I * p4; o4 = I * p3;
    } else if (PLANE == 4) {  // 24
      o1 = p2; o2 = -p1; o3 = -p4; o4 = p3;
    } else {  // 34: diag(i, -i, -i, i)
      o1 = I * p1; o2 = -(I * p2); o3 = -(I * p3); o4 = I * p4;
    }
    o[c] = o1;
    o[c + 3] = o2;
    o[c + 6] = o3;
    o[c + 9] = o4;
  }
}

template <int PLANE>
LMB_D void clover_cotangent_plane(const Cx<double> *d, const Cx<double> *p, double coef, double2 *dF, int64_t V,
                                  int s) {
  Cx<double> gp[12], G[9];
  clover_gamma_apply<PLANE>(p, gp);
#pragma unroll
  for (int k = 0; k < 9; k++) G[k] = Cx<double>(0, 0);
  outer_spin_add(d, gp, coef, G);
  store9(dF + (size_t)PLANE * 9 * V, V, s, G);
}

// stage 2: dF (6 planes of 3x3) = coef sum_spin dr (G_plane psi)^+
template <int = 0>
__global__ void __launch_bounds__(128)
    clover_cotangent_kernel(double2 *dF, const Field<PREC_DOUBLE, 12> dr, const Field<PREC_DOUBLE, 12> psi,
                            const Geom g, double coef) {
  const int s = blockIdx.x * 128 + threadIdx.x;
  if (s >= g.V) return;
  Cx<double> d[12], p[12];
  dr.load(s, d);
  psi.load(s, p);
  clover_cotangent_plane<0>(d, p, coef, dF, g.V, s);
  clover_cotangent_plane<1>(d, p, coef, dF, g.V, s);
  clover_cotangent_plane<2>(d, p, coef, dF, g.V, s);
  clover_cotangent_plane<3>(d, p, coef, dF, g.V, s);
  clover_cotangent_plane<4>(d, p, coef, dF, g.V, s);
  clover_cotangent_plane<5>(d, p, coef, dF, g.V, s);
}

// a = a * b
LMB_D void mat3_mul_inplace(Cx<double> *a, const Cx<double> *b) { mat3_mul(a, b, a); }

// stage 3 for one plane (mu, nu): the links U_mu(x), U_nu(x) of site x gather
// their occurrences in the four leaves of every anchor
template <int = 0>
__global__ void __launch_bounds__(64)
    clover_link_pullback_kernel(double2 *dU, const double2 *U, const double2 *dF, const Geom g, int plane,
                                int mu, int nu) {
  const int s = blockIdx.x * 64 + threadIdx.x;
  if (s >= g.V) return;
  const int64_t V = g.V;
  // leaves of Q(x), 1-based signed directions (the order of the field
  // strength: +mu+nu-mu-nu, +nu-mu-nu+mu, -mu-nu+mu+nu, -nu+mu+nu-mu)
  const int m1 = mu + 1, n1 = nu + 1;
  const int leaves[4][4] = {{m1, n1, -m1, -n1}, {n1, -m1, -n1, m1}, {-m1, -n1, m1, n1}, {-n1, m1, n1, -m1}};
  Cx<double> dmu[9], dnu[9];
#pragma unroll
  for (int k = 0; k < 9; k++) dmu[k] = dnu[k] = Cx<double>(0, 0);
  for (int l = 0; l < 4; l++) {
    for (int K = 0; K < 4; K++) {
      // offset of factor K's link site from the anchor
      int off[4] = {0, 0, 0, 0};
      for (int k = 0; k < K; k++) {
        const int d = leaves[l][k], a = (d > 0 ? d : -d) - 1;
        off[a] += d > 0 ? 1 : -1;
      }
      {
        const int d = leaves[l][K], a = (d > 0 ? d : -d) - 1;
        if (d < 0) off[a] -= 1;
      }
      int anchor = s;
      for (int a = 0; a < 4; a++)
        for (int k = 0; k < (off[a] > 0 ? off[a] : -off[a]); k++) anchor = nb_site(g, anchor, a, off[a] > 0 ? -1 : 1);
      // factors and partial products along the leaf from the anchor
      Cx<double> left[9], right[9], m[9];
#pragma unroll
      for (int k = 0; k < 9; k++) left[k] = right[k] = Cx<double>((k % 4) == 0 ? 1.0 : 0.0, 0);
      int site = anchor;
      for (int k = 0; k < 4; k++) {
        const int d = leaves[l][k], a = (d > 0 ? d : -d) - 1;
        if (d > 0) {
          load9(U + (size_t)a * 9 * V, V, site, m);
          site = nb_site(g, site, a, 1);
        } else {
          site = nb_site(g, site, a, -1);
          Cx<double> t[9];
          load9(U + (size_t)a * 9 * V, V, site, t);
#pragma unroll
          for (int r = 0; r < 3; r++)
#pragma unroll
            for (int cc = 0; cc < 3; cc++) m[r + 3 * cc] = conj(t[cc + 3 * r]);
        }
        if (k < K) mat3_mul_inplace(left, m);
        else if (k > K) mat3_mul_inplace(right, m);
      }
      // dQ = (dF - dF^+)/8 at the anchor
      Cx<double> f[9], dQ[9], h[9], t[9];
      load9(dF + (size_t)plane * 9 * V, V, anchor, f);
#pragma unroll
      for (int r = 0; r < 3; r++)
#pragma unroll
        for (int cc = 0; cc < 3; cc++) {
          const Cx<double> a = f[r + 3 * cc], b = conj(f[cc + 3 * r]);
          dQ[r + 3 * cc] = Cx<double>(0.125 * (a.re - b.re), 0.125 * (a.im - b.im));
        }
      const int dK = leaves[l][K];
      if (dK > 0) {  // left^+ dQ right^+
        mat3_adj_mul(left, dQ, t);
        mat3_mul_adj(t, right, h);
      } else {  // right dQ^+ left
        mat3_mul_adj(right, dQ, t);
        mat3_mul(t, left, h);
      }
      Cx<double> *acc = ((dK > 0 ? dK : -dK) - 1 == mu) ? dmu : dnu;
#pragma unroll
      for (int k = 0; k < 9; k++) acc[k] = acc[k] + h[k];
    }
  }
  Cx<double> o[9];
  load9(dU + (size_t)mu * 9 * V, V, s, o);
#pragma unroll
  for (int k = 0; k < 9; k++) o[k] = o[k] + dmu[k];
  store9(dU + (size_t)mu * 9 * V, V, s, o);
  load9(dU + (size_t)nu * 9 * V, V, s, o);
#pragma unroll
  for (int k = 0; k < 9; k++) o[k] = o[k] + dnu[k];
  store9(dU + (size_t)nu * 9 * V, V, s, o);
}

}  // namespace lmb
