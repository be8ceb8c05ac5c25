// lmb_hisq_force.cuh -- hand-written adjoint of the HISQ chain (FP64):
// thin links -> level-1 Fat7 -> U(3) projection -> level-2 Fat7 + Lepage,
// Naik -> HISQ stencil, for f = coef Re<dr, D(U) psi>
// (hisq_link_pullback!, HISQPullback.jl:620-699).
//
// Convention: the gradient G of a real f with respect to a complex matrix
// field satisfies df = Re sum conj(G_ij) dU_ij, so that for f = Re tr(dT^+ A U B)
// G_U = A^+ dT B^+ and, for a daggered occurrence A U^+ B, G_U = B dT^+ A.
// Every kernel gathers the contributions to the site it owns (no atomics).
//
// Smearing levels are recomputed instead of stored: the Fat7 pullback of a
// direction mu rebuilds that direction's 3- and 5-link staples from the
// level's input links, then runs the factorised forward pass backwards.  The
// staple transport
//   T_nu(M)(x) = U_nu(x) M(x+nu) U_nu(x+mu)^+ + U_nu(x-nu)^+ M(x-nu) U_nu(x-nu+mu)
// is its own adjoint in M (its forward half's adjoint is the backward half
// and vice versa), so dM = T_nu(dT) reuses staple_transport_kernel.
#pragma once
#include "lmb_hisq_smear.cuh"
#include "lmb_staggered.cuh"

namespace lmb {

// dU_nu (+)= coef * d/dU_nu Re<dT, T_nu(M)> for the halves in `signs`
// (1: U_nu(x) M(x+nu) U_nu(x+mu)^+, 2: U_nu(x-nu)^+ M(x-nu) U_nu(x-nu+mu))
template <int = 0>
__global__ void __launch_bounds__(kSmearThreads)
    transport_link_grad_kernel(double2 *dUnu, const double2 *dT, const double2 *M, const double2 *U, const Geom g,
                               int mu, int nu, int signs, double coef) {
  const int z = blockIdx.x * kSmearThreads + threadIdx.x;
  if (z >= g.V) return;
  const int64_t V = g.V;
  const double2 *Unu = U + (size_t)nu * 9 * V;
  Cx<double> acc[9], a[9], b[9], c[9];
#pragma unroll
  for (int k = 0; k < 9; k++) acc[k] = Cx<double>(0, 0);
  const int zpm = nb_site(g, z, mu, 1), zpn = nb_site(g, z, nu, 1), zmm = nb_site(g, z, mu, -1);
  if (signs & 1) {
    // (a) dT(z) U_nu(z+mu) M(z+nu)^+
    load9(dT, V, z, a);
    load9(Unu, V, zpm, b);
    mat3_mul(a, b, a);
    load9(M, V, zpn, c);
    mat3_mul_adj(a, c, a);
#pragma unroll
    for (int k = 0; k < 9; k++) acc[k] = acc[k] + a[k];
    // (b) dT(z-mu)^+ U_nu(z-mu) M(z-mu+nu)
    const int zmm_pn = nb_site(g, zmm, nu, 1);
    load9(dT, V, zmm, a);
    load9(Unu, V, zmm, b);
    mat3_adj_mul(a, b, a);
    load9(M, V, zmm_pn, c);
    mat3_mul(a, c, a);
#pragma unroll
    for (int k = 0; k < 9; k++) acc[k] = acc[k] + a[k];
  }
  if (signs & 2) {
    // (c) M(z) U_nu(z+mu) dT(z+nu)^+
    load9(M, V, z, a);
    load9(Unu, V, zpm, b);
    mat3_mul(a, b, a);
    load9(dT, V, zpn, c);
    mat3_mul_adj(a, c, a);
#pragma unroll
    for (int k = 0; k < 9; k++) acc[k] = acc[k] + a[k];
    // (d) M(z-mu)^+ U_nu(z-mu) dT(z-mu+nu)
    const int zmm_pn = nb_site(g, zmm, nu, 1);
    load9(M, V, zmm, a);
    load9(Unu, V, zmm, b);
    mat3_adj_mul(a, b, a);
    load9(dT, V, zmm_pn, c);
    mat3_mul(a, c, a);
#pragma unroll
    for (int k = 0; k < 9; k++) acc[k] = acc[k] + a[k];
  }
  double2 *out = dUnu + (size_t)nu * 9 * V;
  load9(out, V, z, b);
#pragma unroll
  for (int k = 0; k < 9; k++) b[k] = b[k] + coef * acc[k];
  store9(out, V, z, b);
}

// y (+)= a x over n complex entries
template <int = 0>
__global__ void __launch_bounds__(256)
    axpy_c_kernel(double2 *y, const double2 *x, double a, int64_t n, int accumulate) {
  const int64_t i = (int64_t)blockIdx.x * 256 + threadIdx.x;
  if (i >= n) return;
  const double2 v = x[i];
  if (accumulate) {
    const double2 w = y[i];
    y[i] = make_double2(w.x + a * v.x, w.y + a * v.y);
  } else {
    y[i] = make_double2(a * v.x, a * v.y);
  }
}

// Dirac outer products (HISQPullback.jl:461-513):
//   dX_mu(x) = fc eta_mu(x) [dr(x) psi(x+mu)^+ - psi(x) dr(x+mu)^+]
//   dL_mu(x) = lc eta_mu(x) [dr(x) psi(x+3mu)^+ - psi(x) dr(x+3mu)^+]
// dr, psi: three-component FP64 fields; neighbours carry the fermion phase.
template <int = 0>
__global__ void __launch_bounds__(kSmearThreads)
    hisq_outer_product_kernel(double2 *dX, double2 *dL, const Field<PREC_DOUBLE, 3> dr,
                              const Field<PREC_DOUBLE, 3> psi, const Geom g, double fc, double lc) {
  const int s = blockIdx.x * kSmearThreads + threadIdx.x;
  if (s >= g.V) return;
  const int64_t V = g.V;
  int c[4];
  site_coords(g, s, c);
  const int p0 = c[0] + g.eta_off[0], p1 = p0 + c[1] + g.eta_off[1], p2 = p1 + c[2] + g.eta_off[2];
  const double eta[4] = {1.0, (p0 & 1) ? -1.0 : 1.0, (p1 & 1) ? -1.0 : 1.0, (p2 & 1) ? -1.0 : 1.0};
  Cx<double> r0[3], q0[3];
  dr.load(s, r0);
  psi.load(s, q0);
  for (int mu = 0; mu < 4; mu++) {
    for (int which = 0; which < 2; which++) {
      const int d = which == 0 ? 1 : 3;
      int w;
      const int sp = shift_site_any(g, s, c, mu, d, &w);
      Cx<double> rp[3], qp[3];
      dr.load(sp, rp);
      psi.load(sp, qp);
      apply_wraps(g, mu, w, rp);
      apply_wraps(g, mu, w, qp);
      const double coef = (which == 0 ? fc : lc) * eta[mu];
      double2 *out = (which == 0 ? dX : dL) + (size_t)mu * 9 * V;
#pragma unroll
      for (int row = 0; row < 3; row++)
#pragma unroll
        for (int col = 0; col < 3; col++) {
          const Cx<double> v = r0[row] * conj(qp[col]) - q0[row] * conj(rp[col]);
          out[(row + 3 * col) * V + s] = make_double2(coef * v.re, coef * v.im);
        }
    }
  }
}

// Naik pullback (HISQPullback.jl:426-459), gathered at z for direction mu:
//   dW(z) += dL(z) (W(z+mu) W(z+2mu))^+ + W(z-mu)^+ dL(z-mu) W(z+mu)^+
//            + (W(z-2mu) W(z-mu))^+ dL(z-2mu)
template <int = 0>
__global__ void __launch_bounds__(kSmearThreads)
    naik_pullback_kernel(double2 *dW, const double2 *dL, const double2 *W, const Geom g) {
  const int64_t t = (int64_t)blockIdx.x * kSmearThreads + threadIdx.x;
  if (t >= 4 * g.V) return;
  const int mu = (int)(t / g.V);
  const int z = (int)(t - (int64_t)mu * g.V);
  const int64_t V = g.V;
  const double2 *Wm = W + (size_t)mu * 9 * V, *dLm = dL + (size_t)mu * 9 * V;
  const int zp1 = nb_site(g, z, mu, 1), zp2 = nb_site(g, zp1, mu, 1);
  const int zm1 = nb_site(g, z, mu, -1), zm2 = nb_site(g, zm1, mu, -1);
  Cx<double> acc[9], a[9], b[9];
  // dL(z) (W(z+mu) W(z+2mu))^+
  load9(Wm, V, zp1, a);
  load9(Wm, V, zp2, b);
  mat3_mul(a, b, a);
  load9(dLm, V, z, b);
  mat3_mul_adj(b, a, acc);
  // W(z-mu)^+ dL(z-mu) W(z+mu)^+
  load9(Wm, V, zm1, a);
  load9(dLm, V, zm1, b);
  mat3_adj_mul(a, b, a);
  load9(Wm, V, zp1, b);
  mat3_mul_adj(a, b, a);
#pragma unroll
  for (int k = 0; k < 9; k++) acc[k] = acc[k] + a[k];
  // (W(z-2mu) W(z-mu))^+ dL(z-2mu)
  load9(Wm, V, zm2, a);
  load9(Wm, V, zm1, b);
  mat3_mul(a, b, a);
  load9(dLm, V, zm2, b);
  mat3_adj_mul(a, b, a);
#pragma unroll
  for (int k = 0; k < 9; k++) acc[k] = acc[k] + a[k];
  double2 *out = dW + (size_t)mu * 9 * V;
  load9(out, V, z, b);
#pragma unroll
  for (int k = 0; k < 9; k++) b[k] = b[k] + acc[k];
  store9(out, V, z, b);
}

// U(3) projection pullback (HISQPullback.jl:319-424): with W = V H^{-1},
// H = (V^+V)^{1/2}, the cotangent is dV = W X where X solves the Sylvester
// equation H X + X H = C, C = W^+ dW - dW^+ W.  The reference solves it as a
// 9x9 linear system; here it is solved in closed form from the Cayley-
// Hamilton theorem.  For A X - X B = C, sum_k a_k (A^k X - X B^k) =
// sum_k a_k sum_{j<k} A^j C B^{k-1-j}, and with a_k the coefficients of the
// characteristic polynomial of B the X B^k terms cancel.  Taking A = H,
// B = -H: det(z + H) = z^3 + u z^2 + v z + w (u, v, w the elementary
// symmetric functions of the eigenvalues sqrt(g_i) of H, from the
// projection), so
//   M X = v C + u (H C - C H) + H^2 C - H C H + C H^2,
//   M = H^3 + u H^2 + v H + w,
// M Hermitian positive definite (eigenvalues (h_i + h_j)(h_i + h_k) 2 h_i,
// no differences of eigenvalues), inverted by its adjugate.  Everything
// stays in registers (the 9x9 system took a 1.5 KB local-memory frame).
LMB_D void mat3_inverse(const Cx<double> *m, Cx<double> *inv) {
  // column-major m[r + 3c]; inv = adj(m) / det(m)
  auto at = [&](int r, int c) { return m[r + 3 * c]; };
  Cx<double> cof[9];
  for (int r = 0; r < 3; r++)
    for (int c = 0; c < 3; c++) {
      const int r1 = (r + 1) % 3, r2 = (r + 2) % 3, c1 = (c + 1) % 3, c2 = (c + 2) % 3;
      cof[r + 3 * c] = at(r1, c1) * at(r2, c2) - at(r1, c2) * at(r2, c1);
    }
  Cx<double> det = at(0, 0) * cof[0] + at(0, 1) * cof[3] + at(0, 2) * cof[6];
  const double dn = norm2(det);
  const Cx<double> idet = dn > 0 ? Cx<double>(det.re / dn, -det.im / dn) : Cx<double>(0, 0);
  for (int r = 0; r < 3; r++)
    for (int c = 0; c < 3; c++) inv[r + 3 * c] = cof[c + 3 * r] * idet;  // transpose of the cofactors
}

template <int = 0>
__global__ void __launch_bounds__(64)
    u3_pullback_kernel(double2 *dV, const double2 *dW, const double2 *Vall, int64_t n) {
  const int64_t t = (int64_t)blockIdx.x * 64 + threadIdx.x;
  if (t >= 4 * n) return;
  const int mu = (int)(t / n);
  const int s = (int)(t - (int64_t)mu * n);
  Cx<double> Vm[9], W[9], H[9], C[9];
  load9(Vall + (size_t)mu * 9 * n, n, s, Vm);
  double u, v, w;
  {
    U3Inverse r;
    u3_inverse_sqrt(Vm, r);
    mat3_mul(Vm, r.inv, W);
    mat3_mul(r.Q, r.inv, H);  // H = Q Q^{-1/2}
    u = r.u;
    v = r.v;
    w = r.w;
  }
  {
    Cx<double> dWm[9], a[9];
    load9(dW + (size_t)mu * 9 * n, n, s, dWm);
    mat3_adj_mul(W, dWm, C);
    mat3_adj_mul(dWm, W, a);
#pragma unroll
    for (int k = 0; k < 9; k++) C[k] = C[k] - a[k];
  }
  Cx<double> X[9];
  {
    Cx<double> HC[9], CH[9], t1[9], t2[9];
    mat3_mul(H, C, HC);
    mat3_mul(C, H, CH);
    // v C + u (HC - CH) - H C H, then + H (HC) + (CH) H
    mat3_mul(HC, H, t1);  // H C H
#pragma unroll
    for (int k = 0; k < 9; k++) X[k] = v * C[k] + u * (HC[k] - CH[k]) - t1[k];
    mat3_mul(H, HC, t1);  // H^2 C
    mat3_mul(CH, H, t2);  // C H^2
#pragma unroll
    for (int k = 0; k < 9; k++) X[k] = X[k] + t1[k] + t2[k];
    // M = H^3 + u H^2 + v H + w
    mat3_mul(H, H, t1);   // H^2
    mat3_mul(t1, H, t2);  // H^3
#pragma unroll
    for (int k = 0; k < 9; k++) t2[k] = t2[k] + u * t1[k] + v * H[k];
    for (int i = 0; i < 3; i++) t2[i + 3 * i] = t2[i + 3 * i] + Cx<double>(w, 0);
    mat3_inverse(t2, t1);
    mat3_mul(t1, X, HC);  // X = M^{-1} (...)
#pragma unroll
    for (int k = 0; k < 9; k++) X[k] = HC[k];
  }
  Cx<double> a[9], b[9];
  mat3_mul(W, X, a);
  double2 *out = dV + (size_t)mu * 9 * n;
  load9(out, n, s, b);
#pragma unroll
  for (int k = 0; k < 9; k++) b[k] = b[k] + a[k];
  store9(out, n, s, b);
}

// unpack-accumulate 36 gradient planes into four padded (3,3,...) fields
template <typename T>
__global__ void __launch_bounds__(256)
    accumulate_links_kernel(T *U0, T *U1, T *U2, T *U3, const double2 *src, const Geom g, const Padded pd) {
  const int s = blockIdx.x * 256 + threadIdx.x;
  if (s >= g.V) return;
  int c[4];
  site_coords(g, s, c);
  const int64_t ps = padded_site(pd, c) * 9;
  T *U[4] = {U0, U1, U2, U3};
#pragma unroll
  for (int mu = 0; mu < 4; mu++)
#pragma unroll
    for (int k = 0; k < 9; k++) {
      const double2 t = src[(mu * 9 + k) * g.V + s];
      U[mu][ps + k].x += t.x;
      U[mu][ps + k].y += t.y;
    }
}

}  // namespace lmb
