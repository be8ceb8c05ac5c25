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
// H = (V^+V)^{1/2}, solve H X + X H = W^+ dW - dW^+ W (a 9x9 linear system,
// LU with partial pivoting) and accumulate dV += W X.
LMB_D void solve9(Cx<double> (*A)[9], Cx<double> *b) {
  for (int k = 0; k < 9; k++) {
    int piv = k;
    double best = norm2(A[k][k]);
    for (int r = k + 1; r < 9; r++) {
      const double v = norm2(A[r][k]);
      if (v > best) {
        best = v;
        piv = r;
      }
    }
    if (piv != k) {
      for (int c = 0; c < 9; c++) {
        const Cx<double> t = A[k][c];
        A[k][c] = A[piv][c];
        A[piv][c] = t;
      }
      const Cx<double> t = b[k];
      b[k] = b[piv];
      b[piv] = t;
    }
    const double d = norm2(A[k][k]);
    const Cx<double> inv = d > 0 ? Cx<double>(A[k][k].re / d, -A[k][k].im / d) : Cx<double>(0, 0);
    for (int r = k + 1; r < 9; r++) {
      const Cx<double> f = A[r][k] * inv;
      for (int c = k; c < 9; c++) A[r][c] = A[r][c] - f * A[k][c];
      b[r] = b[r] - f * b[k];
    }
  }
  for (int r = 8; r >= 0; r--) {
    Cx<double> v = b[r];
    for (int c = r + 1; c < 9; c++) v = v - A[r][c] * b[c];
    const double d = norm2(A[r][r]);
    b[r] = d > 0 ? v * Cx<double>(A[r][r].re / d, -A[r][r].im / d) : Cx<double>(0, 0);
  }
}

template <int = 0>
__global__ void __launch_bounds__(64)
    u3_pullback_kernel(double2 *dV, const double2 *dW, const double2 *Vall, int64_t n) {
  const int64_t t = (int64_t)blockIdx.x * 64 + threadIdx.x;
  if (t >= 4 * n) return;
  const int mu = (int)(t / n);
  const int s = (int)(t - (int64_t)mu * n);
  Cx<double> Vm[9], W[9], dWm[9], Q[9], Q2[9], inv[9], H[9];
  load9(Vall + (size_t)mu * 9 * n, n, s, Vm);
  load9(dW + (size_t)mu * 9 * n, n, s, dWm);
  // W and H from the projection formulas
  mat3_adj_mul(Vm, Vm, Q);
  mat3_mul(Q, Q, Q2);
  {
    double c0 = 0, trQ2 = 0, trQ3 = 0;
    for (int i = 0; i < 3; i++) {
      c0 += Q[i + 3 * i].re;
      trQ2 += Q2[i + 3 * i].re;
      for (int j = 0; j < 3; j++) trQ3 += (Q2[i + 3 * j] * Q[j + 3 * i]).re;
    }
    const double c1 = trQ2 / 2, c2 = trQ3 / 3;
    double S = c1 / 3 - c0 * c0 / 18;
    double g0, g1, g2;
    if (fabs(S) < 1e-7) {
      g0 = g1 = g2 = c0 / 3;
    } else {
      S = sqrt(fmax(S, 0.0));
      const double R = c2 / 2 - c0 * c1 / 3 + c0 * c0 * c0 / 27;
      double ratio = fmin(1.0, fmax(-1.0, R / (S * S * S)));
      const double theta = acos(ratio);
      const double tpt = 2.0943951023931954923;
      g0 = c0 / 3 + 2 * S * cos(theta / 3 - tpt);
      g1 = c0 / 3 + 2 * S * cos(theta / 3);
      g2 = c0 / 3 + 2 * S * cos(theta / 3 + tpt);
    }
    const double fl = 2.220446049250313e-16;
    g0 = fmax(g0, fl);
    g1 = fmax(g1, fl);
    g2 = fmax(g2, fl);
    const double u = sqrt(g0) + sqrt(g1) + sqrt(g2);
    const double v = sqrt(g0 * g1) + sqrt(g0 * g2) + sqrt(g1 * g2);
    const double w = sqrt(g0 * g1 * g2);
    const double den = w * (u * v - w);
    const double f0 = (-w * (u * u + v) + u * v * v) / den;
    const double f1 = (-w - u * u * u + 2 * u * v) / den;
    const double f2 = u / den;
    for (int k = 0; k < 9; k++) inv[k] = f1 * Q[k] + f2 * Q2[k];
    for (int i = 0; i < 3; i++) inv[i + 3 * i] = inv[i + 3 * i] + Cx<double>(f0, 0);
  }
  mat3_mul(Vm, inv, W);
  mat3_mul(Q, inv, H);
  // skew = W^+ dW - dW^+ W
  Cx<double> a[9], b[9], rhs[9];
  mat3_adj_mul(W, dWm, a);
  mat3_adj_mul(dWm, W, b);
  for (int k = 0; k < 9; k++) rhs[k] = a[k] - b[k];
  // system[eq = r + 3c][unknown]: sum_k H[r,k] X[k,c] + sum_k X[r,k] H[k,c]
  Cx<double> A[9][9];
  for (int i = 0; i < 9; i++)
    for (int j = 0; j < 9; j++) A[i][j] = Cx<double>(0, 0);
  for (int c = 0; c < 3; c++)
    for (int r = 0; r < 3; r++) {
      const int eq = r + 3 * c;
      for (int k = 0; k < 3; k++) {
        A[eq][k + 3 * c] = A[eq][k + 3 * c] + H[r + 3 * k];
        A[eq][r + 3 * k] = A[eq][r + 3 * k] + H[k + 3 * c];
      }
    }
  solve9(A, rhs);
  mat3_mul(W, rhs, a);
  double2 *out = dV + (size_t)mu * 9 * n;
  load9(out, n, s, b);
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
