// lmb_hisq_smear.cuh -- HISQ link smearing on the GPU (FP64).
//
// Fat7 (+ Lepage) in the factorised form of the reference
// (HISQSmearing.jl:768-974): for a link direction mu with transverse axes
// (a, b, c) and the staple transport
//   T_nu(M)(x) = U_nu(x) M(x+nu) U_nu(x+mu)^+ + U_nu(x-nu)^+ M(x-nu) U_nu(x-nu+mu),
//   S3_nu = T_nu(U_mu),   S5_a = T_b(S3_c) + T_c(S3_b),
//   V_mu = c1 U_mu + c3 sum S3 + c5 sum S5 + c7 sum_a T_a(S5_a) + cL Lepage,
// which sums exactly the 6 three-link, 24 five-link and 48 seven-link paths of
// the direct path lists (HISQSmearing.jl:490-566).  On one GPU every
// intermediate field is defined on the whole periodic lattice, so no enlarged
// domains are needed.  Lepage paths (nu,nu,mu,-nu,-nu), (-nu,-nu,mu,nu,nu)
// are evaluated directly.  U(3) projection W = V (V^+V)^{-1/2} with the
// trigonometric eigenvalues and Cayley-Hamilton coefficients
// (HISQFullSmearing.jl:1-77); Naik links L_mu(x) = W_mu(x) W_mu(x+mu) W_mu(x+2mu)
// (HISQFullSmearing.jl:136-195).
//
// Link planes: (mu*9 + r + 3c) * V + s (double2), as the link caches.
// Single-direction fields (staples): (r + 3c) * V + s.
#pragma once
#include "lmb_pack.cuh"

namespace lmb {

constexpr int kSmearThreads = 128;

LMB_D void load9(const double2 *F, int64_t V, int s, Cx<double> *m) {
#pragma unroll
  for (int k = 0; k < 9; k++) {
    const double2 t = F[k * V + s];
    m[k] = Cx<double>(t.x, t.y);
  }
}
LMB_D void store9(double2 *F, int64_t V, int s, const Cx<double> *m) {
#pragma unroll
  for (int k = 0; k < 9; k++) F[k * V + s] = make_double2(m[k].re, m[k].im);
}
// c = a * b^+
LMB_D void mat3_mul_adj(const Cx<double> *a, const Cx<double> *b, Cx<double> *c) {
  Cx<double> t[9];
#pragma unroll
  for (int r = 0; r < 3; r++)
#pragma unroll
    for (int col = 0; col < 3; col++) {
      Cx<double> v = a[r] * conj(b[col]);
      v = cfma_conj(b[col + 3], a[r + 3], v);
      v = cfma_conj(b[col + 6], a[r + 6], v);
      t[r + 3 * col] = v;
    }
#pragma unroll
  for (int k = 0; k < 9; k++) c[k] = t[k];
}
// c = a^+ * b
LMB_D void mat3_adj_mul(const Cx<double> *a, const Cx<double> *b, Cx<double> *c) {
  Cx<double> t[9];
#pragma unroll
  for (int r = 0; r < 3; r++)
#pragma unroll
    for (int col = 0; col < 3; col++) {
      Cx<double> v = conj(a[3 * r]) * b[3 * col];
      v = cfma_conj(a[3 * r + 1], b[1 + 3 * col], v);
      v = cfma_conj(a[3 * r + 2], b[2 + 3 * col], v);
      t[r + 3 * col] = v;
    }
#pragma unroll
  for (int k = 0; k < 9; k++) c[k] = t[k];
}

LMB_D int nb_site(const Geom &g, int s, int mu, int d) {
  int c[4], w;
  site_coords(g, s, c);
  return d > 0 ? fwd_site(g, s, c, mu, d, &w) : bwd_site(g, s, c, mu, -d, &w);
}

// out (+)= coef * T_nu(M) for link direction mu; signs: 1 forward, 2 backward, 3 both
template <int = 0>
__global__ void __launch_bounds__(kSmearThreads)
    staple_transport_kernel(double2 *out, const double2 *M, const double2 *U, const Geom g, int mu, int nu,
                            int signs, int accumulate, double coef) {
  const int s = blockIdx.x * kSmearThreads + threadIdx.x;
  if (s >= g.V) return;
  const int64_t V = g.V;
  Cx<double> acc[9], a[9], b[9], m[9];
#pragma unroll
  for (int k = 0; k < 9; k++) acc[k] = Cx<double>(0, 0);
  if (signs & 1) {  // U_nu(x) M(x+nu) U_nu(x+mu)^+
    const int xpn = nb_site(g, s, nu, 1), xpm = nb_site(g, s, mu, 1);
    load9(U + (size_t)nu * 9 * V, V, s, a);
    load9(M, V, xpn, m);
    mat3_mul(a, m, a);
    load9(U + (size_t)nu * 9 * V, V, xpm, b);
    mat3_mul_adj(a, b, a);
#pragma unroll
    for (int k = 0; k < 9; k++) acc[k] = acc[k] + a[k];
  }
  if (signs & 2) {  // U_nu(x-nu)^+ M(x-nu) U_nu(x-nu+mu)
    const int xmn = nb_site(g, s, nu, -1);
    const int xmn_pm = nb_site(g, xmn, mu, 1);
    load9(U + (size_t)nu * 9 * V, V, xmn, a);
    load9(M, V, xmn, m);
    mat3_adj_mul(a, m, a);
    load9(U + (size_t)nu * 9 * V, V, xmn_pm, b);
    mat3_mul(a, b, a);
#pragma unroll
    for (int k = 0; k < 9; k++) acc[k] = acc[k] + a[k];
  }
  if (accumulate) {
    load9(out, V, s, m);
#pragma unroll
    for (int k = 0; k < 9; k++) acc[k] = m[k] + coef * acc[k];
  } else {
#pragma unroll
    for (int k = 0; k < 9; k++) acc[k] = coef * acc[k];
  }
  store9(out, V, s, acc);
}

// V_mu = c1 U_mu + c3 (S3_a+S3_b+S3_c) + c5 (S5_a+S5_b+S5_c); fields single-direction
template <int = 0>
__global__ void __launch_bounds__(256)
    fat7_combine_kernel(double2 *Vmu, const double2 *Umu, const double2 *s3a, const double2 *s3b,
                        const double2 *s3c, const double2 *s5a, const double2 *s5b, const double2 *s5c, int64_t V,
                        double c1, double c3, double c5) {
  const int64_t i = (int64_t)blockIdx.x * 256 + threadIdx.x;
  if (i >= 9 * V) return;
  const double2 u = Umu[i], a = s3a[i], b = s3b[i], c = s3c[i], d = s5a[i], e = s5b[i], f = s5c[i];
  Vmu[i] = make_double2(c1 * u.x + c3 * (a.x + b.x + c.x) + c5 * (d.x + e.x + f.x),
                        c1 * u.y + c3 * (a.y + b.y + c.y) + c5 * (d.y + e.y + f.y));
}

// product of links along a signed path (1-based directions) starting at s
LMB_D void path_product_dev(const double2 *U, const Geom &g, int s, const int *path, int len, Cx<double> *out) {
  const int64_t V = g.V;
  Cx<double> m[9];
#pragma unroll
  for (int k = 0; k < 9; k++) out[k] = Cx<double>((k % 4) == 0 ? 1.0 : 0.0, 0);
  int site = s;
  for (int i = 0; i < len; i++) {
    const int d = path[i];
    const int axis = (d > 0 ? d : -d) - 1;
    if (d > 0) {
      load9(U + (size_t)axis * 9 * V, V, site, m);
      mat3_mul(out, m, out);
      site = nb_site(g, site, axis, 1);
    } else {
      site = nb_site(g, site, axis, -1);
      load9(U + (size_t)axis * 9 * V, V, site, m);
      mat3_mul_adj(out, m, out);
    }
  }
}

// V_mu += cL sum_nu [path(nu,nu,mu,-nu,-nu) + path(-nu,-nu,mu,nu,nu)]
template <int = 0>
__global__ void __launch_bounds__(kSmearThreads)
    lepage_kernel(double2 *Vall, const double2 *U, const Geom g, double cL) {
  const int64_t tid = (int64_t)blockIdx.x * kSmearThreads + threadIdx.x;
  if (tid >= 4 * g.V) return;
  const int mu = (int)(tid / g.V);
  const int s = (int)(tid - (int64_t)mu * g.V);
  Cx<double> acc[9], p[9];
#pragma unroll
  for (int k = 0; k < 9; k++) acc[k] = Cx<double>(0, 0);
  for (int nu = 1; nu <= 4; nu++) {
    if (nu == mu + 1) continue;
    const int p1[5] = {nu, nu, mu + 1, -nu, -nu}, p2[5] = {-nu, -nu, mu + 1, nu, nu};
    path_product_dev(U, g, s, p1, 5, p);
#pragma unroll
    for (int k = 0; k < 9; k++) acc[k] = acc[k] + p[k];
    path_product_dev(U, g, s, p2, 5, p);
#pragma unroll
    for (int k = 0; k < 9; k++) acc[k] = acc[k] + p[k];
  }
  double2 *Vm = Vall + (size_t)mu * 9 * g.V;
  Cx<double> v[9];
  load9(Vm, g.V, s, v);
#pragma unroll
  for (int k = 0; k < 9; k++) v[k] = v[k] + cL * acc[k];
  store9(Vm, g.V, s, v);
}

// (V^+V)^{-1/2} for the U(3) projection (HISQFullSmearing.jl:1-77):
// Q = V^+V, its eigenvalues g0, g1, g2 from the trigonometric solution of
// the characteristic cubic (coefficients from traces of Q, Q^2, Q^3), each
// floored at the machine epsilon, and Q^{-1/2} = f0 + f1 Q + f2 Q^2 by
// Cayley-Hamilton, f_k symmetric functions of sqrt(g_i).  Returns Q, Q^2,
// Q^{-1/2} and the elementary symmetric functions u, v, w of the sqrt(g_i)
// (the U(3) pullback needs them).  The smearing and the force share it, so
// both use the same branch thresholds.
struct U3Inverse {
  Cx<double> Q[9], Q2[9], inv[9];
  double u, v, w;
};
LMB_D void u3_inverse_sqrt(const Cx<double> *Vm, U3Inverse &r) {
  mat3_adj_mul(Vm, Vm, r.Q);
  mat3_mul(r.Q, r.Q, r.Q2);
  double c0 = 0, trQ2 = 0, trQ3 = 0;
  for (int i = 0; i < 3; i++) {
    c0 += r.Q[i + 3 * i].re;
    trQ2 += r.Q2[i + 3 * i].re;
    for (int j = 0; j < 3; j++) trQ3 += (r.Q2[i + 3 * j] * r.Q[j + 3 * i]).re;
  }
  const double c1 = trQ2 / 2, c2 = trQ3 / 3;
  double S = c1 / 3 - c0 * c0 / 18;
  double g0, g1, g2;
  if (fabs(S) < 1e-7) {
    g0 = g1 = g2 = c0 / 3;
  } else {
    S = sqrt(fmax(S, 0.0));
    const double R = c2 / 2 - c0 * c1 / 3 + c0 * c0 * c0 / 27;
    double ratio = R / (S * S * S);
    ratio = fmin(1.0, fmax(-1.0, ratio));
    const double theta = acos(ratio);
    const double tpt = 2.0943951023931954923;  // 2 pi / 3
    const double center = c0 / 3, amp = 2 * S;
    g0 = center + amp * cos(theta / 3 - tpt);
    g1 = center + amp * cos(theta / 3);
    g2 = center + amp * cos(theta / 3 + tpt);
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
#pragma unroll
  for (int k = 0; k < 9; k++) r.inv[k] = f1 * r.Q[k] + f2 * r.Q2[k];
  for (int i = 0; i < 3; i++) r.inv[i + 3 * i] = r.inv[i + 3 * i] + Cx<double>(f0, 0);
  r.u = u;
  r.v = v;
  r.w = w;
}

// W = V (V^+V)^{-1/2}
LMB_D void u3_project(const Cx<double> *Vm, Cx<double> *W) {
  U3Inverse r;
  u3_inverse_sqrt(Vm, r);
  mat3_mul(Vm, r.inv, W);
}

template <int = 0>
__global__ void __launch_bounds__(kSmearThreads)
    u3_project_kernel(double2 *W, const double2 *Vall, int64_t n) {
  const int64_t t = (int64_t)blockIdx.x * kSmearThreads + threadIdx.x;
  if (t >= 4 * n) return;
  const int mu = (int)(t / n);
  const int s = (int)(t - (int64_t)mu * n);
  Cx<double> v[9], w[9];
  load9(Vall + (size_t)mu * 9 * n, n, s, v);
  u3_project(v, w);
  store9(W + (size_t)mu * 9 * n, n, s, w);
}

template <int = 0>
__global__ void __launch_bounds__(kSmearThreads)
    naik_kernel(double2 *Lall, const double2 *W, const Geom g) {
  const int64_t t = (int64_t)blockIdx.x * kSmearThreads + threadIdx.x;
  if (t >= 4 * g.V) return;
  const int mu = (int)(t / g.V);
  const int s = (int)(t - (int64_t)mu * g.V);
  const int path[3] = {mu + 1, mu + 1, mu + 1};
  Cx<double> p[9];
  path_product_dev(W, g, s, path, 3, p);
  store9(Lall + (size_t)mu * 9 * g.V, g.V, s, p);
}

// unpack 36 link planes to four padded (3,3,...) fields
template <typename TOUT>
__global__ void __launch_bounds__(256)
    unpack_links_kernel(TOUT *U0, TOUT *U1, TOUT *U2, TOUT *U3, const double2 *src, const Geom g,
                        const Padded pd) {
  const int s = blockIdx.x * 256 + threadIdx.x;
  if (s >= g.V) return;
  int c[4];
  site_coords(g, s, c);
  const int64_t ps = padded_site(pd, c) * 9;
  TOUT *U[4] = {U0, U1, U2, U3};
#pragma unroll
  for (int mu = 0; mu < 4; mu++) {
    if (!U[mu]) continue;
#pragma unroll
    for (int k = 0; k < 9; k++) {
      const double2 t = src[(mu * 9 + k) * g.V + s];
      U[mu][ps + k].x = t.x;
      U[mu][ps + k].y = t.y;
    }
  }
}

}  // namespace lmb
