/*
 * lmb_oracle.c -- FP64 CPU restatement of the LatticeMatrices.jl v1.1.6
 * Dirac-operator / D'D-CG path.  TEST INFRASTRUCTURE: used only as the checker
 * by tests/, __graft_entry__.smoke() and as the timed CPU baseline in bench.py.
 * The product library never links or calls this file.
 *
 * Every routine names the reference file:line whose arithmetic it restates.
 * Paths are relative to the LatticeMatrices.jl source tree.
 */
#include "lmb_oracle.h"

#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef double complex cplx;

int orc_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

void orc_set_num_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

/* ---------------------------------------------------------------------------
 * geometry helpers (Latticeindices.jl:2-33 delinearize, x fastest)
 * ------------------------------------------------------------------------- */
static inline int64_t volume_of(const int *L) {
  return (int64_t)L[0] * L[1] * L[2] * L[3];
}

static inline void coords_of(const int *L, int64_t s, int *c) {
  c[0] = (int)(s % L[0]);
  s /= L[0];
  c[1] = (int)(s % L[1]);
  s /= L[1];
  c[2] = (int)(s % L[2]);
  c[3] = (int)(s / L[2]);
}

static inline int64_t site_of(const int *L, const int *c) {
  return c[0] + (int64_t)L[0] * (c[1] + (int64_t)L[1] * (c[2] + (int64_t)L[2] * c[3]));
}

/* Neighbour at distance `amount` along mu.  *wraps counts lattice-edge
 * crossings (floor division), as in the dense test oracles
 * (test/wilson_clover.jl:5-10) and the halo fill rule
 * (LatticeMatrices_core.jl:707-723): forward wrap * phase, backward * 1/phase. */
static inline int64_t shifted_site(const int *L, const int *c, int mu,
                                   int amount, int *wraps) {
  int cc[4] = {c[0], c[1], c[2], c[3]};
  int raw = c[mu] + amount;
  int w = 0;
  while (raw >= L[mu]) { raw -= L[mu]; w++; }
  while (raw < 0) { raw += L[mu]; w--; }
  cc[mu] = raw;
  if (wraps) *wraps = w;
  return site_of(L, cc);
}

static inline cplx phase_power(const double *phases, int mu, int wraps) {
  cplx ph = phases[2 * mu] + I * phases[2 * mu + 1];
  cplx f = 1.0;
  if (wraps > 0)
    for (int k = 0; k < wraps; k++) f *= ph;
  else if (wraps < 0)
    for (int k = 0; k < -wraps; k++) f /= ph;
  return f;
}

/* ---------------------------------------------------------------------------
 * chiral gamma matrices (Operators.jl:44-66) and (1 +/- gamma_mu)
 * (Operators.jl:71-134: mul_op(Onegamma{pm,mu}) = x + pm * gamma_mu x).
 * ------------------------------------------------------------------------- */
static const double gamma_re[4][4][4] = {
    {{0, 0, 0, 0}, {0, 0, 0, 0}, {0, 0, 0, 0}, {0, 0, 0, 0}},
    {{0, 0, 0, -1}, {0, 0, 1, 0}, {0, 1, 0, 0}, {-1, 0, 0, 0}},
    {{0, 0, 0, 0}, {0, 0, 0, 0}, {0, 0, 0, 0}, {0, 0, 0, 0}},
    {{0, 0, -1, 0}, {0, 0, 0, -1}, {-1, 0, 0, 0}, {0, -1, 0, 0}}};
static const double gamma_im[4][4][4] = {
    {{0, 0, 0, -1}, {0, 0, -1, 0}, {0, 1, 0, 0}, {1, 0, 0, 0}},
    {{0, 0, 0, 0}, {0, 0, 0, 0}, {0, 0, 0, 0}, {0, 0, 0, 0}},
    {{0, 0, -1, 0}, {0, 0, 0, 1}, {1, 0, 0, 0}, {0, -1, 0, 0}},
    {{0, 0, 0, 0}, {0, 0, 0, 0}, {0, 0, 0, 0}, {0, 0, 0, 0}}};

static inline void one_pm_gamma(int pm, int mu, const cplx *x, cplx *v) {
  for (int a = 0; a < 4; a++) {
    cplx g = 0;
    for (int b = 0; b < 4; b++)
      g += (gamma_re[mu][a][b] + I * gamma_im[mu][a][b]) * x[b];
    v[a] = x[a] + pm * g;
  }
}

/* ---------------------------------------------------------------------------
 * Wilson operator (WilsonDiracOperator.jl:57-147 generic-NC kernel,
 * adjoint :420-511, Donly :522-631):
 *   D psi = psi - kappa sum_mu [U_mu(x)(1 - g_mu) psi(x+mu)
 *                               + U_mu(x-mu)^+ (1 + g_mu) psi(x-mu)]
 *   D^+ swaps the projector signs.
 * `scale_hop` multiplies the hopping sum; `copy_input` adds psi(x).
 * ------------------------------------------------------------------------- */
static void wilson_generic(const int *L, const double *phases, int nc,
                           double scale_hop, int copy_input, int dagger,
                           const double *const *Ud, const double *psid,
                           double *outd) {
  const int64_t V = volume_of(L);
  const cplx *psi = (const cplx *)psid;
  cplx *out = (cplx *)outd;
  const int fwd_pm = dagger ? +1 : -1;
  const int bwd_pm = -fwd_pm;
#pragma omp parallel for schedule(static)
  for (int64_t s = 0; s < V; s++) {
    int c[4];
    coords_of(L, s, c);
    cplx acc[64];
    for (int k = 0; k < nc * 4; k++) acc[k] = 0;
    for (int mu = 0; mu < 4; mu++) {
      const cplx *U = (const cplx *)Ud[mu];
      int wp, wm;
      int64_t sp = shifted_site(L, c, mu, +1, &wp);
      int64_t sm = shifted_site(L, c, mu, -1, &wm);
      cplx fp = phase_power(phases, mu, wp);
      cplx fm = phase_power(phases, mu, wm);
      for (int jc = 0; jc < nc; jc++) {
        cplx xp[4], xm[4], vp[4], vm[4];
        for (int a = 0; a < 4; a++) {
          xp[a] = fp * psi[jc + nc * (a + 4 * sp)];
          xm[a] = fm * psi[jc + nc * (a + 4 * sm)];
        }
        one_pm_gamma(fwd_pm, mu, xp, vp);
        one_pm_gamma(bwd_pm, mu, xm, vm);
        for (int ic = 0; ic < nc; ic++) {
          cplx uf = U[ic + nc * (jc + nc * s)];
          cplx ub = conj(U[jc + nc * (ic + nc * sm)]);
          for (int a = 0; a < 4; a++) acc[ic + nc * a] += uf * vp[a] + ub * vm[a];
        }
      }
    }
    for (int a = 0; a < 4; a++)
      for (int ic = 0; ic < nc; ic++) {
        int64_t k = ic + nc * (a + 4 * s);
        out[k] = (copy_input ? psi[k] : 0) + scale_hop * acc[ic + nc * a];
      }
  }
}

void orc_wilson(const int *L, const double *phases, int nc, double kappa,
                int dagger, const double *const *U, const double *psi,
                double *out) {
  wilson_generic(L, phases, nc, -kappa, 1, dagger, U, psi, out);
}

void orc_wilson_donly(const int *L, const double *phases, int nc, int dagger,
                      const double *const *U, const double *psi, double *out) {
  wilson_generic(L, phases, nc, 0.5, 0, dagger, U, psi, out);
}

/* ---------------------------------------------------------------------------
 * Generalised domain-wall operator (DiracOperators_5D.jl:48-115, 226-268,
 * 731-857; Mobius = a 1, b (b+c)/2, c (b-c)/2):
 *   D5 psi = A [psi - F psi + D_W (B psi + C F psi)],
 *   D5^+ psi = q - F^+ q + B D_W^+ q + F^+ (C D_W^+ q),  q = A psi,
 * with A, B, C diagonal in the fifth coordinate s, the 4D Wilson kernel
 *   D_W psi = (4 + M) psi - 1/2 sum_mu [U(1 - g)psi(x+mu) + U^+(1 + g)psi(x-mu)]
 * on every s-slice (fermion phases in x..t), and
 *   (F psi)_s   : spins 1,2 from s-1 (x (-mass) at s = 1), spins 3,4 from s+1
 *                 (x (-mass) at s = L5);
 *   (F^+ psi)_s : spins 1,2 from s+1 (x (-mass) at s = L5), spins 3,4 from s-1
 *                 (x (-mass) at s = 1).
 * Fields: (nc, 4, X, Y, Z, T, L5) column-major, slices contiguous.
 * ------------------------------------------------------------------------- */
static void dw_F(const int *L, int L5, int nc, double mass, int adj, const cplx *in, cplx *out) {
  const int64_t V4 = volume_of(L), n4 = (int64_t)nc * 4 * V4;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n4 * L5; i++) {
    const int s = (int)(i / n4);
    const int64_t r = i - (int64_t)s * n4;
    const int spin = (int)((r / nc) % 4);
    const int low = spin < 2;
    int src;
    double coef = 1.0;
    if (!adj) {
      src = low ? (s + L5 - 1) % L5 : (s + 1) % L5;
      if (low && s == 0) coef = -mass;
      if (!low && s == L5 - 1) coef = -mass;
    } else {
      src = low ? (s + 1) % L5 : (s + L5 - 1) % L5;
      if (low && s == L5 - 1) coef = -mass;
      if (!low && s == 0) coef = -mass;
    }
    out[i] = coef * in[r + (int64_t)src * n4];
  }
}

static void dw_wilson(const int *L, int L5, const double *phases, int nc, double M, int dagger,
                      const double *const *U, const cplx *in, cplx *out) {
  const int64_t n4 = (int64_t)nc * 4 * volume_of(L);
  for (int s = 0; s < L5; s++) {
    wilson_generic(L, phases, nc, -0.5, 0, dagger, U, (const double *)(in + s * n4),
                   (double *)(out + s * n4));
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n4; i++) out[s * n4 + i] += (4.0 + M) * in[s * n4 + i];
  }
}

void orc_domainwall(const int *L, int L5, const double *phases, int nc, double mass, double M,
                    const double *a, const double *b, const double *c, int dagger,
                    const double *const *U, const double *psid, double *outd) {
  const int64_t n4 = (int64_t)nc * 4 * volume_of(L), n = n4 * L5;
  const cplx *psi = (const cplx *)psid;
  cplx *out = (cplx *)outd;
  cplx *t1 = (cplx *)malloc(sizeof(cplx) * n), *t2 = (cplx *)malloc(sizeof(cplx) * n);
  cplx *t3 = (cplx *)malloc(sizeof(cplx) * n);
  if (!dagger) {
    dw_F(L, L5, nc, mass, 0, psi, t1);  /* F psi */
    for (int64_t i = 0; i < n; i++) {
      const int s = (int)(i / n4);
      t2[i] = b[s] * psi[i] + c[s] * t1[i];  /* B psi + C F psi */
    }
    dw_wilson(L, L5, phases, nc, M, 0, U, t2, t3);
    for (int64_t i = 0; i < n; i++) {
      const int s = (int)(i / n4);
      out[i] = a[s] * (psi[i] - t1[i] + t3[i]);
    }
  } else {
    for (int64_t i = 0; i < n; i++) t1[i] = a[i / n4] * psi[i];  /* q */
    dw_wilson(L, L5, phases, nc, M, 1, U, t1, t2);                /* D_W^+ q */
    dw_F(L, L5, nc, mass, 1, t1, t3);                             /* F^+ q */
    for (int64_t i = 0; i < n; i++) out[i] = t1[i] - t3[i] + b[i / n4] * t2[i];
    for (int64_t i = 0; i < n; i++) t2[i] = c[i / n4] * t2[i];    /* C D_W^+ q */
    dw_F(L, L5, nc, mass, 1, t2, t3);
    for (int64_t i = 0; i < n; i++) out[i] += t3[i];
  }
  free(t1);
  free(t2);
  free(t3);
}

/* ---------------------------------------------------------------------------
 * small dense matrix helpers (column-major NC x NC, as the reference stores
 * U[row, col, site])
 * ------------------------------------------------------------------------- */
static inline void mat_load(int nc, const cplx *U, int64_t s, int dag,
                            cplx *m) {
  for (int r = 0; r < nc; r++)
    for (int col = 0; col < nc; col++)
      m[r + nc * col] = dag ? conj(U[col + nc * (r + nc * s)])
                            : U[r + nc * (col + nc * s)];
}

static inline void mat_mul(int nc, const cplx *a, const cplx *b, cplx *c) {
  cplx t[64];
  for (int r = 0; r < nc; r++)
    for (int col = 0; col < nc; col++) {
      cplx v = 0;
      for (int k = 0; k < nc; k++) v += a[r + nc * k] * b[k + nc * col];
      t[r + nc * col] = v;
    }
  memcpy(c, t, sizeof(cplx) * nc * nc);
}

/* ---------------------------------------------------------------------------
 * Clover field strength (WilsonDiracCloverOperator.jl:58-111, 186-226):
 *   F_mu_nu = (Q - Q^+)/8 with Q the sum of the four counter-clockwise leaves.
 * Plane order (12, 13, 14, 23, 24, 34) (WilsonDiracCloverOperator.jl:1).
 * ------------------------------------------------------------------------- */
static const int plane_mu[6] = {0, 0, 0, 1, 1, 2};
static const int plane_nu[6] = {1, 2, 3, 2, 3, 3};

void orc_clover_field_strength(const int *L, int nc, const double *const *Ud,
                               double *const *Fd) {
  const int64_t V = volume_of(L);
  for (int plane = 0; plane < 6; plane++) {
    const int mu = plane_mu[plane], nu = plane_nu[plane];
    const cplx *Um = (const cplx *)Ud[mu];
    const cplx *Un = (const cplx *)Ud[nu];
    cplx *F = (cplx *)Fd[plane];
#pragma omp parallel for schedule(static)
    for (int64_t s = 0; s < V; s++) {
      int c[4];
      coords_of(L, s, c);
      int cpm[4], cpn[4], cmm[4], cmn[4];
      memcpy(cpm, c, sizeof c); cpm[mu] = (c[mu] + 1) % L[mu];
      memcpy(cpn, c, sizeof c); cpn[nu] = (c[nu] + 1) % L[nu];
      memcpy(cmm, c, sizeof c); cmm[mu] = (c[mu] - 1 + L[mu]) % L[mu];
      memcpy(cmn, c, sizeof c); cmn[nu] = (c[nu] - 1 + L[nu]) % L[nu];
      int cpn_mm[4], cmm_mn[4], cpm_mn[4];
      memcpy(cpn_mm, cpn, sizeof c); cpn_mm[mu] = (c[mu] - 1 + L[mu]) % L[mu];
      memcpy(cmm_mn, cmm, sizeof c); cmm_mn[nu] = (c[nu] - 1 + L[nu]) % L[nu];
      memcpy(cpm_mn, cpm, sizeof c); cpm_mn[nu] = (c[nu] - 1 + L[nu]) % L[nu];
      int64_t x = s, xpmu = site_of(L, cpm), xpnu = site_of(L, cpn);
      int64_t xmmu = site_of(L, cmm), xmnu = site_of(L, cmn);
      int64_t xpnu_mmu = site_of(L, cpn_mm), xmmu_mnu = site_of(L, cmm_mn);
      int64_t xpmu_mnu = site_of(L, cpm_mn);
      cplx q[64], a[64], b[64];
      for (int k = 0; k < nc * nc; k++) q[k] = 0;
      /* +mu, +nu, -mu, -nu */
      mat_load(nc, Um, x, 0, a);
      mat_load(nc, Un, xpmu, 0, b); mat_mul(nc, a, b, a);
      mat_load(nc, Um, xpnu, 1, b); mat_mul(nc, a, b, a);
      mat_load(nc, Un, x, 1, b); mat_mul(nc, a, b, a);
      for (int k = 0; k < nc * nc; k++) q[k] += a[k];
      /* +nu, -mu, -nu, +mu */
      mat_load(nc, Un, x, 0, a);
      mat_load(nc, Um, xpnu_mmu, 1, b); mat_mul(nc, a, b, a);
      mat_load(nc, Un, xmmu, 1, b); mat_mul(nc, a, b, a);
      mat_load(nc, Um, xmmu, 0, b); mat_mul(nc, a, b, a);
      for (int k = 0; k < nc * nc; k++) q[k] += a[k];
      /* -mu, -nu, +mu, +nu */
      mat_load(nc, Um, xmmu, 1, a);
      mat_load(nc, Un, xmmu_mnu, 1, b); mat_mul(nc, a, b, a);
      mat_load(nc, Um, xmmu_mnu, 0, b); mat_mul(nc, a, b, a);
      mat_load(nc, Un, xmnu, 0, b); mat_mul(nc, a, b, a);
      for (int k = 0; k < nc * nc; k++) q[k] += a[k];
      /* -nu, +mu, +nu, -mu */
      mat_load(nc, Un, xmnu, 1, a);
      mat_load(nc, Um, xmnu, 0, b); mat_mul(nc, a, b, a);
      mat_load(nc, Un, xpmu_mnu, 0, b); mat_mul(nc, a, b, a);
      mat_load(nc, Um, x, 1, b); mat_mul(nc, a, b, a);
      for (int k = 0; k < nc * nc; k++) q[k] += a[k];
      for (int r = 0; r < nc; r++)
        for (int col = 0; col < nc; col++)
          F[r + nc * (col + nc * s)] =
              0.125 * (q[r + nc * col] - conj(q[col + nc * r]));
    }
  }
}

/* Clover term (WilsonDiracCloverOperator.jl:481-525, kernel_add_clover_term!):
 * out += coefficient * sum_{mu<nu} (gamma_mu gamma_nu) F_mu_nu psi, written
 * in the block form the reference kernel uses. */
void orc_add_clover_term(const int *L, int nc, double coefficient,
                         const double *const *Fd, const double *psid,
                         double *outd) {
  const int64_t V = volume_of(L);
  const cplx *F12 = (const cplx *)Fd[0], *F13 = (const cplx *)Fd[1],
             *F14 = (const cplx *)Fd[2], *F23 = (const cplx *)Fd[3],
             *F24 = (const cplx *)Fd[4], *F34 = (const cplx *)Fd[5];
  const cplx *psi = (const cplx *)psid;
  cplx *out = (cplx *)outd;
#pragma omp parallel for schedule(static)
  for (int64_t s = 0; s < V; s++) {
    for (int color = 0; color < nc; color++) {
      cplx v1 = 0, v2 = 0, v3 = 0, v4 = 0;
      for (int ic = 0; ic < nc; ic++) {
        int64_t k = color + nc * (ic + nc * s);
        cplx f12 = F12[k], f13 = F13[k], f14 = F14[k], f23 = F23[k],
             f24 = F24[k], f34 = F34[k];
        cplx dp = I * (f12 + f34), dm = I * (f12 - f34);
        cplx op = I * (f14 + f23), om = I * (f23 - f14);
        cplx p1 = psi[ic + nc * (0 + 4 * s)], p2 = psi[ic + nc * (1 + 4 * s)];
        cplx p3 = psi[ic + nc * (2 + 4 * s)], p4 = psi[ic + nc * (3 + 4 * s)];
        v1 += dp * p1 + (-f13 + op + f24) * p2;
        v2 += -dp * p2 + (f13 + op - f24) * p1;
        v3 += dm * p3 + (-f13 + om - f24) * p4;
        v4 += -dm * p4 + (f13 + om + f24) * p3;
      }
      out[color + nc * (0 + 4 * s)] += coefficient * v1;
      out[color + nc * (1 + 4 * s)] += coefficient * v2;
      out[color + nc * (2 + 4 * s)] += coefficient * v3;
      out[color + nc * (3 + 4 * s)] += coefficient * v4;
    }
  }
}

/* Fused Wilson + clover (WilsonDiracCloverOperator.jl:537-601): the clover
 * term is Hermitian, so D^+ uses the Wilson adjoint plus the same term. */
void orc_wilson_clover(const int *L, const double *phases, int nc,
                       double kappa, double csw, int dagger,
                       const double *const *U, const double *const *F,
                       const double *psi, double *out) {
  wilson_generic(L, phases, nc, -kappa, 1, dagger, U, psi, out);
  orc_add_clover_term(L, nc, -kappa * csw, F, psi, out);
}

/* ---------------------------------------------------------------------------
 * Staggered (StaggeredDiracOperator.jl:1-17, 94-198; eta from zero-based
 * global coordinates staggered.jl:43-57):
 *   D psi = m psi + (1/2) sum_mu eta_mu(x)[U_mu(x) psi(x+mu) - U_mu(x-mu)^+ psi(x-mu)]
 *   D^+ flips the sign of the hopping term (StaggeredDiracOperator.jl:174-175).
 * ------------------------------------------------------------------------- */
static inline int staggered_eta(const int *c, const int *off, int mu) {
  int sum = 0;
  for (int nu = 0; nu < mu; nu++) sum += c[nu] + off[nu];
  return (sum & 1) ? -1 : 1;
}

static void staggered_hop(const int *L, const double *phases, const int *off,
                          int nc, int distance, double coefficient,
                          const double *const *Ud, const double *psid,
                          cplx *out) {
  const int64_t V = volume_of(L);
  const cplx *psi = (const cplx *)psid;
#pragma omp parallel for schedule(static)
  for (int64_t s = 0; s < V; s++) {
    int c[4];
    coords_of(L, s, c);
    for (int mu = 0; mu < 4; mu++) {
      const cplx *U = (const cplx *)Ud[mu];
      int wp, wm;
      int64_t sp = shifted_site(L, c, mu, distance, &wp);
      int64_t sm = shifted_site(L, c, mu, -distance, &wm);
      cplx fp = phase_power(phases, mu, wp), fm = phase_power(phases, mu, wm);
      double eta = staggered_eta(c, off, mu);
      for (int oc = 0; oc < nc; oc++) {
        cplx fwd = 0, bwd = 0;
        for (int ic = 0; ic < nc; ic++) {
          fwd += U[oc + nc * (ic + nc * s)] * (fp * psi[ic + nc * sp]);
          bwd += conj(U[ic + nc * (oc + nc * sm)]) * (fm * psi[ic + nc * sm]);
        }
        out[oc + nc * s] += coefficient * eta * (fwd - bwd);
      }
    }
  }
}

void orc_staggered(const int *L, const double *phases, const int *eta_offset,
                   int nc, double mass, int dagger, const double *const *U,
                   const double *psid, double *outd) {
  const int64_t V = volume_of(L);
  const cplx *psi = (const cplx *)psid;
  cplx *out = (cplx *)outd;
  int zero_off[4] = {0, 0, 0, 0};
  const int *off = eta_offset ? eta_offset : zero_off;
  for (int64_t k = 0; k < V * nc; k++) out[k] = mass * psi[k];
  staggered_hop(L, phases, off, nc, 1, dagger ? -0.5 : 0.5, U, psid, out);
}

/* HISQ (HISQDiracOperator.jl:55-72 docstring, 202-264 kernel, 350-357
 * coefficients): fat hop +-1 with 1/2, Naik hop +-3 with -(1+eps)/48; the
 * adjoint negates both hopping coefficients. */
void orc_hisq(const int *L, const double *phases, const int *eta_offset,
              int nc, double mass, double naik_epsilon, int dagger,
              const double *const *X, const double *const *Lng,
              const double *psid, double *outd) {
  const int64_t V = volume_of(L);
  const cplx *psi = (const cplx *)psid;
  cplx *out = (cplx *)outd;
  int zero_off[4] = {0, 0, 0, 0};
  const int *off = eta_offset ? eta_offset : zero_off;
  double sign = dagger ? -1.0 : 1.0;
  for (int64_t k = 0; k < V * nc; k++) out[k] = mass * psi[k];
  staggered_hop(L, phases, off, nc, 1, sign * 0.5, X, psid, out);
  staggered_hop(L, phases, off, nc, 3, -sign * (1.0 + naik_epsilon) / 48.0,
                Lng, psid, out);
}

/* ---------------------------------------------------------------------------
 * HISQ smearing.
 * Path products (HISQSmearing.jl:15-93, _hisq_path_row): a positive step d
 * multiplies by U_d(site) and moves to site+d; a negative step moves to
 * site-d and multiplies by U_d(site-d)^+.  Links are periodic.
 * ------------------------------------------------------------------------- */
static void path_product(const int *L, int nc, const cplx *const *U,
                         const int *origin, const int *path, int len,
                         cplx *out) {
  int c[4] = {origin[0], origin[1], origin[2], origin[3]};
  cplx m[64];
  for (int k = 0; k < nc * nc; k++) out[k] = 0;
  for (int k = 0; k < nc; k++) out[k + nc * k] = 1;
  for (int i = 0; i < len; i++) {
    int d = path[i];
    int axis = abs(d) - 1;
    if (d > 0) {
      mat_load(nc, U[axis], site_of(L, c), 0, m);
      mat_mul(nc, out, m, out);
      c[axis] = (c[axis] + 1) % L[axis];
    } else {
      c[axis] = (c[axis] - 1 + L[axis]) % L[axis];
      mat_load(nc, U[axis], site_of(L, c), 1, m);
      mat_mul(nc, out, m, out);
    }
  }
}

static const int five_signs[4][2] = {{1, 1}, {-1, -1}, {1, -1}, {-1, 1}};
static const int seven_signs[8][3] = {{1, 1, 1},  {-1, -1, -1}, {-1, 1, 1},
                                      {1, -1, 1}, {1, 1, -1},   {-1, -1, 1},
                                      {-1, 1, -1}, {1, -1, -1}};

/* Fat7 (+Lepage) with coefficients (c1, c3, c5, c7, cLepage)
 * (HISQSmearing.jl:490-566 staples, 1193-1242 launch order,
 *  level-1 1139-1145, level-2 1335-1339). */
void orc_hisq_fat7(const int *L, int nc, const double *coef,
                   const double *const *Ud, double *const *Vd) {
  const int64_t V = volume_of(L);
  const cplx *U[4] = {(const cplx *)Ud[0], (const cplx *)Ud[1],
                      (const cplx *)Ud[2], (const cplx *)Ud[3]};
#pragma omp parallel for schedule(static)
  for (int64_t s = 0; s < V; s++) {
    int c[4];
    coords_of(L, s, c);
    for (int mu = 1; mu <= 4; mu++) {
      cplx acc[64], sum[64], p[64];
      mat_load(nc, U[mu - 1], s, 0, acc);
      for (int k = 0; k < nc * nc; k++) acc[k] *= coef[0];
      /* three-link staples */
      for (int k = 0; k < nc * nc; k++) sum[k] = 0;
      for (int nu = 1; nu <= 4; nu++) {
        if (nu == mu) continue;
        int p1[3] = {nu, mu, -nu}, p2[3] = {-nu, mu, nu};
        path_product(L, nc, U, c, p1, 3, p);
        for (int k = 0; k < nc * nc; k++) sum[k] += p[k];
        path_product(L, nc, U, c, p2, 3, p);
        for (int k = 0; k < nc * nc; k++) sum[k] += p[k];
      }
      for (int k = 0; k < nc * nc; k++) acc[k] += coef[1] * sum[k];
      /* five-link staples, four sign parts */
      for (int part = 0; part < 4; part++) {
        for (int k = 0; k < nc * nc; k++) sum[k] = 0;
        for (int nu = 1; nu <= 4; nu++) {
          if (nu == mu) continue;
          for (int rho = 1; rho <= 4; rho++) {
            if (rho == mu || rho == nu) continue;
            int sn = five_signs[part][0] * nu, sr = five_signs[part][1] * rho;
            int path[5] = {sn, sr, mu, -sr, -sn};
            path_product(L, nc, U, c, path, 5, p);
            for (int k = 0; k < nc * nc; k++) sum[k] += p[k];
          }
        }
        for (int k = 0; k < nc * nc; k++) acc[k] += coef[2] * sum[k];
      }
      /* seven-link staples, eight sign parts */
      for (int part = 0; part < 8; part++) {
        for (int k = 0; k < nc * nc; k++) sum[k] = 0;
        for (int nu = 1; nu <= 4; nu++) {
          if (nu == mu) continue;
          for (int rho = 1; rho <= 4; rho++) {
            if (rho == mu || rho == nu) continue;
            int sigma = 10 - mu - nu - rho;
            int sn = seven_signs[part][0] * nu, sr = seven_signs[part][1] * rho;
            int ss = seven_signs[part][2] * sigma;
            int path[7] = {sn, sr, ss, mu, -ss, -sr, -sn};
            path_product(L, nc, U, c, path, 7, p);
            for (int k = 0; k < nc * nc; k++) sum[k] += p[k];
          }
        }
        for (int k = 0; k < nc * nc; k++) acc[k] += coef[3] * sum[k];
      }
      /* Lepage */
      if (coef[4] != 0.0) {
        for (int k = 0; k < nc * nc; k++) sum[k] = 0;
        for (int nu = 1; nu <= 4; nu++) {
          if (nu == mu) continue;
          int p1[5] = {nu, nu, mu, -nu, -nu}, p2[5] = {-nu, -nu, mu, nu, nu};
          path_product(L, nc, U, c, p1, 5, p);
          for (int k = 0; k < nc * nc; k++) sum[k] += p[k];
          path_product(L, nc, U, c, p2, 5, p);
          for (int k = 0; k < nc * nc; k++) sum[k] += p[k];
        }
        for (int k = 0; k < nc * nc; k++) acc[k] += coef[4] * sum[k];
      }
      cplx *Vm = (cplx *)Vd[mu - 1];
      for (int r = 0; r < nc; r++)
        for (int col = 0; col < nc; col++)
          Vm[r + nc * (col + nc * s)] = acc[r + nc * col];
    }
  }
}

/* U(3) projection W = V (V^+V)^{-1/2} with the trigonometric eigenvalue
 * solution and Cayley-Hamilton coefficients (HISQFullSmearing.jl:1-77). */
static void u3_project_matrix(const cplx *Vm, cplx *Wm) {
  cplx Q[9], Q2[9], inv[9];
  for (int r = 0; r < 3; r++)
    for (int col = 0; col < 3; col++) {
      cplx v = 0;
      for (int k = 0; k < 3; k++) v += conj(Vm[k + 3 * r]) * Vm[k + 3 * col];
      Q[r + 3 * col] = v;
    }
  mat_mul(3, Q, Q, Q2);
  double c0 = 0, trQ2 = 0, trQ3 = 0;
  for (int i = 0; i < 3; i++) {
    c0 += creal(Q[i + 3 * i]);
    trQ2 += creal(Q2[i + 3 * i]);
    for (int j = 0; j < 3; j++) trQ3 += creal(Q2[i + 3 * j] * Q[j + 3 * i]);
  }
  double c1 = trQ2 / 2, c2 = trQ3 / 3;
  double S = c1 / 3 - c0 * c0 / 18;
  double g0, g1, g2;
  if (fabs(S) < 1e-7) {
    g0 = g1 = g2 = c0 / 3;
  } else {
    S = sqrt(fmax(S, 0.0));
    double R = c2 / 2 - c0 * c1 / 3 + c0 * c0 * c0 / 27;
    double ratio = R / (S * S * S);
    if (ratio > 1) ratio = 1;
    if (ratio < -1) ratio = -1;
    double theta = acos(ratio);
    const double tpt = 2 * M_PI / 3;
    double center = c0 / 3, amp = 2 * S;
    g0 = center + amp * cos(theta / 3 - tpt);
    g1 = center + amp * cos(theta / 3);
    g2 = center + amp * cos(theta / 3 + tpt);
  }
  const double floor_ = 2.220446049250313e-16;
  g0 = fmax(g0, floor_);
  g1 = fmax(g1, floor_);
  g2 = fmax(g2, floor_);
  double u = sqrt(g0) + sqrt(g1) + sqrt(g2);
  double v = sqrt(g0 * g1) + sqrt(g0 * g2) + sqrt(g1 * g2);
  double w = sqrt(g0 * g1 * g2);
  double den = w * (u * v - w);
  double f0 = (-w * (u * u + v) + u * v * v) / den;
  double f1 = (-w - u * u * u + 2 * u * v) / den;
  double f2 = u / den;
  for (int col = 0; col < 3; col++)
    for (int r = 0; r < 3; r++)
      inv[r + 3 * col] = (r == col ? f0 : 0.0) + f1 * Q[r + 3 * col] +
                         f2 * Q2[r + 3 * col];
  mat_mul(3, Vm, inv, Wm);
}

void orc_hisq_project_u3(const int *L, const double *const *Vd,
                         double *const *Wd) {
  const int64_t V = volume_of(L);
  for (int mu = 0; mu < 4; mu++) {
    const cplx *Vm = (const cplx *)Vd[mu];
    cplx *Wm = (cplx *)Wd[mu];
#pragma omp parallel for schedule(static)
    for (int64_t s = 0; s < V; s++) u3_project_matrix(Vm + 9 * s, Wm + 9 * s);
  }
}

/* Forward-anchored Naik transporter L_mu(x) = W_mu(x) W_mu(x+mu) W_mu(x+2mu)
 * (HISQFullSmearing.jl:136-195). */
void orc_hisq_naik(const int *L, int nc, const double *const *Wd,
                   double *const *Ld) {
  const int64_t V = volume_of(L);
  const cplx *W[4] = {(const cplx *)Wd[0], (const cplx *)Wd[1],
                      (const cplx *)Wd[2], (const cplx *)Wd[3]};
  for (int mu = 1; mu <= 4; mu++) {
    cplx *Lm = (cplx *)Ld[mu - 1];
#pragma omp parallel for schedule(static)
    for (int64_t s = 0; s < V; s++) {
      int c[4];
      coords_of(L, s, c);
      int path[3] = {mu, mu, mu};
      cplx p[64];
      path_product(L, nc, W, c, path, 3, p);
      for (int k = 0; k < nc * nc; k++) Lm[k + (int64_t)nc * nc * s] = p[k];
    }
  }
}

/* hisq_links_from_thin! (HISQFullSmearing.jl:284-293): level-1 Fat7, U(3)
 * projection, level-2 Fat7 + Lepage, Naik. */
void orc_hisq_links_from_thin(const int *L, double naik_epsilon,
                              const double *const *U, double *const *X,
                              double *const *Lng) {
  const int64_t V = volume_of(L);
  double *lvl1[4], *W[4];
  for (int mu = 0; mu < 4; mu++) {
    lvl1[mu] = (double *)malloc(sizeof(double) * 18 * V);
    W[mu] = (double *)malloc(sizeof(double) * 18 * V);
  }
  const double c_level1[5] = {1.0 / 8, 1.0 / 16, 1.0 / 64, 1.0 / 384, 0.0};
  const double c_level2[5] = {1.0 + naik_epsilon / 8, 1.0 / 16, 1.0 / 64,
                              1.0 / 384, -1.0 / 8};
  orc_hisq_fat7(L, 3, c_level1, U, lvl1);
  orc_hisq_project_u3(L, (const double *const *)lvl1, W);
  orc_hisq_fat7(L, 3, c_level2, (const double *const *)W, X);
  orc_hisq_naik(L, 3, (const double *const *)W, Lng);
  for (int mu = 0; mu < 4; mu++) {
    free(lvl1[mu]);
    free(W[mu]);
  }
}

/* ---------------------------------------------------------------------------
 * Operator dispatch, dot, and CG (cg.jl:73-137; DiracOperators.jl:104-121)
 * ------------------------------------------------------------------------- */
int64_t orc_field_reals(const orc_operator *op) {
  int64_t V = volume_of(op->L);
  int spins = (op->kind == ORC_OP_WILSON || op->kind == ORC_OP_CLOVER) ? 4 : 1;
  return 2 * V * op->nc * spins;
}

void orc_apply(const orc_operator *op, int dagger, const double *in,
               double *out) {
  switch (op->kind) {
  case ORC_OP_WILSON:
    orc_wilson(op->L, op->phases, op->nc, op->kappa, dagger, op->links, in,
               out);
    break;
  case ORC_OP_CLOVER:
    orc_wilson_clover(op->L, op->phases, op->nc, op->kappa, op->csw, dagger,
                      op->links, op->F, in, out);
    break;
  case ORC_OP_STAGGERED:
    orc_staggered(op->L, op->phases, op->eta_offset, op->nc, op->mass, dagger,
                  op->links, in, out);
    break;
  case ORC_OP_HISQ:
    orc_hisq(op->L, op->phases, op->eta_offset, op->nc, op->mass,
             op->naik_epsilon, dagger, op->links, op->links + 4, in, out);
    break;
  }
}

void orc_apply_ddagd(const orc_operator *op, const double *in, double *tmp,
                     double *out) {
  orc_apply(op, 0, in, tmp);
  orc_apply(op, 1, tmp, out);
}

void orc_dot(int64_t ncomplex, const double *a, const double *b, double *out) {
  /* dot(A, B) = sum conj(A) B (linearalgebra_D.jl:3325-3341) */
  double re = 0, im = 0;
#pragma omp parallel for reduction(+ : re, im) schedule(static)
  for (int64_t k = 0; k < ncomplex; k++) {
    re += a[2 * k] * b[2 * k] + a[2 * k + 1] * b[2 * k + 1];
    im += a[2 * k] * b[2 * k + 1] - a[2 * k + 1] * b[2 * k];
  }
  out[0] = re;
  out[1] = im;
}

static double re_dot(int64_t n, const double *a, const double *b) {
  double re = 0;
#pragma omp parallel for reduction(+ : re) schedule(static)
  for (int64_t k = 0; k < n; k++) re += a[k] * b[k];
  return re;
}

/* y = a*x + b*y for real a, b (axpby!, linearalgebra_D.jl:2-41) */
static void axpby_real(int64_t n, double a, const double *x, double b,
                       double *y) {
#pragma omp parallel for schedule(static)
  for (int64_t k = 0; k < n; k++) y[k] = a * x[k] + b * y[k];
}

static void cg_finish(orc_cg_result *res, int converged, int it, double rn,
                      double bn, int reason) {
  res->converged = converged;
  res->iterations = it;
  res->residual_norm = rn;
  if (bn == 0.0)
    res->relative_residual = (rn == 0.0) ? 0.0 : INFINITY;
  else
    res->relative_residual = rn / bn;
  res->reason = reason;
}

void orc_cg_ddagd(const orc_operator *op, double *x, const double *b,
                  double rtol, double atol, int maxiter, orc_cg_result *res) {
  const int64_t n = orc_field_reals(op);
  double *r = (double *)malloc(sizeof(double) * n);
  double *p = (double *)malloc(sizeof(double) * n);
  double *Ap = (double *)malloc(sizeof(double) * n);
  double *tmp = (double *)malloc(sizeof(double) * n);
  double bb = re_dot(n, b, b);
  if (!isfinite(bb) || bb < 0) {
    cg_finish(res, 0, 0, NAN, NAN, 3);
    goto done;
  }
  double bn = sqrt(bb);
  double tol = fmax(atol, rtol * bn);
  orc_apply_ddagd(op, x, tmp, Ap);
  axpby_real(n, 1.0, b, 0.0, r);
  axpby_real(n, -1.0, Ap, 1.0, r);
  axpby_real(n, 1.0, r, 0.0, p);
  double rr = re_dot(n, r, r);
  if (!isfinite(rr) || rr < 0) {
    cg_finish(res, 0, 0, NAN, bn, 3);
    goto done;
  }
  double rn = sqrt(rr);
  if (rn <= tol) {
    cg_finish(res, 1, 0, rn, bn, 0);
    goto done;
  }
  for (int it = 1; it <= maxiter; it++) {
    orc_apply_ddagd(op, p, tmp, Ap);
    double pAp = re_dot(n, p, Ap);
    if (!isfinite(pAp)) {
      cg_finish(res, 0, it - 1, rn, bn, 3);
      goto done;
    } else if (pAp <= 0) {
      cg_finish(res, 0, it - 1, rn, bn, 2);
      goto done;
    }
    double alpha = rr / pAp;
    axpby_real(n, alpha, p, 1.0, x);
    axpby_real(n, -alpha, Ap, 1.0, r);
    double rr_new = re_dot(n, r, r);
    if (!isfinite(rr_new) || rr_new < 0) {
      cg_finish(res, 0, it, NAN, bn, 3);
      goto done;
    }
    rn = sqrt(rr_new);
    if (rn <= tol) {
      cg_finish(res, 1, it, rn, bn, 0);
      goto done;
    }
    double beta = rr_new / rr;
    axpby_real(n, 1.0, r, beta, p);
    rr = rr_new;
  }
  cg_finish(res, 0, maxiter, rn, bn, 1);
done:
  free(r);
  free(p);
  free(Ap);
  free(tmp);
}

double orc_cg_ddagd_iterations(const orc_operator *op, double *x,
                               const double *b, int iterations) {
  const int64_t n = orc_field_reals(op);
  double *r = (double *)malloc(sizeof(double) * n);
  double *p = (double *)malloc(sizeof(double) * n);
  double *Ap = (double *)malloc(sizeof(double) * n);
  double *tmp = (double *)malloc(sizeof(double) * n);
  memset(x, 0, sizeof(double) * n);
  memcpy(r, b, sizeof(double) * n);
  memcpy(p, b, sizeof(double) * n);
  double rr = re_dot(n, r, r);
  double t0 = 0;
#ifdef _OPENMP
  t0 = omp_get_wtime();
#endif
  for (int it = 0; it < iterations; it++) {
    orc_apply_ddagd(op, p, tmp, Ap);
    double pAp = re_dot(n, p, Ap);
    double alpha = rr / pAp;
    axpby_real(n, alpha, p, 1.0, x);
    axpby_real(n, -alpha, Ap, 1.0, r);
    double rr_new = re_dot(n, r, r);
    double beta = rr_new / rr;
    axpby_real(n, 1.0, r, beta, p);
    rr = rr_new;
  }
  double t1 = 0;
#ifdef _OPENMP
  t1 = omp_get_wtime();
#endif
  free(r);
  free(p);
  free(Ap);
  free(tmp);
  return t1 - t0;
}

/* ---------------------------------------------------------------------------
 * Seeded inputs.
 * Philox4x32-10 counter-based generator (Salmon, Moraes, Dror and Shaw,
 * "Parallel random numbers: as easy as 1, 2, 3", SC 2011), the same family
 * as the reference's Philox site streams (utilities/randomgenerator.jl:247-340).
 * ------------------------------------------------------------------------- */
void orc_philox4x32(const uint32_t *counter, const uint32_t *key,
                    uint32_t *out) {
  uint32_t c0 = counter[0], c1 = counter[1], c2 = counter[2], c3 = counter[3];
  uint32_t k0 = key[0], k1 = key[1];
  for (int round = 0; round < 10; round++) {
    uint64_t p0 = (uint64_t)0xD2511F53u * c0;
    uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
    uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
    c0 = n0;
    c1 = lo1;
    c2 = n2;
    c3 = lo0;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  out[0] = c0;
  out[1] = c1;
  out[2] = c2;
  out[3] = c3;
}

/* two Box-Muller normals from one Philox block (53-bit uniforms in (0,1)) */
static void philox_normals(uint32_t site, uint32_t lane, uint32_t draw,
                           uint32_t tag, uint64_t seed, double *g) {
  uint32_t ctr[4] = {site, lane, draw, tag};
  uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32) ^ 0x4C4D4232u};
  uint32_t w[4];
  orc_philox4x32(ctr, key, w);
  double u1 = ((double)(w[0] >> 5) * 67108864.0 + (double)(w[1] >> 6) + 0.5) /
              9007199254740992.0;
  double u2 = ((double)(w[2] >> 5) * 67108864.0 + (double)(w[3] >> 6) + 0.5) /
              9007199254740992.0;
  double rad = sqrt(-2.0 * log(u1));
  g[0] = rad * cos(2.0 * M_PI * u2);
  g[1] = rad * sin(2.0 * M_PI * u2);
}

/* Gram-Schmidt on rows 1 and 2 and row 3 = conj(row1 x row2)
 * (linearalgebra_D.jl:2371-2424, kernel_normalize_NC3!).  m is column-major
 * 3x3 complex (18 doubles). */
void orc_reunitarize_su3(double *md) {
  cplx *u = (cplx *)md;
#define UE(r, c) u[(r) + 3 * (c)]
  cplx w1 = 0;
  double w2 = 0;
  for (int ic = 0; ic < 3; ic++) {
    w1 += UE(1, ic) * conj(UE(0, ic));
    w2 += creal(UE(0, ic) * conj(UE(0, ic)));
  }
  w1 = -w1 / w2;
  cplx x4 = UE(1, 0) + w1 * UE(0, 0);
  cplx x5 = UE(1, 1) + w1 * UE(0, 1);
  cplx x6 = UE(1, 2) + w1 * UE(0, 2);
  double w3 = creal(x4 * conj(x4) + x5 * conj(x5) + x6 * conj(x6));
  UE(1, 0) = x4;
  UE(1, 1) = x5;
  UE(1, 2) = x6;
  w3 = 1.0 / sqrt(w3);
  w2 = 1.0 / sqrt(w2);
  for (int ic = 0; ic < 3; ic++) {
    UE(0, ic) *= w2;
    UE(1, ic) *= w3;
  }
  UE(2, 0) = conj(UE(0, 1) * UE(1, 2) - UE(0, 2) * UE(1, 1));
  UE(2, 1) = conj(UE(0, 2) * UE(1, 0) - UE(0, 0) * UE(1, 2));
  UE(2, 2) = conj(UE(0, 0) * UE(1, 1) - UE(0, 1) * UE(1, 0));
#undef UE
}

/* exp(M) by scaling and squaring of a degree-16 Taylor polynomial (M = i a H
 * has a small norm, so 2^-k scaling to ||M|| < 1/8 keeps the truncation below
 * 1e-20 before squaring). */
static void expm3(const cplx *M, cplx *E) {
  double nrm = 0;
  for (int k = 0; k < 9; k++) nrm += creal(M[k] * conj(M[k]));
  nrm = sqrt(nrm);
  int sq = 0;
  while (nrm > 0.125) { nrm *= 0.5; sq++; }
  double scale = ldexp(1.0, -sq);
  cplx A[9], term[9];
  for (int k = 0; k < 9; k++) A[k] = M[k] * scale;
  for (int k = 0; k < 9; k++) { E[k] = 0; term[k] = 0; }
  for (int k = 0; k < 3; k++) { E[k + 3 * k] = 1; term[k + 3 * k] = 1; }
  for (int n = 1; n <= 16; n++) {
    mat_mul(3, term, A, term);
    for (int k = 0; k < 9; k++) term[k] /= n;
    for (int k = 0; k < 9; k++) E[k] += term[k];
  }
  for (int s = 0; s < sq; s++) mat_mul(3, E, E, E);
}

/* U_mu(x) = reunitarize(exp(i a H)), H traceless Hermitian with Gaussian
 * entries: diagonal N(0,1) minus its mean, off-diagonal (N + iN)/sqrt(2).
 * Stream: counter (site, mu, draw, 0x4C4B) under `seed`.  The lattice site
 * index is the global lexicographic index, so the field does not depend on
 * how it is later decomposed. */
void orc_random_su3_links(const int *L, double amplitude, uint64_t seed,
                          double *const *Ud) {
  const int64_t V = volume_of(L);
#pragma omp parallel for schedule(static)
  for (int64_t s = 0; s < V; s++) {
    for (int mu = 0; mu < 4; mu++) {
      double g[10];
      for (int d = 0; d < 5; d++)
        philox_normals((uint32_t)s, (uint32_t)mu, (uint32_t)d, 0x4C4Bu, seed,
                       g + 2 * d);
      cplx H[9];
      double mean = (g[0] + g[1] + g[2]) / 3.0;
      H[0] = g[0] - mean;
      H[4] = g[1] - mean;
      H[8] = g[2] - mean;
      const double r2 = 0.70710678118654752440;
      cplx h01 = (g[3] + I * g[4]) * r2, h02 = (g[5] + I * g[6]) * r2,
           h12 = (g[7] + I * g[8]) * r2;
      H[0 + 3 * 1] = h01; H[1 + 3 * 0] = conj(h01);
      H[0 + 3 * 2] = h02; H[2 + 3 * 0] = conj(h02);
      H[1 + 3 * 2] = h12; H[2 + 3 * 1] = conj(h12);
      cplx M[9], E[9];
      for (int k = 0; k < 9; k++) M[k] = I * amplitude * H[k];
      expm3(M, E);
      orc_reunitarize_su3((double *)E);
      memcpy(Ud[mu] + 18 * s, E, sizeof(E));
    }
  }
}

/* Unit-variance complex Gaussian field: re and im each N(0, 1/2)
 * (benchmark/ddagd_cg/README.md:161-162).  `components` complex numbers per
 * site, stream (site, component pair, 0, 0x5350) under `seed`. */
void orc_gaussian_field(const int *L, int components, uint64_t seed,
                        double *out) {
  const int64_t V = volume_of(L);
  const double r2 = 0.70710678118654752440;
#pragma omp parallel for schedule(static)
  for (int64_t s = 0; s < V; s++) {
    for (int k = 0; k < components; k++) {
      double g[2];
      philox_normals((uint32_t)s, (uint32_t)k, 0u, 0x5350u, seed, g);
      out[2 * (k + (int64_t)components * s)] = g[0] * r2;
      out[2 * (k + (int64_t)components * s) + 1] = g[1] * r2;
    }
  }
}
