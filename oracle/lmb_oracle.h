/*
 * lmb_oracle.h -- CPU restatement (FP64) of the LatticeMatrices.jl Dirac-operator
 * hot path.  TEST INFRASTRUCTURE ONLY: the product (liblmb200.so) never links,
 * loads or calls anything declared here.  Only tests/, __graft_entry__.smoke()
 * and bench.py's CPU-baseline leg use it, as the checker or as the timed CPU
 * baseline.
 *
 * Field layout: the reference's core layout without halo (nw = 0), column-major
 * (NC1, NC2, X, Y, Z, T) complex128, x fastest (LatticeMatrices_core.jl:4-9,
 * 361-363).  Gauge link mu: (NC, NC, sites); Wilson spinor: (NC, 4, sites);
 * staggered field: (NC, 1, sites).
 *
 * Boundary phases: a neighbour read that wraps forward across the lattice edge
 * is multiplied by phase[mu], a backward wrap by 1/phase[mu]
 * (LatticeMatrices_core.jl:707-723, exchange_dim_local!).  Gauge links are
 * periodic.
 */
#ifndef LMB_ORACLE_H
#define LMB_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* geometry: L[4] lattice extents, phases[8] = (re, im) per direction,
 * eta_offset[4] = global coordinate of the local origin (0 on one rank). */

/* generalised domain-wall operator D5 (dagger = 1: D5^+), fields
 * (nc, 4, X, Y, Z, T, L5); a, b, c: L5 coefficients each */
void orc_domainwall(const int *L, int L5, const double *phases, int nc, double mass, double M,
                    const double *a, const double *b, const double *c, int dagger,
                    const double *const *U, const double *psi, double *out);
void orc_wilson(const int *L, const double *phases, int nc, double kappa,
                int dagger, const double *const *U, const double *psi,
                double *out);
void orc_wilson_donly(const int *L, const double *phases, int nc, int dagger,
                      const double *const *U, const double *psi, double *out);
void orc_clover_field_strength(const int *L, int nc, const double *const *U,
                               double *const *F);
void orc_add_clover_term(const int *L, int nc, double coefficient,
                         const double *const *F, const double *psi,
                         double *out);
void orc_wilson_clover(const int *L, const double *phases, int nc,
                       double kappa, double csw, int dagger,
                       const double *const *U, const double *const *F,
                       const double *psi, double *out);
void orc_staggered(const int *L, const double *phases, const int *eta_offset,
                   int nc, double mass, int dagger, const double *const *U,
                   const double *psi, double *out);
void orc_hisq(const int *L, const double *phases, const int *eta_offset,
              int nc, double mass, double naik_epsilon, int dagger,
              const double *const *X, const double *const *Lng,
              const double *psi, double *out);

void orc_hisq_fat7(const int *L, int nc, const double *coefficients,
                   const double *const *U, double *const *V);
void orc_hisq_project_u3(const int *L, const double *const *V,
                         double *const *W);
void orc_hisq_naik(const int *L, int nc, const double *const *W,
                   double *const *Lng);
void orc_hisq_links_from_thin(const int *L, double naik_epsilon,
                              const double *const *U, double *const *X,
                              double *const *Lng);

/* op kinds for the CG driver */
enum { ORC_OP_WILSON = 0, ORC_OP_CLOVER = 1, ORC_OP_STAGGERED = 2,
       ORC_OP_HISQ = 3 };

typedef struct {
  int kind;
  int nc;
  int L[4];
  double phases[8];
  int eta_offset[4];
  double kappa, csw, mass, naik_epsilon;
  const double *links[8]; /* Wilson/clover/staggered: U[0..3]; HISQ: X[0..3], L[0..3] */
  const double *F[6];     /* clover field strength (12,13,14,23,24,34) */
} orc_operator;

typedef struct {
  int converged;
  int iterations;
  double residual_norm;
  double relative_residual;
  int reason; /* 0 converged, 1 maximum_iterations, 2 nonpositive_curvature,
                 3 numerical_breakdown */
} orc_cg_result;

int64_t orc_field_reals(const orc_operator *op);
void orc_apply(const orc_operator *op, int dagger, const double *in,
               double *out);
void orc_apply_ddagd(const orc_operator *op, const double *in, double *tmp,
                     double *out);
void orc_cg_ddagd(const orc_operator *op, double *x, const double *b,
                  double rtol, double atol, int maxiter, orc_cg_result *res);
/* Time-boxed CG: runs at most `iterations` CG iterations on D'D (zero start),
 * returns the wall seconds spent in the iterations. */
double orc_cg_ddagd_iterations(const orc_operator *op, double *x,
                               const double *b, int iterations);

void orc_dot(int64_t ncomplex, const double *a, const double *b, double *out);

/* seeded inputs */
void orc_philox4x32(const uint32_t *counter, const uint32_t *key,
                    uint32_t *out);
void orc_random_su3_links(const int *L, double amplitude, uint64_t seed,
                          double *const *U);
void orc_gaussian_field(const int *L, int components, uint64_t seed,
                        double *out);
void orc_reunitarize_su3(double *m);

int orc_num_threads(void);
void orc_set_num_threads(int n);

#ifdef __cplusplus
}
#endif
#endif
