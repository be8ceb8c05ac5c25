/*
 * lmb200.h -- C ABI of liblmb200.so, the B200 (sm_100a) implementation of the
 * LatticeMatrices.jl Dirac-operator hot path.
 *
 * Plain C types only: device pointers are `void *` to the reference's
 * halo-padded field storage (the CuArray behind a LatticeMatrix, column-major
 * (NC1, NC2, X+2nw, Y+2nw, Z+2nw, T+2nw), LatticeMatrices_core.jl:4-9,
 * 361-363), streams are `void *` (cudaStream_t; NULL = legacy default
 * stream).  Every call writes only the core sites of its outputs; the caller
 * marks the output halo dirty exactly as _parallel_for_mutating! does
 * (LatticeMatrices_core.jl:216-219).
 *
 * Errors: every int-returning entry point returns LMB_OK (0) or a negative
 * LMB_ERR_* code and never traps or throws; lmb_last_error() holds the text.
 * Threading: one context per host thread / stream; a context is not
 * re-entrant.  Calls are ordered on the caller's stream; only lmb_cg_ddagd and
 * lmb_field_dot synchronise with the host, as the reference's `cg!` and `dot`
 * return host scalars.
 */
#ifndef LMB200_H
#define LMB200_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LMB_OK 0
#define LMB_ERR_ARG (-1)         /* validation failure (ArgumentError)     */
#define LMB_ERR_CUDA (-2)        /* CUDA runtime error                     */
#define LMB_ERR_STATE (-3)       /* geometry or links not set              */
#define LMB_ERR_UNSUPPORTED (-4) /* combination not provided by this build */

#define LMB_DTYPE_C128 0 /* ComplexF64 fields */
#define LMB_DTYPE_C64 1  /* ComplexF32 fields */

#define LMB_PREC_DOUBLE 0 /* FP64 storage and arithmetic                       */
#define LMB_PREC_SINGLE 1 /* FP32 storage and arithmetic                       */
#define LMB_PREC_HALF 2   /* int16 storage (per-site norm), FP32 arithmetic    */

#define LMB_OP_WILSON 0
#define LMB_OP_WILSON_CLOVER 1
#define LMB_OP_STAGGERED 2
#define LMB_OP_HISQ 3
#define LMB_OP_DOMAINWALL 4 /* lmb_domainwall_set parameters, 5D fields */

#define LMB_LINKS_THIN 0 /* Wilson / clover / staggered links U_mu      */
#define LMB_LINKS_FAT 1  /* HISQ fat links X_mu (HISQLinks4D)           */
#define LMB_LINKS_LONG 2 /* HISQ Naik links L_mu (HISQLinks4D)          */

/* CG status, mirroring CGResult.reason (LinearAlgebras/cg.jl:1-13) */
#define LMB_CG_CONVERGED 0
#define LMB_CG_MAXIMUM_ITERATIONS 1
#define LMB_CG_NONPOSITIVE_CURVATURE 2
#define LMB_CG_NUMERICAL_BREAKDOWN 3

typedef struct lmb_ctx lmb_ctx;

typedef struct {
  int op;              /* LMB_OP_*                                              */
  double kappa, csw;   /* Wilson / Wilson-clover                                */
  double mass;         /* staggered / HISQ                                      */
  double naik_epsilon; /* HISQ                                                  */
  double rtol, atol;   /* stop when |r| <= max(atol, rtol |b|) (cg.jl:61-63)    */
  int maxiter;
  int precision;       /* LMB_PREC_DOUBLE: plain FP64 CG (cg.jl:73-137);
                          SINGLE / HALF: inner D'D at that precision with FP64
                          reliable updates and an FP64 true-residual stop        */
  double delta;        /* reliable-update threshold (mixed only), e.g. 0.1      */
  int check_interval;  /* iterations between host status checks (0 = default)  */
  int profile;         /* 1: time every stencil launch with CUDA events        */
} lmb_cg_params;

typedef struct {
  int converged;
  int iterations;
  double residual_norm;     /* recursive (plain) or FP64 true residual (mixed) */
  double relative_residual; /* residual_norm / |b| (cg.jl:16-22)               */
  int reason;               /* LMB_CG_*                                        */
  int reliable_updates;
  double true_residual_norm; /* |b - D'D x| in FP64 (mixed, and plain on exit) */
  /* profile = 1: device time of the two stencil kernels of an iteration */
  double dslash_ms, update_ms; /* K1 (tmp = D p, |tmp|^2) and K2 (D'tmp + axpy) */
  int dslash_launches, update_launches;
  long long kernel_launches; /* liblmb200 kernels launched by this solve    */
  int link_reals;            /* reals stored per link by the iterated stencil:
                                18, or 12 for SU(3) links (third row rebuilt) */
} lmb_cg_result;

/* ---- context --------------------------------------------------------------
 * The context owns the repacked link / clover caches and the solver
 * workspaces (WilsonDiracCloverOperator.jl:418-432 CloverCacheState;
 * HISQFullSmearing.jl:340-354 HISQCacheState).  Field memory stays the
 * caller's (CuArray or any device allocation). */
lmb_ctx *lmb_create(int device);
void lmb_destroy(lmb_ctx *ctx);
const char *lmb_last_error(const lmb_ctx *ctx);
int lmb_version(void);

/* Lattice geometry of every field passed afterwards: local extents L (x
 * fastest), halo width nw, fermion boundary phases (LatticeMatrix.phases,
 * LatticeMatrices_core.jl:159-184; forward wrap * phase, backward wrap / phase,
 * :707-723), Cartesian rank coordinates for the global staggered eta
 * (LinearAlgebras/staggered.jl:43-57) and the element type of the fields
 * (LMB_DTYPE_*).  Replaces the per-call ensure_halo!/set_halo! of a single
 * rank (LatticeMatrices_core.jl:550-588) by in-kernel periodic indexing. */
int lmb_set_geometry(lmb_ctx *ctx, const int L[4], int nw,
                     const double phase_re[4], const double phase_im[4],
                     const int coords[4], int dtype);

/* Upload (repack) four link fields.  The cache is keyed by the pointers and
 * the core epochs (halo_epoch.core), as _clover_cache_is_current
 * (WilsonDiracCloverOperator.jl:603-625) and _ensure_hisq_cache_current!
 * (HISQFullSmearing.jl:435-441): an unchanged (pointer, epoch) set is not
 * re-read.  which = LMB_LINKS_*. */
int lmb_links_upload(lmb_ctx *ctx, int which, const void *const U[4],
                     const uint64_t epoch[4], void *stream);

/* mul!(out, WilsonDiracOperator4D(U, kappa), in) and its adjoint
 * (Operators/WilsonDiracOperator.jl:60-76, 420-438).  out != in. */
int lmb_wilson_apply(lmb_ctx *ctx, void *out, const void *in, double kappa,
                     int dagger, int precision, void *stream);

/* mul!(out, WilsonDiracCloverOperator4D(U, kappa, cSW), in) / adjoint and
 * mul_cached_clover! / mul_cached_clover_adjoint!
 * (Operators/WilsonDiracCloverOperator.jl:561-601, 642-668).  The clover
 * blocks are rebuilt when the links or kappa*cSW change (update_clover!,
 * :392-399, 468-479). */
int lmb_wilson_clover_apply(lmb_ctx *ctx, void *out, const void *in,
                            double kappa, double csw, int dagger,
                            int precision, void *stream);

/* mul!(out, StaggeredDiracOperator4D(U, mass), in) / adjoint
 * (Operators/StaggeredDiracOperator.jl:165-198): thin links from
 * lmb_links_upload(LMB_LINKS_THIN), 3 complex per site (NC x 1 fields). */
int lmb_staggered_apply(lmb_ctx *ctx, void *out, const void *in, double mass,
                        int dagger, int precision, void *stream);

/* mul!(out, HISQDiracOperator4D(HISQLinks4D(X, L), mass; naik_epsilon), in)
 * / adjoint and mul_cached_hisq! (Operators/HISQDiracOperator.jl:359-435,
 * HISQFullSmearing.jl:457-485): fat and Naik links from
 * lmb_links_upload(LMB_LINKS_FAT / LMB_LINKS_LONG). */
int lmb_hisq_apply(lmb_ctx *ctx, void *out, const void *in, double mass,
                   double naik_epsilon, int dagger, int precision,
                   void *stream);

/* HISQ smearing (FP64), on padded (3,3,...) link fields.
 * lmb_hisq_fat7: Fat7 + Lepage with coefficients (c1, c3, c5, c7, cLepage):
 *   hisq_fat7_level1! uses (1/8, 1/16, 1/64, 1/384, 0), hisq_fat7_level2!
 *   (1 + eps/8, 1/16, 1/64, 1/384, -1/8) (Operators/HISQSmearing.jl:1112-1148,
 *   1313-1379; factorised form :768-974).
 * lmb_hisq_project_u3: W = V (V^+V)^{-1/2} (HISQFullSmearing.jl:100-128).
 * lmb_hisq_naik: L_mu(x) = W_mu(x) W_mu(x+mu) W_mu(x+2mu)
 *   (HISQFullSmearing.jl:136-195). */
int lmb_hisq_fat7(lmb_ctx *ctx, const void *const U[4],
                  const double coefficients[5], void *const V[4],
                  void *stream);
int lmb_hisq_project_u3(lmb_ctx *ctx, const void *const V[4],
                        void *const W[4], void *stream);
int lmb_hisq_naik(lmb_ctx *ctx, const void *const W[4], void *const L[4],
                  void *stream);

/* hisq_links_from_thin! (HISQFullSmearing.jl:261-338): level-1 Fat7, U(3)
 * projection, level-2 Fat7 + Lepage, Naik.  The fat and Naik links become the
 * context's LMB_LINKS_FAT / LMB_LINKS_LONG sets for lmb_hisq_apply and the
 * HISQ CG, cached by thin-link pointer + epoch + naik_epsilon as
 * HISQDiracCache4D / _ensure_hisq_cache_current! (HISQFullSmearing.jl:
 * 340-441), so mul_cached_hisq! re-smears only when a link changes.  X and L
 * (four padded fields each) receive copies when non-NULL. */
int lmb_hisq_links_from_thin(lmb_ctx *ctx, const void *const U[4],
                             const uint64_t epoch[4], double naik_epsilon,
                             void *const X[4], void *const L[4],
                             void *stream);

/* hisq_link_pullback!(dU, cache, U, result_cotangent, psi; coefficient)
 * (Operators/HISQPullback.jl:620-699): accumulates into the four padded thin-
 * link fields dU the gradient G of f = coefficient Re<result_cotangent,
 * D_HISQ(U) psi> through Naik, level-2 Fat7 + Lepage, U(3) projection and
 * level-1 Fat7 (df = Re sum conj(G) dU).  The smearing levels and staples are
 * recomputed from U, not stored.  FP64. */
int lmb_hisq_link_pullback(lmb_ctx *ctx, const void *const U[4],
                           double naik_epsilon, double coefficient,
                           const void *result_cotangent, const void *psi,
                           void *const dU[4], void *stream);

/* Fermion force dS/dU of S = phi^+ (D^+D)^-1 phi for the HISQ operator built
 * from thin links U (dSFdU, ext/LatticeMatricesEnzymeExt.jl:387-460): solves
 * eta = (D^+D)^-1 phi with lmb_cg_ddagd (cg->precision, rtol, ...), chi =
 * D eta, then accumulates -2 d/dU Re<chi, D(U) eta> into dU.  result receives
 * the CG status. */
int lmb_hisq_fermion_force(lmb_ctx *ctx, const void *const U[4],
                           const uint64_t epoch[4], double mass,
                           double naik_epsilon, const void *phi,
                           void *const dU[4], const lmb_cg_params *cg,
                           lmb_cg_result *result, void *stream);

/* D5DW_GeneralizedDomainwallOperator5D(U, L5, mass, M, a, b, c)
 * (Operators/DiracOperators_5D.jl:48-115, 204-268; Mobius(b, c) is a = 1,
 * b_s = (b + c)/2, c_s = (b - c)/2, :8-46, 171-202):
 *   D5 psi = A [psi - F psi + D_W (B psi + C F psi)],
 * D_W the 4D Wilson kernel (4 + M) - 1/2 hopping with the uploaded links
 * (LMB_LINKS_THIN) and the geometry's phases, F the chiral fifth-coordinate
 * hop with -mass across the walls.  Sets the parameters used by
 * lmb_domainwall_apply and by lmb_cg_ddagd with op = LMB_OP_DOMAINWALL; a, b,
 * c hold L5 values each (copied).  Synchronises the stream. */
int lmb_domainwall_set(lmb_ctx *ctx, int L5, double mass, double M,
                       const double *a, const double *b, const double *c,
                       void *stream);

/* mul!(out, D5DW_*DomainwallOperator5D, in) / adjoint (DiracOperators_5D.jl:
 * 171-268, 1500-2084) on 5D padded fields (NC=3, 4, X+2nw, .., T+2nw,
 * L5+2nw) of the context geometry. */
int lmb_domainwall_apply(lmb_ctx *ctx, void *out, const void *in, int dagger,
                         int precision, void *stream);

/* wilson_clover_link_pullback!(dU, cache, U, result_cotangent, psi;
 * coefficient) (Operators/WilsonCloverPullback.jl:342-403): accumulates into
 * the four padded link fields dU the gradient G of f = coefficient
 * Re<result_cotangent, D(U) psi> for the Wilson-clover operator with kappa,
 * cSW (df = Re sum conj(G) dU): hopping outer products and, through
 * F_mu_nu = (Q - Q^+)/8, the four-leaf clover term.  FP64.  dU must not alias
 * U; the fields share the context geometry. */
int lmb_wilson_clover_link_pullback(lmb_ctx *ctx, const void *const U[4],
                                    double kappa, double csw,
                                    double coefficient,
                                    const void *result_cotangent,
                                    const void *psi, void *const dU[4],
                                    void *stream);

/* Fermion force dS/dU of S = phi^+ (D^+D)^-1 phi for the Wilson-clover
 * operator (the clover counterpart of lmb_hisq_fermion_force; dSFdU,
 * ext/LatticeMatricesEnzymeExt.jl:387-460): uploads U (epoch = halo_epoch.core),
 * solves eta = (D^+D)^-1 phi with lmb_cg_ddagd (cg->precision, rtol, ...),
 * chi = D eta, then accumulates -2 d/dU Re<chi, D(U) eta> into dU. */
int lmb_wilson_clover_fermion_force(lmb_ctx *ctx, const void *const U[4],
                                    const uint64_t epoch[4], double kappa,
                                    double csw, const void *phi,
                                    void *const dU[4], const lmb_cg_params *cg,
                                    lmb_cg_result *result, void *stream);

/* CloverFieldStrength4D(U) components (12,13,14,23,24,34) written to six
 * padded (3,3,...) fields (Operators/WilsonDiracCloverOperator.jl:28-35,
 * 392-399). */
int lmb_clover_field_strength(lmb_ctx *ctx, void *const F[6], void *stream);

/* set_halo! (LatticeMatrices_core.jl:550-567) of a single-rank padded field
 * (exchange_dim_local!, :707-723): the nw-deep ghost layer of every one of
 * the D (4 or 5) dimensions is filled from the periodic image of the core,
 * times phase_d on the plus side and 1/phase_d on the minus side, corners
 * with the product of the phases they wrap in -- the values the reference's
 * dimension-by-dimension exchange leaves.  field: (ncomp complex, L_1+2nw,
 * ..., L_D+2nw) column-major, dtype LMB_DTYPE_C128 or LMB_DTYPE_C64; the core
 * is read, only ghosts are written.  Needs no context (no state); returns
 * LMB_ERR_ARG for bad sizes, nw > L_d or a zero phase.  Stream-ordered. */
int lmb_set_halo(void *field, int dtype, int ncomp, int D, const int *L,
                 int nw, const double *phase_re, const double *phase_im,
                 void *stream);

/* Solve D x = b for the Wilson or Wilson-clover operator (params->op,
 * kappa, csw) by even/odd (Schur) preconditioning: the even half lattice
 * carries Dh = A_ee - kappa^2 H_eo A_oo^-1 H_oe, solved by CG on Dh Dh^+
 * (CGNE) with the CG driver of lmb_cg_ddagd (FP64, or FP32 / int16 inner
 * iterations with FP64 reliable updates), then x_o = A_oo^-1 (b_o +
 * kappa H_oe x_e).  Parity as the reference's even/odd kernels
 * (_global_site_is_even, LatticeMatrices.jl:357-363; linearalgebra_D.jl:
 * 2815-2930).  The reference reaches D x = b as cg!(x, DdagDOp(D), D'b);
 * this entry stops on the FP64 residual of D x = b itself:
 * |b - D x| <= max(atol, rtol |b|), reported in result->true_residual_norm.
 * All lattice extents must be even; x's initial content is ignored (zero
 * start).  Synchronises the stream. */
int lmb_solve_evenodd(lmb_ctx *ctx, const lmb_cg_params *params, void *x,
                      const void *b, lmb_cg_result *result, void *stream);

/* cg!(x, DdagDOp(D, temp), b, r, p, Ap; rtol, atol, maxiter)
 * (LinearAlgebras/cg.jl:73-137, Operators/DiracOperators.jl:93-143,
 * benchmark/ddagd_cg/ddagd_cg.jl:587-644).  x holds the initial guess on entry
 * and the solution on return; the work fields live in the context.
 * Synchronises the stream. */
int lmb_cg_ddagd(lmb_ctx *ctx, const lmb_cg_params *params, void *x,
                 const void *b, lmb_cg_result *result, void *stream);

/* Batched D'D CG: several lattices of different sizes, each with several
 * right-hand sides, solved together (no reference counterpart: the reference
 * solves one right-hand side per cg! call, cg.jl:73-137, which this applies
 * to every right-hand side).  Wilson operator, FP32 inner iterations with
 * FP64 reliable updates (params->precision = LMB_PREC_SINGLE) and an FP64
 * true-residual stop per right-hand side.  One launch per CG stage covers
 * all lattices and right-hand sides; an iteration is replayed from a CUDA
 * graph; the right-hand-side block and threads per block are autotuned on
 * the first call for a given set of lattice shapes and cached in the
 * context.  Links must be SU(3).  results has one entry per right-hand side
 * (lattice-major). */
typedef struct {
  int L[4];
  int nw;
  double phase_re[4], phase_im[4];
  const void *U[4];   /* ComplexF64 padded gauge links */
  uint64_t epoch[4];  /* halo_epoch.core of the links (cache key) */
  double kappa;
  int nrhs;
  void *const *x;     /* nrhs ComplexF64 padded fields: guess in, solution out */
  const void *const *b;
} lmb_batch_lattice;

typedef struct {
  int rhs_block;            /* right-hand sides sharing each link load */
  int threads;              /* sites per block */
  double ms_per_iteration;  /* device time of one batched CG iteration
                               (K1 + K2 + K3, averaged over the replays) */
  int graph_iterations;     /* iterations replayed from the CUDA graph */
  int kernel_family;        /* 0: links in registers (rhs_block <= 4);
                               1: links staged in shared memory (up to 16) */
  double ms_stencils;       /* tuner's K1 + K2 time of one iteration with
                               every system running */
} lmb_batch_tuning;

int lmb_cg_ddagd_batched(lmb_ctx *ctx, const lmb_cg_params *params,
                         int nlattices, const lmb_batch_lattice *lattices,
                         lmb_cg_result *results, lmb_batch_tuning *tuning,
                         void *stream);

/* Application rate of an operator on the library's resident fields: no
 * reference counterpart (it replaces the timing loop of
 * benchmark/hisq_dirac_scaling.jl:82-100, which times mul! on one pair of
 * fields).  `in` (padded layout) is packed once; the operator of params->op
 * (kappa / csw / mass / naik_epsilon of params, domain wall as set by
 * lmb_domainwall_set) is then applied 2 + napply times between two internal
 * fields at params->precision, input and output swapped after every
 * application; *ms_per_apply is the device time of the last napply
 * applications divided by napply (CUDA events on `stream`).  Synchronises
 * the stream. */
int lmb_operator_timing(lmb_ctx *ctx, const lmb_cg_params *params,
                        const void *in, int napply, int dagger,
                        double *ms_per_apply, void *stream);

/* Process grid (the reference's Cartesian decomposition,
 * LatticeMatrices_core.jl:350-358, with exchange_dim! :742-921 and the
 * Allreduce of every reduction, LatticeMatrices.jl:1024-1128).  After this
 * call the context's geometry (lmb_set_geometry: local extents L = the
 * block, coords = this rank's grid coordinates) is the block of `rank` in a
 * grid of dims[4] ranks; the dimensions of split_mask (bit mu) exchange
 * faces with the neighbour ranks nb_minus[mu] / nb_plus[mu] over an NCCL
 * communicator created from the 128-byte nccl_id (lmb_nccl_unique_id on one
 * rank, shared by the caller) -- every rank calls it collectively.  A split
 * dimension may hold one rank (its neighbours are itself).  Then the Wilson,
 * Wilson-clover, staggered and HISQ applications and lmb_cg_ddagd run on the
 * block: faces packed by kernels, exchanged on a communication stream while
 * the interior sites are computed, then the boundary sites from the ghost
 * layers; each CG reduction is summed over the ranks (one FP64 all-reduce).
 * The caller's padded links must hold a filled halo (set_halo!) of width >= 1
 * (Wilson, staggered) or 3 (HISQ).  nccl_id NULL releases the grid.  NCCL is
 * loaded at run time (libnccl.so.2); LMB_ERR_UNSUPPORTED without it. */
int lmb_nccl_unique_id(void *id128);
int lmb_set_process_grid(lmb_ctx *ctx, const void *nccl_id, int nranks,
                         int rank, const int dims[4], const int coords[4],
                         unsigned split_mask, const int nb_minus[4],
                         const int nb_plus[4]);

/* dot(a, b) = sum conj(a) b over the core (LinearAlgebras/linearalgebra_D.jl:
 * 3325-3341) of two padded fields with ncomp complex numbers per site.
 * out[0] = Re, out[1] = Im.  Synchronises the stream. */
int lmb_field_dot(lmb_ctx *ctx, const void *a, const void *b, int ncomp,
                  double out[2], void *stream);


/* Seeded synthetic inputs, decomposition independent (Philox4x32-10 site
 * streams as utilities/randomgenerator.jl:247-340):
 * U_mu(x) = reunitarize(exp(i amplitude H)) with H traceless Hermitian
 * Gaussian (normalize_matrix!, LinearAlgebras/linearalgebra_D.jl:2340-2425),
 * written to four padded (3,3,...) fields; and a unit-variance complex
 * Gaussian field with ncomp numbers per site (randomize_gaussian_matrix!,
 * linearalgebra_D.jl:2611-2652; re, im ~ N(0, 1/2) as
 * benchmark/ddagd_cg/README.md:161-162). */
int lmb_random_su3_links(lmb_ctx *ctx, void *const U[4], double amplitude,
                         uint64_t seed, void *stream);
int lmb_gaussian_field(lmb_ctx *ctx, void *out, int ncomp, uint64_t seed,
                       void *stream);


/* Inner product that allocates nothing: no reference counterpart.  The same
 * sum as lmb_field_dot, for callers that cannot call cudaMalloc
 * (pool-managed device memory near its limit, host applications that forbid
 * allocations outside their own allocator, loops where an allocation would
 * synchronise the device).
 * No context: the geometry (L, nw, dtype as in lmb_set_geometry) is passed
 * directly, the result (Re, Im) is written to the device array out_device[2]
 * on `stream`, and nothing synchronises.  ncomp is 1, 3, 9 or 12 complex
 * numbers per site (LMB_ERR_UNSUPPORTED otherwise).  Scratch is a 1 MiB
 * static device array inside the library, so one call takes at most
 * 16,777,216 sites (LMB_ERR_ARG beyond); every call shares it, so calls that
 * overlap on the GPU (unordered streams) race.  Every call looks up the
 * array's device address (cudaGetSymbolAddress, no allocation), so a device
 * reset never leaves a stale address.  Under CUDA's lazy module loading the
 * first call on a device loads the module that holds the array, which takes
 * device memory: make one call per device at initialisation, before a pool
 * allocator fills the device and outside any stream capture. */
int lmb_field_dot_noalloc(const void *a, const void *b, const int L[4],
                          int nw, int dtype, int ncomp, double *out_device,
                          void *stream);

#ifdef __cplusplus
}
#endif
#endif /* LMB200_H */
