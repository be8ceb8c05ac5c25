// lmb_force_ops.cu -- HISQ smearing chain (Fat7 / Lepage, U(3) projection,
// Naik), the HISQ and Wilson-clover link pullbacks and fermion forces.
#include "lmb_clover_force.cuh"
#include "lmb_hisq_force.cuh"
#include "lmb_op_staggered.cuh"
#include "lmb_op_wilson.cuh"

using namespace lmb;

namespace lmb {

// V = Fat7(U) with coefficients (c1, c3, c5, c7, cLepage)
int fat7_planes(lmb_ctx *ctx, const double2 *U, double2 *V, const double *coef, cudaStream_t st) {
  const int64_t n = ctx->g.V;
  double2 *work = (double2 *)workspace(ctx, "smear_staples", sizeof(double2) * 54 * n);
  if (!work) return fail(ctx, LMB_ERR_CUDA, "out of device memory (smearing staples)");
  double2 *S3[3] = {work, work + 9 * n, work + 18 * n};
  double2 *S5[3] = {work + 27 * n, work + 36 * n, work + 45 * n};
  const unsigned grid = grid_for(n, kSmearThreads);
  for (int mu = 0; mu < 4; mu++) {
    int axes[3], k = 0;
    for (int d = 0; d < 4; d++)
      if (d != mu) axes[k++] = d;
    const double2 *Umu = U + (size_t)mu * 9 * n;
    double2 *Vmu = V + (size_t)mu * 9 * n;
    for (int slot = 0; slot < 3; slot++)
      staple_transport_kernel<<<grid, kSmearThreads, 0, st>>>(S3[slot], Umu, U, ctx->g, mu, axes[slot], 3, 0, 1.0);
    for (int slot = 0; slot < 3; slot++) {
      const int bs = slot == 0 ? 1 : 0, cs = slot == 2 ? 1 : 2;
      staple_transport_kernel<<<grid, kSmearThreads, 0, st>>>(S5[slot], S3[cs], U, ctx->g, mu, axes[bs], 3, 0, 1.0);
      staple_transport_kernel<<<grid, kSmearThreads, 0, st>>>(S5[slot], S3[bs], U, ctx->g, mu, axes[cs], 3, 1, 1.0);
    }
    fat7_combine_kernel<<<grid_for(9 * n, 256), 256, 0, st>>>(Vmu, Umu, S3[0], S3[1], S3[2], S5[0], S5[1], S5[2],
                                                               n, coef[0], coef[1], coef[2]);
    for (int slot = 0; slot < 3; slot++)
      staple_transport_kernel<<<grid, kSmearThreads, 0, st>>>(Vmu, S5[slot], U, ctx->g, mu, axes[slot], 3, 1,
                                                              coef[3]);
  }
  if (coef[4] != 0.0) lepage_kernel<<<grid_for(4 * n, kSmearThreads), kSmearThreads, 0, st>>>(V, U, ctx->g, coef[4]);
  LMB_CHECK_LAUNCH(ctx);
  return LMB_OK;
}

int project_u3_planes(lmb_ctx *ctx, const double2 *V, double2 *W, cudaStream_t st) {
  u3_project_kernel<<<grid_for(4 * ctx->g.V, kSmearThreads), kSmearThreads, 0, st>>>(W, V, ctx->g.V);
  LMB_CHECK_LAUNCH(ctx);
  return LMB_OK;
}

int naik_planes(lmb_ctx *ctx, const double2 *W, double2 *L, cudaStream_t st) {
  naik_kernel<<<grid_for(4 * ctx->g.V, kSmearThreads), kSmearThreads, 0, st>>>(L, W, ctx->g);
  LMB_CHECK_LAUNCH(ctx);
  return LMB_OK;
}

// install 36-plane links as a link set of the context (derived, not uploaded)
int install_links(lmb_ctx *ctx, int which, const double2 *planes, cudaStream_t st) {
  LinkSet &ls = ctx->links[which];
  const int64_t V = ctx->g.V;
  if (!ls.d) LMB_CUDA(ctx, cudaMalloc(&ls.d, sizeof(double2) * 36 * V));
  LMB_CUDA(ctx, cudaMemcpyAsync(ls.d, planes, sizeof(double2) * 36 * V, cudaMemcpyDeviceToDevice, st));
  int rc;
  ls.scale = device_absmax(ctx, ls.d, 36 * V, st, &rc);
  if (rc) return rc;
  ls.su3_dev = 1.0;  // smeared links are not SU(3): never reconstruct
  for (int mu = 0; mu < 4; mu++) {
    ls.ptr[mu] = nullptr;
    ls.epoch[mu] = 0;
  }
  ls.valid = true;
  ls.version++;
  return LMB_OK;
}

// ---------------------------------------------------------------------------
// HISQ force: reverse pass of the factorised Fat7 with staple recomputation
// ---------------------------------------------------------------------------
int fat7_pullback_planes(lmb_ctx *ctx, const double2 *U, const double2 *dV, double2 *dU, const double *coef,
                         cudaStream_t st) {
  const int64_t n = ctx->g.V;
  double2 *work = (double2 *)workspace(ctx, "force_staples", sizeof(double2) * 9 * 16 * n);
  if (!work) return fail(ctx, LMB_ERR_CUDA, "out of device memory (force staples)");
  double2 *S3[3], *S5[3], *dS3[3], *dS5[3];
  for (int i = 0; i < 3; i++) {
    S3[i] = work + (size_t)(0 + i) * 9 * n;
    S5[i] = work + (size_t)(3 + i) * 9 * n;
    dS3[i] = work + (size_t)(6 + i) * 9 * n;
    dS5[i] = work + (size_t)(9 + i) * 9 * n;
  }
  double2 *Pp = work + (size_t)12 * 9 * n, *Pm = work + (size_t)13 * 9 * n;
  double2 *dPp = work + (size_t)14 * 9 * n, *dPm = work + (size_t)15 * 9 * n;
  const Geom &g = ctx->g;
  const unsigned grid = grid_for(n, kSmearThreads), ag = grid_for(9 * n, 256);
  const double c1 = coef[0], c3 = coef[1], c5 = coef[2], c7 = coef[3], cL = coef[4];
  for (int mu = 0; mu < 4; mu++) {
    int axes[3], k = 0;
    for (int d = 0; d < 4; d++)
      if (d != mu) axes[k++] = d;
    const double2 *Umu = U + (size_t)mu * 9 * n;
    const double2 *dVmu = dV + (size_t)mu * 9 * n;
    double2 *dUmu = dU + (size_t)mu * 9 * n;
    // recompute the staples of this direction
    for (int sl = 0; sl < 3; sl++)
      staple_transport_kernel<<<grid, kSmearThreads, 0, st>>>(S3[sl], Umu, U, g, mu, axes[sl], 3, 0, 1.0);
    for (int sl = 0; sl < 3; sl++) {
      const int bs = sl == 0 ? 1 : 0, cs = sl == 2 ? 1 : 2;
      staple_transport_kernel<<<grid, kSmearThreads, 0, st>>>(S5[sl], S3[cs], U, g, mu, axes[bs], 3, 0, 1.0);
      staple_transport_kernel<<<grid, kSmearThreads, 0, st>>>(S5[sl], S3[bs], U, g, mu, axes[cs], 3, 1, 1.0);
    }
    // seven-link terms c7 T_a(S5_a), and the five-link cotangents
    for (int sl = 0; sl < 3; sl++) {
      staple_transport_kernel<<<grid, kSmearThreads, 0, st>>>(dS5[sl], dVmu, U, g, mu, axes[sl], 3, 0, c7);
      axpy_c_kernel<<<ag, 256, 0, st>>>(dS5[sl], dVmu, c5, 9 * n, 1);
      transport_link_grad_kernel<<<grid, kSmearThreads, 0, st>>>(dU, dVmu, S5[sl], U, g, mu, axes[sl], 3, c7);
    }
    for (int sl = 0; sl < 3; sl++) axpy_c_kernel<<<ag, 256, 0, st>>>(dS3[sl], dVmu, c3, 9 * n, 0);
    // five-link terms S5_a = T_b(S3_c) + T_c(S3_b)
    for (int sl = 0; sl < 3; sl++) {
      const int bs = sl == 0 ? 1 : 0, cs = sl == 2 ? 1 : 2;
      staple_transport_kernel<<<grid, kSmearThreads, 0, st>>>(dS3[cs], dS5[sl], U, g, mu, axes[bs], 3, 1, 1.0);
      transport_link_grad_kernel<<<grid, kSmearThreads, 0, st>>>(dU, dS5[sl], S3[cs], U, g, mu, axes[bs], 3, 1.0);
      staple_transport_kernel<<<grid, kSmearThreads, 0, st>>>(dS3[bs], dS5[sl], U, g, mu, axes[cs], 3, 1, 1.0);
      transport_link_grad_kernel<<<grid, kSmearThreads, 0, st>>>(dU, dS5[sl], S3[bs], U, g, mu, axes[cs], 3, 1.0);
    }
    // three-link terms S3_nu = T_nu(U_mu)
    for (int sl = 0; sl < 3; sl++) {
      staple_transport_kernel<<<grid, kSmearThreads, 0, st>>>(dUmu, dS3[sl], U, g, mu, axes[sl], 3, 1, 1.0);
      transport_link_grad_kernel<<<grid, kSmearThreads, 0, st>>>(dU, dS3[sl], Umu, U, g, mu, axes[sl], 3, 1.0);
    }
    axpy_c_kernel<<<ag, 256, 0, st>>>(dUmu, dVmu, c1, 9 * n, 1);
    // Lepage: T+_nu(T+_nu(U_mu)) + T-_nu(T-_nu(U_mu)); the adjoint of T+ is T-
    if (cL != 0.0) {
      for (int sl = 0; sl < 3; sl++) {
        const int nu = axes[sl];
        staple_transport_kernel<<<grid, kSmearThreads, 0, st>>>(Pp, Umu, U, g, mu, nu, 1, 0, 1.0);
        staple_transport_kernel<<<grid, kSmearThreads, 0, st>>>(Pm, Umu, U, g, mu, nu, 2, 0, 1.0);
        staple_transport_kernel<<<grid, kSmearThreads, 0, st>>>(dPp, dVmu, U, g, mu, nu, 2, 0, cL);
        staple_transport_kernel<<<grid, kSmearThreads, 0, st>>>(dPm, dVmu, U, g, mu, nu, 1, 0, cL);
        transport_link_grad_kernel<<<grid, kSmearThreads, 0, st>>>(dU, dVmu, Pp, U, g, mu, nu, 1, cL);
        transport_link_grad_kernel<<<grid, kSmearThreads, 0, st>>>(dU, dVmu, Pm, U, g, mu, nu, 2, cL);
        staple_transport_kernel<<<grid, kSmearThreads, 0, st>>>(dUmu, dPp, U, g, mu, nu, 2, 1, 1.0);
        staple_transport_kernel<<<grid, kSmearThreads, 0, st>>>(dUmu, dPm, U, g, mu, nu, 1, 1, 1.0);
        transport_link_grad_kernel<<<grid, kSmearThreads, 0, st>>>(dU, dPp, Umu, U, g, mu, nu, 1, 1.0);
        transport_link_grad_kernel<<<grid, kSmearThreads, 0, st>>>(dU, dPm, Umu, U, g, mu, nu, 2, 1.0);
      }
    }
  }
  LMB_CHECK_LAUNCH(ctx);
  return LMB_OK;
}

// dU_planes += d/dU [coef Re<dr, D_HISQ(U) psi>] through the whole chain
int hisq_pullback_planes(lmb_ctx *ctx, const double2 *thin, const Field<PREC_DOUBLE, 3> &dr,
                         const Field<PREC_DOUBLE, 3> &psi, double naik_epsilon, double coefficient, double2 *dU,
                         cudaStream_t st) {
  const int64_t n = ctx->g.V;
  const size_t L36 = sizeof(double2) * 36 * n;
  double2 *V1 = (double2 *)workspace(ctx, "force_V1", L36), *W = (double2 *)workspace(ctx, "force_W", L36);
  double2 *dX = (double2 *)workspace(ctx, "force_dX", L36), *dL = (double2 *)workspace(ctx, "force_dL", L36);
  double2 *dW = (double2 *)workspace(ctx, "force_dW", L36), *dV1 = (double2 *)workspace(ctx, "force_dV1", L36);
  if (!V1 || !W || !dX || !dL || !dW || !dV1) return fail(ctx, LMB_ERR_CUDA, "out of device memory (force)");
  const double c_level1[5] = {1.0 / 8, 1.0 / 16, 1.0 / 64, 1.0 / 384, 0.0};
  const double c_level2[5] = {1.0 + naik_epsilon / 8, 1.0 / 16, 1.0 / 64, 1.0 / 384, -1.0 / 8};
  int rc;
  // recompute the smearing levels the pullback needs
  if ((rc = fat7_planes(ctx, thin, V1, c_level1, st))) return rc;
  if ((rc = project_u3_planes(ctx, V1, W, st))) return rc;
  // Dirac outer products
  const double fc = coefficient / 2, lc = -coefficient * (1.0 + naik_epsilon) / 48.0;
  hisq_outer_product_kernel<<<grid_for(n, kSmearThreads), kSmearThreads, 0, st>>>(dX, dL, dr, psi, ctx->g, fc, lc);
  LMB_CHECK_LAUNCH(ctx);
  // Naik and level-2 Fat7 -> dW
  LMB_CUDA(ctx, cudaMemsetAsync(dW, 0, L36, st));
  naik_pullback_kernel<<<grid_for(4 * n, kSmearThreads), kSmearThreads, 0, st>>>(dW, dL, W, ctx->g);
  LMB_CHECK_LAUNCH(ctx);
  if ((rc = fat7_pullback_planes(ctx, W, dX, dW, c_level2, st))) return rc;
  // U(3) projection -> dV1
  LMB_CUDA(ctx, cudaMemsetAsync(dV1, 0, L36, st));
  u3_pullback_kernel<<<grid_for(4 * n, 64), 64, 0, st>>>(dV1, dW, V1, n);
  LMB_CHECK_LAUNCH(ctx);
  // level-1 Fat7 -> thin links
  return fat7_pullback_planes(ctx, thin, dV1, dU, c_level1, st);
}

// grad (36 planes) += d/dU [coef Re<dr, D_clover(U) psi>]
int clover_pullback_planes(lmb_ctx *ctx, const double2 *thin, const Field<PREC_DOUBLE, 12> &dr,
                           const Field<PREC_DOUBLE, 12> &psi, double kappa, double csw, double coefficient,
                           double2 *grad, cudaStream_t st) {
  const int64_t n = ctx->g.V;
  wilson_outer_product_kernel<<<grid_for(n, 128), 128, 0, st>>>(grad, dr, psi, ctx->g, -kappa * coefficient);
  LMB_CHECK_LAUNCH(ctx);
  if (csw == 0.0) return LMB_OK;
  double2 *dF = (double2 *)workspace(ctx, "force_dF", sizeof(double2) * 54 * n);
  if (!dF) return fail(ctx, LMB_ERR_CUDA, "out of device memory (clover force)");
  clover_cotangent_kernel<<<grid_for(n, 128), 128, 0, st>>>(dF, dr, psi, ctx->g, -kappa * csw * coefficient);
  LMB_CHECK_LAUNCH(ctx);
  static const int pmu[6] = {0, 0, 0, 1, 1, 2}, pnu[6] = {1, 2, 3, 2, 3, 3};
  for (int plane = 0; plane < 6; plane++) {
    clover_link_pullback_kernel<<<grid_for(n, 64), 64, 0, st>>>(grad, thin, dF, ctx->g, plane, pmu[plane],
                                                                 pnu[plane]);
    LMB_CHECK_LAUNCH(ctx);
  }
  return LMB_OK;
}

int accumulate_links_to(lmb_ctx *ctx, void *const dU[4], const double2 *planes, cudaStream_t st) {
  const unsigned grid = grid_for(ctx->g.V, 256);
  if (ctx->dtype == LMB_DTYPE_C128)
    accumulate_links_kernel<double2><<<grid, 256, 0, st>>>((double2 *)dU[0], (double2 *)dU[1], (double2 *)dU[2],
                                                            (double2 *)dU[3], planes, ctx->g, ctx->pd);
  else
    accumulate_links_kernel<float2><<<grid, 256, 0, st>>>((float2 *)dU[0], (float2 *)dU[1], (float2 *)dU[2],
                                                           (float2 *)dU[3], planes, ctx->g, ctx->pd);
  LMB_CHECK_LAUNCH(ctx);
  return LMB_OK;
}


}  // namespace lmb

extern "C" {

int lmb_hisq_fat7(lmb_ctx *ctx, const void *const U[4], const double coefficients[5], void *const V[4],
                  void *stream) {
  if (!ctx_ok(ctx)) return LMB_ERR_ARG;
  if (!ctx->geom_set) return fail(ctx, LMB_ERR_STATE, "lmb_set_geometry has not been called");
  int rc = check_links_arg(ctx, U, "input link");
  if (rc) return rc;
  if ((rc = check_links_arg(ctx, (const void *const *)V, "output link"))) return rc;
  if (!coefficients) return fail(ctx, LMB_ERR_ARG, "null coefficients");
  cudaStream_t st = as_stream(stream);
  const int64_t n = ctx->g.V;
  double2 *in = (double2 *)workspace(ctx, "smear_in", sizeof(double2) * 36 * n);
  double2 *out = (double2 *)workspace(ctx, "smear_out", sizeof(double2) * 36 * n);
  if (!in || !out) return fail(ctx, LMB_ERR_CUDA, "out of device memory (smearing)");
  if ((rc = pack_links_to(ctx, in, U, st))) return rc;
  if ((rc = fat7_planes(ctx, in, out, coefficients, st))) return rc;
  return unpack_links_from(ctx, V, out, st);
}

int lmb_hisq_project_u3(lmb_ctx *ctx, const void *const V[4], void *const W[4], void *stream) {
  if (!ctx_ok(ctx)) return LMB_ERR_ARG;
  if (!ctx->geom_set) return fail(ctx, LMB_ERR_STATE, "lmb_set_geometry has not been called");
  int rc = check_links_arg(ctx, V, "input link");
  if (rc) return rc;
  if ((rc = check_links_arg(ctx, (const void *const *)W, "output link"))) return rc;
  cudaStream_t st = as_stream(stream);
  const int64_t n = ctx->g.V;
  double2 *in = (double2 *)workspace(ctx, "smear_in", sizeof(double2) * 36 * n);
  double2 *out = (double2 *)workspace(ctx, "smear_out", sizeof(double2) * 36 * n);
  if (!in || !out) return fail(ctx, LMB_ERR_CUDA, "out of device memory (smearing)");
  if ((rc = pack_links_to(ctx, in, V, st))) return rc;
  if ((rc = project_u3_planes(ctx, in, out, st))) return rc;
  return unpack_links_from(ctx, W, out, st);
}

int lmb_hisq_naik(lmb_ctx *ctx, const void *const W[4], void *const L[4], void *stream) {
  if (!ctx_ok(ctx)) return LMB_ERR_ARG;
  if (!ctx->geom_set) return fail(ctx, LMB_ERR_STATE, "lmb_set_geometry has not been called");
  int rc = check_links_arg(ctx, W, "input link");
  if (rc) return rc;
  if ((rc = check_links_arg(ctx, (const void *const *)L, "output link"))) return rc;
  cudaStream_t st = as_stream(stream);
  const int64_t n = ctx->g.V;
  double2 *in = (double2 *)workspace(ctx, "smear_in", sizeof(double2) * 36 * n);
  double2 *out = (double2 *)workspace(ctx, "smear_out", sizeof(double2) * 36 * n);
  if (!in || !out) return fail(ctx, LMB_ERR_CUDA, "out of device memory (smearing)");
  if ((rc = pack_links_to(ctx, in, W, st))) return rc;
  if ((rc = naik_planes(ctx, in, out, st))) return rc;
  return unpack_links_from(ctx, L, out, st);
}

int lmb_hisq_links_from_thin(lmb_ctx *ctx, const void *const U[4], const uint64_t epoch[4], double naik_epsilon,
                             void *const X[4], void *const L[4], void *stream) {
  if (!ctx_ok(ctx)) return LMB_ERR_ARG;
  if (!ctx->geom_set) return fail(ctx, LMB_ERR_STATE, "lmb_set_geometry has not been called");
  int rc = check_links_arg(ctx, U, "thin link");
  if (rc) return rc;
  if (!std::isfinite(naik_epsilon)) return fail(ctx, LMB_ERR_ARG, "naik_epsilon must be finite");
  cudaStream_t st = as_stream(stream);
  lmb_smear_key &key = ctx->smear;
  bool same = key.valid && key.naik_epsilon == naik_epsilon && ctx->links[LMB_LINKS_FAT].valid &&
              ctx->links[LMB_LINKS_LONG].valid && epoch;
  for (int mu = 0; mu < 4 && same; mu++) same = key.ptr[mu] == U[mu] && key.epoch[mu] == epoch[mu];
  const int64_t n = ctx->g.V;
  if (!same) {
    double2 *thin = (double2 *)workspace(ctx, "smear_thin", sizeof(double2) * 36 * n);
    double2 *lvl1 = (double2 *)workspace(ctx, "smear_lvl1", sizeof(double2) * 36 * n);
    double2 *w = (double2 *)workspace(ctx, "smear_w", sizeof(double2) * 36 * n);
    double2 *xo = (double2 *)workspace(ctx, "smear_out", sizeof(double2) * 36 * n);
    if (!thin || !lvl1 || !w || !xo) return fail(ctx, LMB_ERR_CUDA, "out of device memory (smearing)");
    // hisq_links_from_thin! (HISQFullSmearing.jl:284-293)
    const double c_level1[5] = {1.0 / 8, 1.0 / 16, 1.0 / 64, 1.0 / 384, 0.0};
    const double c_level2[5] = {1.0 + naik_epsilon / 8, 1.0 / 16, 1.0 / 64, 1.0 / 384, -1.0 / 8};
    if ((rc = pack_links_to(ctx, thin, U, st))) return rc;
    if ((rc = fat7_planes(ctx, thin, lvl1, c_level1, st))) return rc;
    if ((rc = project_u3_planes(ctx, lvl1, w, st))) return rc;
    if ((rc = fat7_planes(ctx, w, xo, c_level2, st))) return rc;
    if ((rc = install_links(ctx, LMB_LINKS_FAT, xo, st))) return rc;
    if ((rc = naik_planes(ctx, w, xo, st))) return rc;
    if ((rc = install_links(ctx, LMB_LINKS_LONG, xo, st))) return rc;
    for (int mu = 0; mu < 4; mu++) {
      key.ptr[mu] = U[mu];
      key.epoch[mu] = epoch ? epoch[mu] : 0;
    }
    key.naik_epsilon = naik_epsilon;
    key.valid = epoch != nullptr;
  }
  if (X) {
    if ((rc = check_links_arg(ctx, (const void *const *)X, "fat link"))) return rc;
    if ((rc = unpack_links_from(ctx, X, ctx->links[LMB_LINKS_FAT].d, st))) return rc;
  }
  if (L) {
    if ((rc = check_links_arg(ctx, (const void *const *)L, "long link"))) return rc;
    if ((rc = unpack_links_from(ctx, L, ctx->links[LMB_LINKS_LONG].d, st))) return rc;
  }
  return LMB_OK;
}


int lmb_hisq_link_pullback(lmb_ctx *ctx, const void *const U[4], double naik_epsilon, double coefficient,
                           const void *result_cotangent, const void *psi, void *const dU[4], void *stream) {
  if (!ctx_ok(ctx)) return LMB_ERR_ARG;
  if (!ctx->geom_set) return fail(ctx, LMB_ERR_STATE, "lmb_set_geometry has not been called");
  int rc = check_links_arg(ctx, U, "thin link");
  if (rc) return rc;
  if ((rc = check_links_arg(ctx, (const void *const *)dU, "thin-link cotangent"))) return rc;
  if (!result_cotangent || !psi) return fail(ctx, LMB_ERR_ARG, "null fermion field");
  if (!std::isfinite(naik_epsilon) || !std::isfinite(coefficient))
    return fail(ctx, LMB_ERR_ARG, "naik_epsilon and coefficient must be finite");
  for (int mu = 0; mu < 4; mu++)
    for (int nu = 0; nu < 4; nu++)
      if (dU[mu] == U[nu]) return fail(ctx, LMB_ERR_ARG, "HISQ thin-link cotangents must not alias primal links");
  cudaStream_t st = as_stream(stream);
  const int64_t n = ctx->g.V;
  double2 *thin = (double2 *)workspace(ctx, "force_thin", sizeof(double2) * 36 * n);
  double2 *grad = (double2 *)workspace(ctx, "force_grad", sizeof(double2) * 36 * n);
  Field<PREC_DOUBLE, 3> dr, ps;
  if (!thin || !grad || !make_field(ctx, "force_dr", dr) || !make_field(ctx, "force_psi", ps))
    return fail(ctx, LMB_ERR_CUDA, "out of device memory (force)");
  if ((rc = pack_links_to(ctx, thin, U, st))) return rc;
  if ((rc = pack_in(ctx, dr, result_cotangent, st))) return rc;
  if ((rc = pack_in(ctx, ps, psi, st))) return rc;
  LMB_CUDA(ctx, cudaMemsetAsync(grad, 0, sizeof(double2) * 36 * n, st));
  if ((rc = hisq_pullback_planes(ctx, thin, dr, ps, naik_epsilon, coefficient, grad, st))) return rc;
  return accumulate_links_to(ctx, dU, grad, st);
}

int lmb_hisq_fermion_force(lmb_ctx *ctx, const void *const U[4], const uint64_t epoch[4], double mass,
                           double naik_epsilon, const void *phi, void *const dU[4], const lmb_cg_params *cg,
                           lmb_cg_result *result, void *stream) {
  if (!ctx_ok(ctx)) return LMB_ERR_ARG;
  if (!ctx->geom_set) return fail(ctx, LMB_ERR_STATE, "lmb_set_geometry has not been called");
  if (!cg || !result || !phi) return fail(ctx, LMB_ERR_ARG, "null argument");
  int rc = check_links_arg(ctx, U, "thin link");
  if (rc) return rc;
  if ((rc = check_links_arg(ctx, (const void *const *)dU, "force"))) return rc;
  cudaStream_t st = as_stream(stream);
  // fat / long links for the solve (cached by thin-link pointer + epoch)
  if ((rc = lmb_hisq_links_from_thin(ctx, U, epoch, naik_epsilon, nullptr, nullptr, stream))) return rc;
  // eta = (D^+D)^-1 phi, chi = D eta, in padded scratch fields of the context geometry
  size_t padded = 3;
  for (int mu = 0; mu < 4; mu++) padded *= (size_t)ctx->pd.P[mu];
  const size_t elem = ctx->dtype == LMB_DTYPE_C128 ? 16 : 8;
  void *eta = workspace(ctx, "force_eta", padded * elem), *chi = workspace(ctx, "force_chi", padded * elem);
  if (!eta || !chi) return fail(ctx, LMB_ERR_CUDA, "out of device memory (force fields)");
  LMB_CUDA(ctx, cudaMemsetAsync(eta, 0, padded * elem, st));
  lmb_cg_params prm = *cg;
  prm.op = LMB_OP_HISQ;
  prm.mass = mass;
  prm.naik_epsilon = naik_epsilon;
  if ((rc = lmb_cg_ddagd(ctx, &prm, eta, phi, result, stream))) return rc;
  if ((rc = apply_dispatch(ctx, StaggeredPolicy{true, mass, naik_epsilon}, chi, eta, 0, PREC_DOUBLE, stream))) return rc;
  // dS/dU = -2 d/dU Re<chi, D(U) eta> with chi, eta fixed (dSFdU,
  // ext/LatticeMatricesEnzymeExt.jl:387-460)
  return lmb_hisq_link_pullback(ctx, U, naik_epsilon, -2.0, chi, eta, dU, stream);
}

int lmb_wilson_clover_link_pullback(lmb_ctx *ctx, const void *const U[4], double kappa, double csw,
                                    double coefficient, const void *result_cotangent, const void *psi,
                                    void *const dU[4], void *stream) {
  if (!ctx_ok(ctx)) return LMB_ERR_ARG;
  if (!ctx->geom_set) return fail(ctx, LMB_ERR_STATE, "lmb_set_geometry has not been called");
  int rc = check_links_arg(ctx, U, "primal link");
  if (rc) return rc;
  if ((rc = check_links_arg(ctx, (const void *const *)dU, "link cotangent"))) return rc;
  if (!result_cotangent || !psi) return fail(ctx, LMB_ERR_ARG, "null fermion field");
  if (!std::isfinite(kappa) || !std::isfinite(csw) || !std::isfinite(coefficient))
    return fail(ctx, LMB_ERR_ARG, "kappa, cSW and coefficient must be finite");
  for (int mu = 0; mu < 4; mu++)
    for (int nu = 0; nu < 4; nu++)
      if (dU[mu] == U[nu])
        return fail(ctx, LMB_ERR_ARG, "Wilson--clover link cotangents must not alias primal links");
  cudaStream_t st = as_stream(stream);
  const int64_t n = ctx->g.V;
  double2 *thin = (double2 *)workspace(ctx, "force_thin", sizeof(double2) * 36 * n);
  double2 *grad = (double2 *)workspace(ctx, "force_grad", sizeof(double2) * 36 * n);
  Field<PREC_DOUBLE, 12> dr, ps;
  if (!thin || !grad || !make_field(ctx, "force_dr12", dr) || !make_field(ctx, "force_psi12", ps))
    return fail(ctx, LMB_ERR_CUDA, "out of device memory (force)");
  if ((rc = pack_links_to(ctx, thin, U, st))) return rc;
  if ((rc = pack_in(ctx, dr, result_cotangent, st))) return rc;
  if ((rc = pack_in(ctx, ps, psi, st))) return rc;
  LMB_CUDA(ctx, cudaMemsetAsync(grad, 0, sizeof(double2) * 36 * n, st));
  if ((rc = clover_pullback_planes(ctx, thin, dr, ps, kappa, csw, coefficient, grad, st))) return rc;
  return accumulate_links_to(ctx, dU, grad, st);
}

int lmb_wilson_clover_fermion_force(lmb_ctx *ctx, const void *const U[4], const uint64_t epoch[4], double kappa,
                                    double csw, const void *phi, void *const dU[4], const lmb_cg_params *cg,
                                    lmb_cg_result *result, void *stream) {
  if (!ctx_ok(ctx)) return LMB_ERR_ARG;
  if (!ctx->geom_set) return fail(ctx, LMB_ERR_STATE, "lmb_set_geometry has not been called");
  if (!cg || !result || !phi || !epoch) return fail(ctx, LMB_ERR_ARG, "null argument");
  int rc = check_links_arg(ctx, U, "primal link");
  if (rc) return rc;
  if ((rc = check_links_arg(ctx, (const void *const *)dU, "force"))) return rc;
  cudaStream_t st = as_stream(stream);
  if ((rc = lmb_links_upload(ctx, LMB_LINKS_THIN, U, epoch, stream))) return rc;
  // eta = (D^+D)^-1 phi, chi = D eta, in padded scratch fields of the context geometry
  size_t padded = 12;
  for (int mu = 0; mu < 4; mu++) padded *= (size_t)ctx->pd.P[mu];
  const size_t elem = ctx->dtype == LMB_DTYPE_C128 ? 16 : 8;
  void *eta = workspace(ctx, "force_eta12", padded * elem), *chi = workspace(ctx, "force_chi12", padded * elem);
  if (!eta || !chi) return fail(ctx, LMB_ERR_CUDA, "out of device memory (force fields)");
  LMB_CUDA(ctx, cudaMemsetAsync(eta, 0, padded * elem, st));
  lmb_cg_params prm = *cg;
  prm.op = csw != 0.0 ? LMB_OP_WILSON_CLOVER : LMB_OP_WILSON;
  prm.kappa = kappa;
  prm.csw = csw;
  if ((rc = lmb_cg_ddagd(ctx, &prm, eta, phi, result, stream))) return rc;
  if ((rc = apply_dispatch(ctx, WilsonPolicy{prm.op, kappa, csw}, chi, eta, 0, PREC_DOUBLE, stream))) return rc;
  // dS/dU = -2 d/dU Re<chi, D(U) eta> with chi, eta fixed
  return lmb_wilson_clover_link_pullback(ctx, U, kappa, csw, -2.0, chi, eta, dU, stream);
}


}  // extern "C"
