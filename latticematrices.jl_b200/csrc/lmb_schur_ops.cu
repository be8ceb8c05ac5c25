// lmb_schur_ops.cu -- even/odd Schur-preconditioned solve of D x = b
// (lmb_solve_evenodd): clover block inverses, parity-ordered copies of the
// links and blocks, and the CG drivers on the Schur operator.
#include "lmb_op_schur.cuh"
#include "lmb_op_wilson.cuh"

using namespace lmb;

namespace lmb {

// A^-1 blocks of the current clover blocks (ensure_clover first)
int ensure_clover_inverse(lmb_ctx *ctx, int prec, cudaStream_t st) {
  CloverCache &cc = ctx->clover, &ci = ctx->clover_inv;
  const int64_t V = ctx->g.V;
  if (!cc.d_valid) return fail(ctx, LMB_ERR_STATE, "clover blocks have not been built");
  if (!ci.d_valid || ci.src_version != cc.d_version) {
    if (!ci.d) LMB_CUDA(ctx, cudaMalloc(&ci.d, sizeof(double2) * 36 * V));
    unsigned *bad = (unsigned *)workspace(ctx, "clover_inv_bad", sizeof(unsigned));
    if (!bad) return fail(ctx, LMB_ERR_CUDA, "out of device memory (clover inverse)");
    LMB_CUDA(ctx, cudaMemsetAsync(bad, 0, sizeof(unsigned), st));
    clover_invert_kernel<<<grid_for(2 * V, 128), 128, 0, st>>>(ci.d, cc.d, V, bad);
    LMB_CHECK_LAUNCH(ctx);
    unsigned hb = 0;
    LMB_CUDA(ctx, cudaMemcpyAsync(&hb, bad, sizeof hb, cudaMemcpyDeviceToHost, st));
    LMB_CUDA(ctx, cudaStreamSynchronize(st));
    if (hb) {
      ci.d_valid = false;
      return fail(ctx, LMB_ERR_ARG, "%u clover blocks are singular: the even/odd solve needs A invertible", hb);
    }
    ci.d_valid = true;
    ci.src_version = cc.d_version;
    ci.d_version++;
  }
  return clover_convert(ctx, ci, prec, st);
}

// or the buffer changes (*stale: an earlier region of the buffer was rebuilt)
template <typename T>
int eo_copy(lmb_ctx *ctx, const std::string &name, size_t bytes, size_t off, const T *src, int nplanes,
            uint64_t version, bool *stale, cudaStream_t st) {
  char *buf = (char *)workspace(ctx, name, bytes);
  if (!buf) return fail(ctx, LMB_ERR_CUDA, "out of device memory (parity-ordered copy)");
  auto it = ctx->eo_tags.find(name);
  if (*stale || it == ctx->eo_tags.end() || it->second.version != version || it->second.V != ctx->g.V ||
      it->second.ptr != buf) {
    *stale = true;
    eo_permute_kernel<T><<<grid_for(ctx->g.V, 256), 256, 0, st>>>((T *)(buf + off), src, nplanes, ctx->g);
    LMB_CHECK_LAUNCH(ctx);
  }
  return LMB_OK;
}
void eo_tag(lmb_ctx *ctx, const std::string &name, uint64_t version) {
  ctx->eo_tags[name] = lmb_ctx::EoTag{version, ctx->g.V, workspace(ctx, name, 0)};
}
const char *eo_buffer(lmb_ctx *ctx, const std::string &name) { return (const char *)workspace(ctx, name, 0); }

// parity-ordered links (thin set) and clover blocks in precision prec
int ensure_eo_copies(lmb_ctx *ctx, int prec, bool clover, cudaStream_t st) {
  const LinkSet &ls = ctx->links[LMB_LINKS_THIN];
  const int64_t V = ctx->g.V;
  const char *tag = prec == PREC_DOUBLE ? "d" : (prec == PREC_SINGLE ? "s" : "h");
  int rc;
  bool stale = false;
  const std::string un = std::string("eo_U_") + tag;
  if (ls.recon(prec)) {
    if (prec == PREC_DOUBLE) rc = eo_copy(ctx, un, sizeof(double2) * 24 * V, 0, ls.d12, 24, ls.version, &stale, st);
    else if (prec == PREC_SINGLE) rc = eo_copy(ctx, un, sizeof(float4) * 12 * V, 0, ls.f12, 12, ls.version, &stale, st);
    else rc = eo_copy(ctx, un, sizeof(int4) * 6 * V, 0, ls.h12, 6, ls.version, &stale, st);
  } else {
    if (prec == PREC_DOUBLE) {
      rc = eo_copy(ctx, un, sizeof(double2) * 36 * V, 0, ls.d, 36, ls.version, &stale, st);
    } else if (prec == PREC_SINGLE) {
      const size_t nb = sizeof(float2) * 36 * V;
      rc = eo_copy(ctx, un, nb, 0, (const float4 *)ls.f, 16, ls.version, &stale, st);
      if (!rc)
        rc = eo_copy(ctx, un, nb, sizeof(float4) * 16 * V, (const float2 *)((const float4 *)ls.f + 16 * V), 4,
                     ls.version, &stale, st);
    } else {
      rc = eo_copy(ctx, un, sizeof(int) * 36 * V, 0, ls.h, 36, ls.version, &stale, st);
    }
  }
  if (rc) return rc;
  eo_tag(ctx, un, ls.version);
  if (!clover) return LMB_OK;
  const CloverCache *caches[2] = {&ctx->clover, &ctx->clover_inv};
  const char *names[2] = {"eo_A_", "eo_Ai_"};
  for (int w = 0; w < 2; w++) {
    const CloverCache &cc = *caches[w];
    const std::string n = std::string(names[w]) + tag;
    stale = false;
    if (prec == PREC_DOUBLE) {
      rc = eo_copy(ctx, n, sizeof(double2) * 36 * V, 0, cc.d, 36, cc.d_version, &stale, st);
    } else if (prec == PREC_SINGLE) {
      rc = eo_copy(ctx, n, sizeof(float4) * 18 * V, 0, cc.f, 18, cc.d_version, &stale, st);
    } else {
      const size_t nb = sizeof(int4) * 8 * V + sizeof(int2) * 2 * V;
      rc = eo_copy(ctx, n, nb, 0, cc.h, 8, cc.d_version, &stale, st);
      if (!rc) rc = eo_copy(ctx, n, nb, sizeof(int4) * 8 * V, cc.ht, 2, cc.d_version, &stale, st);
    }
    if (rc) return rc;
    eo_tag(ctx, n, cc.d_version);
  }
  return LMB_OK;
}


LMB_OP_INSTANCES(, SchurPolicy)

}  // namespace lmb

extern "C" {

int lmb_solve_evenodd(lmb_ctx *ctx, const lmb_cg_params *prm, void *x, const void *b, lmb_cg_result *res,
                      void *stream) {
  if (!ctx_ok(ctx)) return LMB_ERR_ARG;
  if (!prm || !res || !x || !b) return fail(ctx, LMB_ERR_ARG, "null argument");
  if (x == b) return fail(ctx, LMB_ERR_ARG, "fields x and b must not alias");
  if (prm->op != LMB_OP_WILSON && prm->op != LMB_OP_WILSON_CLOVER)
    return fail(ctx, LMB_ERR_ARG, "the even/odd solve takes the Wilson or Wilson-clover operator");
  if (!(prm->rtol >= 0) || !std::isfinite(prm->rtol)) return fail(ctx, LMB_ERR_ARG, "rtol must be finite and nonnegative");
  if (!(prm->atol >= 0) || !std::isfinite(prm->atol)) return fail(ctx, LMB_ERR_ARG, "atol must be finite and nonnegative");
  if (prm->maxiter < 0) return fail(ctx, LMB_ERR_ARG, "maxiter must be nonnegative");
  if (prm->precision != PREC_DOUBLE && !(prm->delta > 0 && prm->delta < 1))
    return fail(ctx, LMB_ERR_ARG, "reliable-update delta must lie in (0, 1)");
  std::memset(res, 0, sizeof *res);
  cudaStream_t st = as_stream(stream);
  const bool clover = prm->op == LMB_OP_WILSON_CLOVER;
  const SchurPolicy op{clover, prm->kappa, prm->csw};
  int rc = op.prepare(ctx, PREC_DOUBLE, st);
  if (rc) return rc;
  const int64_t V = ctx->g.V, Vh = V / 2;
  Field<PREC_DOUBLE, 12> be, bo, tb, bh, y, xe, xo, xf, bf;
  if (!make_field(ctx, "eo_be", be, Vh) || !make_field(ctx, "eo_bo", bo, Vh) || !make_field(ctx, "eo_tb", tb, Vh) ||
      !make_field(ctx, "eo_bh", bh, Vh) || !make_field(ctx, "eo_y", y, Vh) || !make_field(ctx, "eo_xe", xe, Vh) ||
      !make_field(ctx, "eo_xo", xo, Vh))
    return fail(ctx, LMB_ERR_CUDA, "out of device memory (even/odd fields)");
  double *dscal = (double *)workspace(ctx, "eo_scalars", 2 * sizeof(double));
  if (!dscal) return fail(ctx, LMB_ERR_CUDA, "out of device memory (even/odd scalars)");
  if (!ensure_partials(ctx, grid_for(V, 128), 2)) return fail(ctx, LMB_ERR_CUDA, "out of device memory (partials)");
  const unsigned pgrid = grid_for(V, 256);
  if (ctx->dtype == LMB_DTYPE_C128)
    eo_pack_kernel<double2><<<pgrid, 256, 0, st>>>(be, bo, (const double2 *)b, ctx->g, ctx->pd);
  else
    eo_pack_kernel<float2><<<pgrid, 256, 0, st>>>(be, bo, (const float2 *)b, ctx->g, ctx->pd);
  eo_norm2_kernel<<<grid_for(Vh, 256), 256, 0, st>>>(be, bo, Vh, ctx->partials, ctx->counter, dscal);
  LMB_CHECK_LAUNCH(ctx);
  double bb = 0.0;
  LMB_CUDA(ctx, cudaMemcpyAsync(&bb, dscal, sizeof bb, cudaMemcpyDeviceToHost, st));
  LMB_CUDA(ctx, cudaStreamSynchronize(st));
  const double bnorm = std::sqrt(bb);
  const double tol = std::max(prm->atol, prm->rtol * bnorm);
  const bool r12 = ctx->links[LMB_LINKS_THIN].recon(PREC_DOUBLE);
  if (clover)
    rc = r12 ? evenodd_setup_g<true>(ctx, eo_gauge12_view<PREC_DOUBLE>(ctx), prm->kappa, be, bo, tb, bh, st)
             : evenodd_setup_g<true>(ctx, eo_gauge_view<PREC_DOUBLE>(ctx), prm->kappa, be, bo, tb, bh, st);
  else
    rc = r12 ? evenodd_setup_g<false>(ctx, eo_gauge12_view<PREC_DOUBLE>(ctx), prm->kappa, be, bo, tb, bh, st)
             : evenodd_setup_g<false>(ctx, eo_gauge_view<PREC_DOUBLE>(ctx), prm->kappa, be, bo, tb, bh, st);
  if (rc) return rc;
  // CGNE on the Schur system; its residual is the full system's, so the
  // stopping rule is |b - D x| <= max(atol, rtol |b|)
  LMB_CUDA(ctx, cudaMemsetAsync(y.data, 0, Field<PREC_DOUBLE, 12>::bytes(Vh), st));
  lmb_cg_params p2 = *prm;
  p2.rtol = 0.0;
  p2.atol = tol;
  rc = cg_dispatch(ctx, &p2, op, (void *)&y, (const void *)&bh, res, st);
  if (rc) return rc;
  // x_e = Dh^+ y, x_o = A_oo^-1 (b_o + k H_oe x_e)
  {
    EpiStore<PREC_DOUBLE, 12> e{xe, nullptr};
    rc = op.launch<PREC_DOUBLE, 0>(ctx, y, e, st);
    if (rc) return rc;
  }
  if (clover)
    rc = r12 ? evenodd_odd_g<true>(ctx, eo_gauge12_view<PREC_DOUBLE>(ctx), prm->kappa, xe, bo, xo, st)
             : evenodd_odd_g<true>(ctx, eo_gauge_view<PREC_DOUBLE>(ctx), prm->kappa, xe, bo, xo, st);
  else
    rc = r12 ? evenodd_odd_g<false>(ctx, eo_gauge12_view<PREC_DOUBLE>(ctx), prm->kappa, xe, bo, xo, st)
             : evenodd_odd_g<false>(ctx, eo_gauge_view<PREC_DOUBLE>(ctx), prm->kappa, xe, bo, xo, st);
  if (rc) return rc;
  if (ctx->dtype == LMB_DTYPE_C128)
    eo_unpack_kernel<double2><<<pgrid, 256, 0, st>>>((double2 *)x, xe, xo, ctx->g, ctx->pd);
  else
    eo_unpack_kernel<float2><<<pgrid, 256, 0, st>>>((float2 *)x, xe, xo, ctx->g, ctx->pd);
  LMB_CHECK_LAUNCH(ctx);
  // |b - D x| with the full operator in FP64
  if (!make_field(ctx, "eo_xf", xf, V) || !make_field(ctx, "eo_bf", bf, V))
    return fail(ctx, LMB_ERR_CUDA, "out of device memory (even/odd residual)");
  rc = pack_in(ctx, xf, x, st);
  if (rc) return rc;
  rc = pack_in(ctx, bf, b, st);
  if (rc) return rc;
  if (!ensure_partials(ctx, grid_for(V, kDslashThreads), 2))
    return fail(ctx, LMB_ERR_CUDA, "out of device memory (partials)");
  const WilsonPolicy full{prm->op, prm->kappa, prm->csw};
  EpiResidualNorm<12> er{bf, ctx->partials, ctx->counter, dscal + 1};
  rc = full.launch<PREC_DOUBLE, 0>(ctx, xf, er, st);
  if (rc) return rc;
  double rr = 0.0;
  LMB_CUDA(ctx, cudaMemcpyAsync(&rr, dscal + 1, sizeof rr, cudaMemcpyDeviceToHost, st));
  LMB_CUDA(ctx, cudaStreamSynchronize(st));
  const double rn = std::sqrt(rr);
  res->true_residual_norm = rn;
  res->residual_norm = rn;
  res->relative_residual = bnorm > 0 ? rn / bnorm : (rn == 0 ? 0.0 : INFINITY);
  res->converged = res->converged && rn <= tol * (1.0 + 1e-6) + 1e-300;
  if (!res->converged && res->reason == LMB_CG_CONVERGED) res->reason = LMB_CG_MAXIMUM_ITERATIONS;
  res->kernel_launches += 11;
  return LMB_OK;
}


}  // extern "C"
