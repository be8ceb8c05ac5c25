// lmb_op_dw.cuh -- domain-wall (5D) operator policy and its field hooks.
#pragma once
#include "lmb_domainwall.cuh"
#include "lmb_driver.cuh"

namespace lmb {

// generalised / Mobius domain-wall operator on V4 * L5 sites
// (lmb_domainwall_set gives L5, mass, M, a, b, c)
struct DWPolicy {
  static constexpr int NC = 12;
  int prepare(lmb_ctx *ctx, int prec, cudaStream_t st) const {
    if (!ctx->geom_set) return fail(ctx, LMB_ERR_STATE, "lmb_set_geometry has not been called");
    if (!ctx->links[LMB_LINKS_THIN].valid) return fail(ctx, LMB_ERR_STATE, "gauge links have not been uploaded");
    if (ctx->dw_L5 <= 0) return fail(ctx, LMB_ERR_STATE, "lmb_domainwall_set has not been called");
    int rc = check_prec(ctx, prec);
    if (rc) return rc;
    return ensure_link_precision(ctx, ctx->links[LMB_LINKS_THIN], prec, st);
  }
  static bool one_pass(const lmb_ctx *ctx) { return ctx->dw_L5 <= kDslashThreads && !ctx->dw_two_pass; }
  // blocks of the largest launch (the one-pass adjoint holds whole 4D points)
  static int64_t max_blocks(const lmb_ctx *ctx) {
    const int64_t flat = grid_for(ctx->g.V * ctx->dw_L5, kDslashThreads);
    if (!one_pass(ctx)) return flat;
    const int64_t pts = grid_for(ctx->g.V, kDslashThreads / ctx->dw_L5);
    return pts > flat ? pts : flat;
  }
  DWParams params(const lmb_ctx *ctx) const {
    const int L5 = ctx->dw_L5;
    return DWParams{L5, ctx->dw_mass, ctx->dw_M, ctx->dw_coef, ctx->dw_coef + L5, ctx->dw_coef + 2 * L5};
  }
  template <int P, int DAG, class G, class Epi>
  int launch_g(lmb_ctx *ctx, const Field<P, 12> &in, const G &U, const Epi &epi, cudaStream_t st) const {
    typedef typename Real<P>::type R;
    const int64_t V4 = ctx->g.V, V5 = V4 * ctx->dw_L5;
    Field<P, 12> tmp;
    if (!make_field(ctx, P == PREC_DOUBLE ? "dw_tmp_d" : (P == PREC_SINGLE ? "dw_tmp_s" : "dw_tmp_h"), tmp, V5))
      return fail(ctx, LMB_ERR_CUDA, "out of device memory (domain-wall workspace)");
    const DWParams d = params(ctx);
    const unsigned grid = grid_for(V5, kDslashThreads);
    if (one_pass(ctx)) {
      if constexpr (!DAG) {
        dw_forward_kernel<R><<<grid, kDslashThreads, 0, st>>>(ctx->g, in, U, d, epi);
      } else {
        const int npts = kDslashThreads / d.L5;
        dw_adjoint_kernel<R><<<grid_for(V4, npts), kDslashThreads, 0, st>>>(ctx->g, in, U, d, npts, epi);
      }
      LMB_CHECK_LAUNCH(ctx);
      return LMB_OK;
    }
    if constexpr (!DAG) {
      dw_fifth_kernel<P><<<grid, kDslashThreads, 0, st>>>(tmp, in, V4, d, epi);
      dw_stencil_kernel<R, 0, 1><<<grid, kDslashThreads, 0, st>>>(ctx->g, tmp, in, U, d, epi);
    } else {
      const EpiStoreFollow<P, Epi> e1{tmp, epi};
      dw_stencil_kernel<R, 1, 0><<<grid, kDslashThreads, 0, st>>>(ctx->g, in, in, U, d, e1);
      dw_adjoint_local_kernel<R><<<grid, kDslashThreads, 0, st>>>(in, tmp, V4, d, epi);
    }
    LMB_CHECK_LAUNCH(ctx);
    return LMB_OK;
  }
  template <int P, int DAG, class Epi>
  int launch(lmb_ctx *ctx, const Field<P, 12> &in, const Epi &epi, cudaStream_t st) const {
    const LinkSet &ls = ctx->links[LMB_LINKS_THIN];
    if (ls.recon(P)) return launch_g<P, DAG>(ctx, in, gauge12_view<P>(ls, ctx->g.V), epi, st);
    return launch_g<P, DAG>(ctx, in, gauge_view<P>(ls, ctx->g.V), epi, st);
  }
  int link_reals(const lmb_ctx *ctx, int prec) const { return ctx->links[LMB_LINKS_THIN].recon(prec) ? 12 : 18; }
  bool links_finite(const lmb_ctx *ctx) const { return ctx->links[LMB_LINKS_THIN].finite(); }
};

inline int64_t op_volume(const lmb_ctx *ctx, const DWPolicy &) { return ctx->g.V * ctx->dw_L5; }
inline int64_t op_max_blocks(const lmb_ctx *ctx, const DWPolicy &) { return DWPolicy::max_blocks(ctx); }
template <int PS, int NC>
int op_pack_in(lmb_ctx *ctx, const DWPolicy &, Field<PS, NC> &f, const void *src, cudaStream_t st) {
  const unsigned grid = grid_for(ctx->g.V * ctx->dw_L5, 256);
  if (ctx->dtype == LMB_DTYPE_C128)
    pack_field5_kernel<double2, PS, NC><<<grid, 256, 0, st>>>(f, (const double2 *)src, ctx->g, ctx->pd, ctx->dw_L5);
  else
    pack_field5_kernel<float2, PS, NC><<<grid, 256, 0, st>>>(f, (const float2 *)src, ctx->g, ctx->pd, ctx->dw_L5);
  LMB_CHECK_LAUNCH(ctx);
  return LMB_OK;
}
template <int PS, int NC>
int op_unpack_out(lmb_ctx *ctx, const DWPolicy &, void *dst, const Field<PS, NC> &f, cudaStream_t st) {
  const unsigned grid = grid_for(ctx->g.V * ctx->dw_L5, 256);
  if (ctx->dtype == LMB_DTYPE_C128)
    unpack_field5_kernel<double2, PS, NC><<<grid, 256, 0, st>>>((double2 *)dst, f, ctx->g, ctx->pd, ctx->dw_L5);
  else
    unpack_field5_kernel<float2, PS, NC><<<grid, 256, 0, st>>>((float2 *)dst, f, ctx->g, ctx->pd, ctx->dw_L5);
  LMB_CHECK_LAUNCH(ctx);
  return LMB_OK;
}

LMB_OP_INSTANCES(extern, DWPolicy)

}  // namespace lmb
