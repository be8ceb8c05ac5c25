// lmb_op_schur.cuh -- even/odd Schur operator policy, its views of the
// parity-ordered caches and the setup / reconstruction launches.
#pragma once
#include "lmb_evenodd.cuh"
#include "lmb_driver.cuh"

namespace lmb {

template <int P> Gauge<P> eo_gauge_view(lmb_ctx *ctx);
template <> inline Gauge<PREC_DOUBLE> eo_gauge_view<PREC_DOUBLE>(lmb_ctx *ctx) {
  return {(const double2 *)eo_buffer(ctx, "eo_U_d"), ctx->g.V, ctx->links[LMB_LINKS_THIN].scale};
}
template <> inline Gauge<PREC_SINGLE> eo_gauge_view<PREC_SINGLE>(lmb_ctx *ctx) {
  return {(const float4 *)eo_buffer(ctx, "eo_U_s"), ctx->g.V, ctx->links[LMB_LINKS_THIN].scale};
}
template <> inline Gauge<PREC_HALF> eo_gauge_view<PREC_HALF>(lmb_ctx *ctx) {
  return {(const int *)eo_buffer(ctx, "eo_U_h"), ctx->g.V,
          base_of_exponent(pow2_exponent(ctx->links[LMB_LINKS_THIN].scale))};
}
template <int P> Gauge12<P> eo_gauge12_view(lmb_ctx *ctx);
template <> inline Gauge12<PREC_DOUBLE> eo_gauge12_view<PREC_DOUBLE>(lmb_ctx *ctx) {
  return {(const double2 *)eo_buffer(ctx, "eo_U_d"), ctx->g.V, 1.f};
}
template <> inline Gauge12<PREC_SINGLE> eo_gauge12_view<PREC_SINGLE>(lmb_ctx *ctx) {
  return {(const float4 *)eo_buffer(ctx, "eo_U_s"), ctx->g.V, 1.f};
}
template <> inline Gauge12<PREC_HALF> eo_gauge12_view<PREC_HALF>(lmb_ctx *ctx) {
  return {(const int4 *)eo_buffer(ctx, "eo_U_h"), ctx->g.V, 1.f};
}
template <int P> Clover<P> eo_clover_view(lmb_ctx *ctx, int inverse);
template <> inline Clover<PREC_DOUBLE> eo_clover_view<PREC_DOUBLE>(lmb_ctx *ctx, int inverse) {
  return {(const double2 *)eo_buffer(ctx, inverse ? "eo_Ai_d" : "eo_A_d"), ctx->g.V, 1.f};
}
template <> inline Clover<PREC_SINGLE> eo_clover_view<PREC_SINGLE>(lmb_ctx *ctx, int inverse) {
  return {(const float4 *)eo_buffer(ctx, inverse ? "eo_Ai_s" : "eo_A_s"), ctx->g.V, 1.f};
}
template <> inline Clover<PREC_HALF> eo_clover_view<PREC_HALF>(lmb_ctx *ctx, int inverse) {
  Clover<PREC_HALF> c;
  const char *buf = eo_buffer(ctx, inverse ? "eo_Ai_h" : "eo_A_h");
  c.data = (const int4 *)buf;
  c.tail = buf ? (const int2 *)(buf + sizeof(int4) * 8 * ctx->g.V) : nullptr;
  c.V = ctx->g.V;
  c.scale = (inverse ? ctx->clover_inv : ctx->clover).scale;
  return c;
}

// even/odd Schur operator Dh = A_ee - k^2 H_eo A_oo^-1 H_oe on the V/2 even
// sites (checkerboard order), as the CG driver sees it: launch<P, 0> applies
// Dh^+ and launch<P, 1> applies Dh, so the CG solves
// Dh Dh^+ y = bh (CGNE).  Two kernels per application: t_o = A_oo^-1 H_oe in
// (A^-1 applied in the hop kernel), then A_ee in - k^2 H_eo t_o with the
// CG epilogue.
struct SchurPolicy {
  static constexpr int NC = 12;
  bool clover;
  double kappa, csw;
  int prepare(lmb_ctx *ctx, int prec, cudaStream_t st) const {
    if (!ctx->geom_set) return fail(ctx, LMB_ERR_STATE, "lmb_set_geometry has not been called");
    if (!ctx->links[LMB_LINKS_THIN].valid) return fail(ctx, LMB_ERR_STATE, "gauge links have not been uploaded");
    for (int mu = 0; mu < 4; mu++)
      if (ctx->g.L[mu] % 2)
        return fail(ctx, LMB_ERR_ARG, "even/odd preconditioning needs even lattice extents; dimension %d has %d",
                    mu + 1, ctx->g.L[mu]);
    int rc = check_prec(ctx, prec);
    if (rc) return rc;
    rc = ensure_link_precision(ctx, ctx->links[LMB_LINKS_THIN], prec, st);
    if (rc) return rc;
    if (clover) {
      rc = ensure_clover(ctx, -kappa * csw, PREC_DOUBLE, st);
      if (rc) return rc;
      rc = ensure_clover(ctx, -kappa * csw, prec, st);
      if (rc) return rc;
      rc = ensure_clover_inverse(ctx, prec, st);
      if (rc) return rc;
    }
    return ensure_eo_copies(ctx, prec, clover, st);
  }
  template <int P, bool CL, int DAG, class G, class Epi>
  void launch_cl(lmb_ctx *ctx, const Field<P, 12> &in, const Field<P, 12> &t, const G &U, const Epi &epi,
                 cudaStream_t st) const {
    typedef typename Real<P>::type R;
    const Clover<P> A = eo_clover_view<P>(ctx, 0), Ai = eo_clover_view<P>(ctx, 1);
    const unsigned grid = grid_for(ctx->g.V / 2, kDslashThreads);
    const EpiStoreFollow<P, Epi> e1{t, epi};
    eo_hop_kernel<R, DAG, 0, true, CL><<<grid, kDslashThreads, 0, st>>>(ctx->g, 1, in, in, U, A, Ai, (R)0, (R)1, e1);
    eo_hop_kernel<R, DAG, 2, false, CL><<<grid, kDslashThreads, 0, st>>>(ctx->g, 0, t, in, U, A, Ai, (R)1,
                                                                         (R)(-kappa * kappa), epi);
  }
  template <int P, int DAG, class G, class Epi>
  int launch_g(lmb_ctx *ctx, const Field<P, 12> &in, const G &U, const Epi &epi, cudaStream_t st) const {
    Field<P, 12> t;
    if (!make_field(ctx, P == PREC_DOUBLE ? "eo_t_d" : (P == PREC_SINGLE ? "eo_t_s" : "eo_t_h"), t, ctx->g.V / 2))
      return fail(ctx, LMB_ERR_CUDA, "out of device memory (even/odd workspace)");
    if (clover) launch_cl<P, true, 1 - DAG>(ctx, in, t, U, epi, st);
    else launch_cl<P, false, 1 - DAG>(ctx, in, t, U, epi, st);
    LMB_CHECK_LAUNCH(ctx);
    return LMB_OK;
  }
  template <int P, int DAG, class Epi>
  int launch(lmb_ctx *ctx, const Field<P, 12> &in, const Epi &epi, cudaStream_t st) const {
    if (ctx->links[LMB_LINKS_THIN].recon(P)) return launch_g<P, DAG>(ctx, in, eo_gauge12_view<P>(ctx), epi, st);
    return launch_g<P, DAG>(ctx, in, eo_gauge_view<P>(ctx), epi, st);
  }
  int link_reals(const lmb_ctx *ctx, int prec) const { return ctx->links[LMB_LINKS_THIN].recon(prec) ? 12 : 18; }
  bool links_finite(const lmb_ctx *ctx) const { return ctx->links[LMB_LINKS_THIN].finite(); }
};

// the CG driver's b and x of the Schur system are FP64 half fields of the
// even/odd solve (passed as Field pointers), not padded reference arrays
inline int64_t op_volume(const lmb_ctx *ctx, const SchurPolicy &) { return ctx->g.V / 2; }
template <int PS, int NC>
int op_pack_in(lmb_ctx *ctx, const SchurPolicy &, Field<PS, NC> &f, const void *src, cudaStream_t st) {
  const Field<PREC_DOUBLE, NC> &h = *(const Field<PREC_DOUBLE, NC> *)src;
  convert_kernel<PS, PREC_DOUBLE, NC><<<grid_for(ctx->g.V / 2, kBlasThreads), kBlasThreads, 0, st>>>(f, h, ctx->g.V / 2);
  LMB_CHECK_LAUNCH(ctx);
  return LMB_OK;
}
template <int PS, int NC>
int op_unpack_out(lmb_ctx *ctx, const SchurPolicy &, void *dst, const Field<PS, NC> &f, cudaStream_t st) {
  Field<PREC_DOUBLE, NC> &h = *(Field<PREC_DOUBLE, NC> *)dst;
  convert_kernel<PREC_DOUBLE, PS, NC><<<grid_for(ctx->g.V / 2, kBlasThreads), kBlasThreads, 0, st>>>(h, f, ctx->g.V / 2);
  LMB_CHECK_LAUNCH(ctx);
  return LMB_OK;
}

// FP64 views of the links and clover blocks for the even/odd setup kernels
template <bool CL, class G>
int evenodd_setup_g(lmb_ctx *ctx, const G &U, double kappa, const Field<PREC_DOUBLE, 12> &be,
                    const Field<PREC_DOUBLE, 12> &bo, Field<PREC_DOUBLE, 12> &tb, Field<PREC_DOUBLE, 12> &bh,
                    cudaStream_t st) {
  const Clover<PREC_DOUBLE> A = eo_clover_view<PREC_DOUBLE>(ctx, 0), Ai = eo_clover_view<PREC_DOUBLE>(ctx, 1);
  const int64_t Vh = ctx->g.V / 2;
  eo_local_kernel<CL><<<grid_for(Vh, 256), 256, 0, st>>>(tb, bo, ctx->g, 1, Ai);  // A_oo^-1 b_o
  EpiStore<PREC_DOUBLE, 12> e{bh, nullptr};
  eo_hop_kernel<double, 0, 1, false, CL><<<grid_for(Vh, kDslashThreads), kDslashThreads, 0, st>>>(
      ctx->g, 0, tb, be, U, A, Ai, 1.0, kappa, e);  // bh_e = b_e + k H_eo A_oo^-1 b_o
  LMB_CHECK_LAUNCH(ctx);
  return LMB_OK;
}
template <bool CL, class G>
int evenodd_odd_g(lmb_ctx *ctx, const G &U, double kappa, const Field<PREC_DOUBLE, 12> &xe,
                  const Field<PREC_DOUBLE, 12> &bo, Field<PREC_DOUBLE, 12> &xo, cudaStream_t st) {
  const Clover<PREC_DOUBLE> A = eo_clover_view<PREC_DOUBLE>(ctx, 0), Ai = eo_clover_view<PREC_DOUBLE>(ctx, 1);
  EpiStore<PREC_DOUBLE, 12> e{xo, nullptr};
  eo_hop_kernel<double, 0, 1, true, CL><<<grid_for(ctx->g.V / 2, kDslashThreads), kDslashThreads, 0, st>>>(
      ctx->g, 1, xe, bo, U, A, Ai, 1.0, kappa, e);  // x_o = A_oo^-1 (b_o + k H_oe x_e)
  LMB_CHECK_LAUNCH(ctx);
  return LMB_OK;
}


LMB_OP_INSTANCES(extern, SchurPolicy)

}  // namespace lmb
