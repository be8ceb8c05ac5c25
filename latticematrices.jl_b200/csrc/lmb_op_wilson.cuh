// lmb_op_wilson.cuh -- Wilson / Wilson-clover stencil launches and the
// operator policy the apply and CG drivers take.
#pragma once
#include "lmb_driver.cuh"

namespace lmb {

// ---------------------------------------------------------------------------
// stencil launch (DAG: 0 = D, 1 = D^+)
// ---------------------------------------------------------------------------
// rg: the sites to compute (the whole lattice, or the interior slab of a
// block split along t, whose pairs of x-adjacent sites it keeps whole)
template <int PS, int PG, bool CLOVER, int PHM, int DAG, class G, class CL, class Epi>
void launch_wilson_cl(lmb_ctx *ctx, const Field<PS, 12> &in, const G &U, const CL &A, double kappa,
                      const Epi &epi, cudaStream_t st, const SiteRange rg) {
  typedef typename Real<PS>::type R;
  const Geom &g = ctx->g;
  const bool all = rg.lo == 0 && rg.hi == (int)g.V;
  if constexpr (PS == PREC_HALF && std::is_same<G, Gauge12<PREC_HALF>>::value) {
    if (ctx->pair_sites && ctx->adj_sites && g.L[0] % 2 == 0) {
      const unsigned ntiles = grid_for((rg.hi - rg.lo) / 2, kDslashThreads);
      if constexpr (PersistentEpi<Epi>::value) {
        if (ctx->persistent) {
          auto kern = wilson_half_adj_persistent_kernel<DAG, CLOVER, PHM, CL, Epi>;
          const unsigned grid = std::min(ntiles, resident_grid(ctx, kern));
          kern<<<grid, kDslashThreads, 0, st>>>(g, in, U, A, (float)kappa, epi, (int)ntiles, rg);
          return;
        }
      }
      wilson_half_adj_kernel<DAG, CLOVER, PHM><<<ntiles, kDslashThreads, 0, st>>>(g, in, U, A, (float)kappa, epi,
                                                                                   rg);
      return;
    }
  }
  if constexpr (PS != PREC_DOUBLE) {
    if (all && ctx->pair_sites && g.L[3] % 2 == 0) {  // pairs (t, t + T/2): the whole lattice only
      wilson_dslash_pair_kernel<DAG, CLOVER, PHM><<<grid_for(g.V / 2, kDslashThreads), kDslashThreads, 0, st>>>(
          g, in, U, A, (float)kappa, epi);
      return;
    }
  }
  wilson_dslash_kernel<R, DAG, CLOVER, PHM><<<grid_for(rg.hi - rg.lo, kDslashThreads), kDslashThreads, 0, st>>>(
      g, in, U, A, (R)kappa, epi, rg);
}

template <int PS, int PG, bool CLOVER, int PHM, int DAG, class G, class Epi>
void launch_wilson_phm(lmb_ctx *ctx, const Field<PS, 12> &in, const G &U, double kappa, const Epi &epi,
                       cudaStream_t st) {
  if constexpr (CLOVER)
    launch_wilson_cl<PS, PG, true, PHM, DAG>(ctx, in, U, clover_view<PG>(ctx->clover, ctx->g.V), kappa, epi, st,
                                             whole(ctx->g));
  else
    launch_wilson_cl<PS, PG, false, PHM, DAG>(ctx, in, U, NoClover{ctx->g.V}, kappa, epi, st, whole(ctx->g));
}

template <int PS, int PG, bool CLOVER, int DAG, class G, class Epi>
int launch_wilson_g(lmb_ctx *ctx, const Field<PS, 12> &in, const G &U, double kappa, const Epi &epi,
                    cudaStream_t st) {
  if (phase_mode_of(ctx->g.phase_mask) == PH_T)
    launch_wilson_phm<PS, PG, CLOVER, PH_T, DAG>(ctx, in, U, kappa, epi, st);
  else
    launch_wilson_phm<PS, PG, CLOVER, PH_ANY, DAG>(ctx, in, U, kappa, epi, st);
  LMB_CHECK_LAUNCH(ctx);
  return LMB_OK;
}

template <int PS, int PG, bool CLOVER, int DAG, class Epi>
int launch_wilson(lmb_ctx *ctx, const Field<PS, 12> &in, double kappa, const Epi &epi, cudaStream_t st) {
  const LinkSet &ls = ctx->links[LMB_LINKS_THIN];
  if (ls.recon(PG))
    return launch_wilson_g<PS, PG, CLOVER, DAG>(ctx, in, gauge12_view<PG>(ls, ctx->g.V), kappa, epi, st);
  return launch_wilson_g<PS, PG, CLOVER, DAG>(ctx, in, gauge_view<PG>(ls, ctx->g.V), kappa, epi, st);
}

// ---------------------------------------------------------------------------
// operator policy: what to prepare and how to launch one stencil
// ---------------------------------------------------------------------------
struct WilsonPolicy {
  static constexpr int NC = 12;
  int op;
  double kappa, csw;
  int prepare(lmb_ctx *ctx, int prec, cudaStream_t st) const {
    if (!ctx->geom_set) return fail(ctx, LMB_ERR_STATE, "lmb_set_geometry has not been called");
    if (!ctx->links[LMB_LINKS_THIN].valid) return fail(ctx, LMB_ERR_STATE, "gauge links have not been uploaded");
    int rc = check_prec(ctx, prec);
    if (rc) return rc;
    rc = ensure_link_precision(ctx, ctx->links[LMB_LINKS_THIN], prec, st);
    if (rc) return rc;
    if (op == LMB_OP_WILSON_CLOVER) return ensure_clover(ctx, -kappa * csw, prec, st);
    return LMB_OK;
  }
  template <int P, int DAG, class Epi>
  int launch(lmb_ctx *ctx, const Field<P, 12> &in, const Epi &epi, cudaStream_t st) const {
    if (op == LMB_OP_WILSON_CLOVER) return launch_wilson<P, P, true, DAG>(ctx, in, kappa, epi, st);
    return launch_wilson<P, P, false, DAG>(ctx, in, kappa, epi, st);
  }
  int link_reals(const lmb_ctx *ctx, int prec) const { return ctx->links[LMB_LINKS_THIN].recon(prec) ? 12 : 18; }
  bool links_finite(const lmb_ctx *ctx) const { return ctx->links[LMB_LINKS_THIN].finite(); }
};

LMB_OP_INSTANCES(extern, WilsonPolicy)

}  // namespace lmb
