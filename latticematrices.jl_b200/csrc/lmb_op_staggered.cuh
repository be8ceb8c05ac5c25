// lmb_op_staggered.cuh -- staggered / HISQ stencil launches and their
// operator policy.
#pragma once
#include "lmb_driver.cuh"

namespace lmb {

// epilogues the FP64 pair stencil drives: one site at a time through
// site_acc(s, active, v[3], red), then finish(red) once per block
template <class Epi> struct PairSiteAcc { static constexpr bool value = false; };
template <> struct PairSiteAcc<EpiStore<PREC_DOUBLE, 3>> { static constexpr bool value = true; };
template <> struct PairSiteAcc<EpiStoreNorm<PREC_DOUBLE, 3>> { static constexpr bool value = true; };
template <> struct PairSiteAcc<EpiCGUpdate<PREC_DOUBLE, PREC_DOUBLE, 3>> { static constexpr bool value = true; };

struct StaggeredPolicy {
  static constexpr int NC = 3;
  bool naik;  // HISQ: fat links X (LMB_LINKS_FAT) and Naik links L (LMB_LINKS_LONG)
  double mass, eps;
  int prepare(lmb_ctx *ctx, int prec, cudaStream_t st) const {
    if (!ctx->geom_set) return fail(ctx, LMB_ERR_STATE, "lmb_set_geometry has not been called");
    int rc = check_prec(ctx, prec);
    if (rc) return rc;
    if (naik) {
      if (!ctx->links[LMB_LINKS_FAT].valid || !ctx->links[LMB_LINKS_LONG].valid)
        return fail(ctx, LMB_ERR_STATE, "HISQ fat and long links have not been uploaded");
      rc = ensure_link_precision(ctx, ctx->links[LMB_LINKS_FAT], prec, st, false);
      if (rc) return rc;
      return ensure_link_precision(ctx, ctx->links[LMB_LINKS_LONG], prec, st, false);
    }
    if (!ctx->links[LMB_LINKS_THIN].valid) return fail(ctx, LMB_ERR_STATE, "gauge links have not been uploaded");
    return ensure_link_precision(ctx, ctx->links[LMB_LINKS_THIN], prec, st);
  }
  // rg: the sites to compute (the whole lattice, or the interior slab of a
  // block split along t)
  template <int P, int PHM, int DAG, class Epi>
  void launch_phm(lmb_ctx *ctx, const Field<P, 3> &in, const Epi &epi, cudaStream_t st, const SiteRange rg) const {
    typedef typename Real<P>::type R;
    const Geom &g = ctx->g;
    const unsigned grid = grid_for(rg.hi - rg.lo, kStagThreads);
    const R fc = (R)(DAG ? -0.5 : 0.5);
    const R lc = (R)(DAG ? (1.0 + eps) / 48.0 : -(1.0 + eps) / 48.0);
    if constexpr ((P == PREC_SINGLE || P == PREC_HALF) && PHM == PH_T) {
      // x-adjacent two-site kernel: even x extent, 18-real FP32 or int16 links
      const LinkSet &thin = ctx->links[LMB_LINKS_THIN];
      if (ctx->pair_sites && ctx->adj_sites && g.L[0] % 2 == 0 && (naik || !thin.recon(P))) {
        const unsigned grid2 = grid_for((rg.hi - rg.lo) / 2, kStagThreads);
        if (naik) {
          const Gauge<P> X = gauge_view<P>(ctx->links[LMB_LINKS_FAT], g.V);
          const Gauge<P> Lk = gauge_view<P>(ctx->links[LMB_LINKS_LONG], g.V);
          if constexpr (PersistentEpi<Epi>::value) {
            if (ctx->persistent) {
              auto kern = staggered_adj_persistent_kernel<true, P, Epi>;
              const unsigned g2 = std::min(grid2, resident_grid(ctx, kern));
              kern<<<g2, kStagThreads, 0, st>>>(g, in, X, Lk, mass, fc, lc, epi, (int)grid2, rg);
              return;
            }
          }
          staggered_adj_kernel<true, P><<<grid2, kStagThreads, 0, st>>>(g, in, X, Lk, mass, fc, lc, epi, rg);
        } else {
          const Gauge<P> X = gauge_view<P>(thin, g.V);
          staggered_adj_kernel<false, P><<<grid2, kStagThreads, 0, st>>>(g, in, X, X, mass, fc, lc, epi, rg);
        }
        return;
      }
    }
    if (naik) {
      const Gauge<P> X = gauge_view<P>(ctx->links[LMB_LINKS_FAT], g.V);
      const Gauge<P> Lk = gauge_view<P>(ctx->links[LMB_LINKS_LONG], g.V);
      if constexpr (PersistentEpi<Epi>::value && P == PREC_DOUBLE) {
        if (ctx->persistent) {
          auto kern = staggered_persistent_kernel<R, true, PHM, Field<P, 3>, Gauge<P>, Gauge<P>, Epi>;
          const unsigned g2 = std::min(grid, resident_grid(ctx, kern));
          kern<<<g2, kStagThreads, 0, st>>>(g, in, X, Lk, (R)mass, fc, lc, epi, (int)grid, rg);
          return;
        }
      }
      staggered_dslash_kernel<R, true, PHM><<<grid, kStagThreads, 0, st>>>(g, in, X, Lk, (R)mass, fc, lc, epi, rg);
    } else {
      const LinkSet &ls = ctx->links[LMB_LINKS_THIN];
      const NoLinks none{g.V};
      if (ls.recon(P))
        staggered_dslash_kernel<R, false, PHM><<<grid, kStagThreads, 0, st>>>(g, in, gauge12_view<P>(ls, g.V),
                                                                               none, (R)mass, fc, lc, epi, rg);
      else
        staggered_dslash_kernel<R, false, PHM><<<grid, kStagThreads, 0, st>>>(g, in, gauge_view<P>(ls, g.V),
                                                                               none, (R)mass, fc, lc, epi, rg);
    }
  }
  template <int P, int DAG, class Epi>
  int launch(lmb_ctx *ctx, const Field<P, 3> &in, const Epi &epi, cudaStream_t st) const {
    // PH_T needs at most one edge crossing per hop: every extent >= 3.  The
    // FP64 HISQ stencils measured faster on B200 with the branch form (PH_ANY).
    return launch_range<P, DAG>(ctx, in, epi, st, whole(ctx->g));
  }
  // FP64 x-adjacent pair stencil (PH_T, even x extent, 18-real links, an
  // even range of sites); false when it does not apply
  template <int DAG, class Epi>
  bool launch_pair_d(lmb_ctx *ctx, const Field<PREC_DOUBLE, 3> &in, const Epi &epi, cudaStream_t st,
                     const SiteRange rg) const {
    const Geom &g = ctx->g;
    const LinkSet &thin = ctx->links[LMB_LINKS_THIN];
    if (!ctx->pair_sites || !ctx->adj_sites || g.L[0] % 2 || ((rg.lo | rg.hi) & 1) ||
        (!naik && thin.recon(PREC_DOUBLE)))
      return false;
    const double fc = DAG ? -0.5 : 0.5;
    const double lc = DAG ? (1.0 + eps) / 48.0 : -(1.0 + eps) / 48.0;
    const unsigned ntiles = grid_for((rg.hi - rg.lo) / 2, kStagThreads);
    const Gauge<PREC_DOUBLE> X = gauge_view<PREC_DOUBLE>(naik ? ctx->links[LMB_LINKS_FAT] : thin, g.V);
    const Gauge<PREC_DOUBLE> Lk = naik ? gauge_view<PREC_DOUBLE>(ctx->links[LMB_LINKS_LONG], g.V) : X;
    auto kern = naik ? staggered_adj_d_kernel<true, Epi> : staggered_adj_d_kernel<false, Epi>;
    unsigned grid = ntiles;
    if (PersistentEpi<Epi>::value && ctx->persistent) grid = std::min(ntiles, resident_grid(ctx, kern));
    kern<<<grid, kStagThreads, 0, st>>>(g, in, X, Lk, mass, fc, lc, epi, (int)ntiles, rg);
    return true;
  }
  template <int P, int DAG, class Epi>
  int launch_range(lmb_ctx *ctx, const Field<P, 3> &in, const Epi &epi, cudaStream_t st, const SiteRange rg) const {
    const int *L = ctx->g.L;
    const bool pht = phase_mode_of(ctx->g.phase_mask) == PH_T && L[0] >= 3 && L[1] >= 3 && L[2] >= 3 && L[3] >= 3;
    if constexpr (P == PREC_DOUBLE && PairSiteAcc<Epi>::value) {
      if (pht && launch_pair_d<DAG>(ctx, in, epi, st, rg)) {
        LMB_CHECK_LAUNCH(ctx);
        return LMB_OK;
      }
    }
    if (P != PREC_DOUBLE && pht)
      launch_phm<P, PH_T, DAG>(ctx, in, epi, st, rg);
    else
      launch_phm<P, PH_ANY, DAG>(ctx, in, epi, st, rg);
    LMB_CHECK_LAUNCH(ctx);
    return LMB_OK;
  }
  int link_reals(const lmb_ctx *ctx, int prec) const {
    return (!naik && ctx->links[LMB_LINKS_THIN].recon(prec)) ? 12 : 18;
  }
  bool links_finite(const lmb_ctx *ctx) const {
    if (naik) return ctx->links[LMB_LINKS_FAT].finite() && ctx->links[LMB_LINKS_LONG].finite();
    return ctx->links[LMB_LINKS_THIN].finite();
  }
};

LMB_OP_INSTANCES(extern, StaggeredPolicy)

}  // namespace lmb
