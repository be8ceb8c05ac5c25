// lmb_op_dist.cuh -- operator policies of the sharded (process-grid) path:
// the Wilson / Wilson-clover and staggered / HISQ stencils on a block of a
// process grid, with the face exchange overlapped with the interior sites.
// The CG driver (lmb_driver.cuh) runs on them unchanged; each reduction of
// an iteration is summed over the ranks (one NCCL all-reduce of the
// interior and boundary totals) before its scalar step.
#pragma once
#include "lmb_dist_host.cuh"
#include "lmb_op_staggered.cuh"
#include "lmb_op_wilson.cuh"

namespace lmb {

// epilogues the x-adjacent pair stencils drive (pair_adj)
template <class Epi> struct HasPairAdj { static constexpr bool value = false; };
template <int PS> struct HasPairAdj<EpiStore<PS, 12>> { static constexpr bool value = true; };
template <int PS> struct HasPairAdj<EpiStoreNorm<PS, 12>> { static constexpr bool value = true; };
template <int PS, int PX> struct HasPairAdj<EpiCGUpdate<PS, PX, 12>> { static constexpr bool value = true; };

template <int P, int NC>
int dist_exchange(lmb_ctx *ctx, const Field<P, NC> &in, const DistView &dv, GhostSpinors<P, NC> &gh,
                  cudaStream_t st) {
  lmb_dist *d = ctx->dist;
  const NcclApi &nc = nccl_api();
  const char *tag = P == PREC_DOUBLE ? "d" : (P == PREC_SINGLE ? "s" : "h");
  Field<P, NC> sm[4], sp[4];
  size_t span[4] = {0, 0, 0, 0};
  FacePack<P, NC> fp{};
  int nsplit = 0;
  int64_t vmax = 0;
  const Geom &g = ctx->g;
  for (int mu = 0; mu < 4; mu++) {
    if (!((dv.split >> mu) & 1)) continue;
    const int64_t Vg = (int64_t)dv.depth * dv.face[mu];
    const std::string k = std::string(tag) + std::to_string(NC) + "_" + std::to_string(mu);
    if (!make_field(ctx, "dist_sm" + k, sm[mu], Vg) || !make_field(ctx, "dist_sp" + k, sp[mu], Vg) ||
        !make_field(ctx, "dist_gm" + k, gh.m[mu], Vg) || !make_field(ctx, "dist_gp" + k, gh.p[mu], Vg))
      return fail(ctx, LMB_ERR_CUDA, "out of device memory (ghost buffers)");
    const size_t nb = Field<P, NC>::bytes(Vg), mb = Field<P, NC>::norm_bytes(Vg);
    span[mu] = mb ? ((nb + 255) / 256) * 256 + mb : nb;
    // the rank holding global coordinate 0 sends its minus face across the
    // edge (x phase); the one holding the last coordinate its plus face (/ phase)
    const double2 one = make_double2(1.0, 0.0);
    fp.send_m[nsplit] = sm[mu];
    fp.send_p[nsplit] = sp[mu];
    fp.ph_m[nsplit] = d->coords[mu] == 0 ? make_double2(g.ph_fwd[mu][0], g.ph_fwd[mu][1]) : one;
    fp.ph_p[nsplit] = d->coords[mu] == d->dims[mu] - 1 ? make_double2(g.ph_bwd[mu][0], g.ph_bwd[mu][1]) : one;
    fp.mu[nsplit] = mu;
    nsplit++;
    if (Vg > vmax) vmax = Vg;
  }
  if (nsplit) {
    pack_faces_kernel<P, NC><<<dim3(grid_for(vmax, 256), nsplit), 256, 0, st>>>(in, fp, g, dv);
    LMB_CHECK_LAUNCH(ctx);
  }
  LMB_CUDA(ctx, cudaEventRecord(d->ev_packed, st));
  LMB_CUDA(ctx, cudaStreamWaitEvent(d->comm_stream, d->ev_packed, 0));
  ncclResult_t r = nc.GroupStart();
  for (int mu = 0; mu < 4 && r == ncclSuccess; mu++) {
    if (!((dv.split >> mu) & 1)) continue;
    // the k-th message from one rank to a peer meets the peer's k-th receive
    // from it: plus face -> plus neighbour's minus ghost, minus face -> minus
    // neighbour's plus ghost (also right for 1 or 2 ranks along mu)
    r = nc.Send(sp[mu].data, span[mu], ncclInt8, d->nb_plus[mu], d->comm, d->comm_stream);
    if (r == ncclSuccess) r = nc.Recv(gh.m[mu].data, span[mu], ncclInt8, d->nb_minus[mu], d->comm, d->comm_stream);
    if (r == ncclSuccess) r = nc.Send(sm[mu].data, span[mu], ncclInt8, d->nb_minus[mu], d->comm, d->comm_stream);
    if (r == ncclSuccess) r = nc.Recv(gh.p[mu].data, span[mu], ncclInt8, d->nb_plus[mu], d->comm, d->comm_stream);
  }
  const ncclResult_t r2 = nc.GroupEnd();
  if (r != ncclSuccess || r2 != ncclSuccess)
    return fail(ctx, LMB_ERR_CUDA, "NCCL face exchange: %s", nc.GetErrorString(r != ncclSuccess ? r : r2));
  LMB_CUDA(ctx, cudaEventRecord(d->ev_comm, d->comm_stream));
  return LMB_OK;
}

// ghost link views of link set `which` (direction mu of each dimension)
template <class G, int P>
GhostLinks<G> ghost_views(const lmb_ctx *ctx, int which, const DistView &dv, bool recon) {
  GhostLinks<G> gu{};
  for (int mu = 0; mu < 4; mu++) {
    if (!((dv.split >> mu) & 1)) continue;
    const int64_t Vg = (int64_t)dv.depth * dv.face[mu];
    if constexpr (std::is_same<G, Gauge12<P>>::value) gu.m[mu] = gauge12_view<P>(ctx->dist->ghost[which][mu], Vg);
    else gu.m[mu] = gauge_view<P>(ctx->dist->ghost[which][mu], Vg);
  }
  (void)recon;
  return gu;
}

// interior launch on `st`; the boundary launch on the boundary stream once
// the faces have arrived, beside the interior (its blocks take SMs as the
// interior's retire; separate reduction scratch); then `st` waits for it and
// the two totals are summed over the ranks
// (pairs: the interior runs on x-adjacent pairs that are wholly interior, so
// the boundary list also holds the x partners of boundary sites)
template <class Epi, class Interior, class Boundary>
int dist_stencil(lmb_ctx *ctx, int depth, const Epi &epi, cudaStream_t st, Interior interior, Boundary boundary,
                 bool pairs = false) {
  lmb_dist *d = ctx->dist;
  const int *list = nullptr;
  int n = 0;
  int rc = dist_boundary(ctx, depth, pairs, &list, &n);
  if (rc) return rc;
  Epi e0 = epi, e1 = epi;
  if constexpr (ReducingEpi<Epi>::value) {
    e0.local = d->sums;
    e1.local = d->sums + 1;
    // one slot per block of the boundary launch (at least 32 threads a block)
    e1.partials = (double *)workspace(ctx, "dist_bpartials", sizeof(double) * grid_for(ctx->g.V, 32));
    if (!e1.partials) return fail(ctx, LMB_ERR_CUDA, "out of device memory (boundary partials)");
    e1.counter = d->bcounter;
  }
  interior(e0);
  LMB_CHECK_LAUNCH(ctx);
  if (n > 0) {
    // the boundary stream's inputs were all produced on `st` before the face
    // packing, so the arrival of the faces orders it after them
    LMB_CUDA(ctx, cudaStreamWaitEvent(d->bnd_stream, d->ev_comm, 0));
    boundary(e1, list, n, d->bnd_stream);
    LMB_CHECK_LAUNCH(ctx);
    LMB_CUDA(ctx, cudaEventRecord(d->ev_bnd, d->bnd_stream));
    LMB_CUDA(ctx, cudaStreamWaitEvent(st, d->ev_bnd, 0));
  } else {
    LMB_CUDA(ctx, cudaStreamWaitEvent(st, d->ev_comm, 0));
  }
  if constexpr (ReducingEpi<Epi>::value) {
    // no split dimension: no boundary kernel, and its total is zero
    if (n == 0) LMB_CUDA(ctx, cudaMemsetAsync(d->sums + 1, 0, sizeof(double), st));
    if ((rc = dist_allreduce_sums(ctx, st))) return rc;
    dist_finalize_kernel<<<1, 32, 0, st>>>(epi, d->sums);
    LMB_CHECK_LAUNCH(ctx);
  }
  return LMB_OK;
}

struct DistWilsonPolicy {
  static constexpr int NC = 12;
  WilsonPolicy base;
  int prepare(lmb_ctx *ctx, int prec, cudaStream_t st) const {
    int rc = base.prepare(ctx, prec, st);
    if (rc) return rc;
    return dist_link_ghosts(ctx, LMB_LINKS_THIN, 1, prec, true, st);
  }
  template <int P, int DAG, bool CLOVER, class G, class CL, class Epi>
  int launch_cl(lmb_ctx *ctx, const DistView &dv, const Field<P, 12> &in, const GhostSpinors<P, 12> &gh, const G &U,
                const GhostLinks<G> &gu, const CL &A, const Epi &epi, cudaStream_t st) const {
    typedef typename Real<P>::type R;
    const Geom g = ctx->g;
    const R kappa = (R)base.kappa;
    const SiteRange slab = t_slab(g, dv);
    // any other split of an int16 block with even x: the interior on the
    // x-adjacent pair stencil, pairs with both sites interior
    bool pairs = false;
    if constexpr (P == PREC_HALF && std::is_same<G, Gauge12<PREC_HALF>>::value && HasPairAdj<Epi>::value)
      pairs = slab.hi <= slab.lo && ctx->pair_sites && ctx->adj_sites && g.L[0] % 2 == 0;
    return dist_stencil(
        ctx, 1, epi, st,
        [&](const Epi &e) {
          if (slab.hi > slab.lo) {  // split along t only: the single-lattice kernels on the slab
            if (phase_mode_of(g.phase_mask) == PH_T)
              launch_wilson_cl<P, P, CLOVER, PH_T, DAG>(ctx, in, U, A, base.kappa, e, st, slab);
            else
              launch_wilson_cl<P, P, CLOVER, PH_ANY, DAG>(ctx, in, U, A, base.kappa, e, st, slab);
            return;
          }
          if constexpr (P == PREC_HALF && std::is_same<G, Gauge12<PREC_HALF>>::value && HasPairAdj<Epi>::value) {
            if (pairs) {
              // one block at least: a reducing epilogue writes its (zero) block total
              const unsigned grid = std::max(1u, (unsigned)grid_for(dv.npairs, kDslashThreads));
              if (phase_mode_of(g.phase_mask) == PH_T)
                wilson_half_adj_interior_kernel<DAG, CLOVER, PH_T><<<grid, kDslashThreads, 0, st>>>(
                    g, dv, in, U, A, (float)base.kappa, e);
              else
                wilson_half_adj_interior_kernel<DAG, CLOVER, PH_ANY><<<grid, kDslashThreads, 0, st>>>(
                    g, dv, in, U, A, (float)base.kappa, e);
              return;
            }
          }
          wilson_interior_kernel<R, DAG, CLOVER, PH_ANY>
              <<<std::max(1u, grid_for(dv.nsites, kDslashThreads)), kDslashThreads, 0, st>>>(
              g, dv, in, U, A, kappa, e);
        },
        [&](const Epi &e, const int *list, int n, cudaStream_t bs) {
          if constexpr (P == PREC_HALF && std::is_same<G, Gauge12<PREC_HALF>>::value && HasPairAdj<Epi>::value) {
            // t-only split, x even: the two slabs on the x-adjacent pair stencil
            if (slab.hi > slab.lo && ctx->pair_sites && ctx->adj_sites && g.L[0] % 2 == 0) {
              const int F = g.stride[3];
              if (phase_mode_of(g.phase_mask) == PH_T)
                wilson_half_tslab_kernel<DAG, CLOVER, PH_T><<<grid_for(F, kDslashThreads), kDslashThreads, 0, bs>>>(
                    g, in, gh.m[3], gh.p[3], U, gu.m[3], A, (float)base.kappa, e);
              else
                wilson_half_tslab_kernel<DAG, CLOVER, PH_ANY><<<grid_for(F, kDslashThreads), kDslashThreads, 0, bs>>>(
                    g, in, gh.m[3], gh.p[3], U, gu.m[3], A, (float)base.kappa, e);
              return;
            }
            // x-only split, x extent >= 4: its boundary is the two face pairs of every row
            if (pairs && dv.split == 1u && g.L[0] >= 4) {
              const unsigned grid = grid_for(2 * (g.V / g.L[0]), kDslashThreads);
              if (phase_mode_of(g.phase_mask) == PH_T)
                wilson_half_xface_kernel<DAG, CLOVER, PH_T><<<grid, kDslashThreads, 0, bs>>>(
                    g, in, gh.m[0], gh.p[0], U, gu.m[0], A, (float)base.kappa, e);
              else
                wilson_half_xface_kernel<DAG, CLOVER, PH_ANY><<<grid, kDslashThreads, 0, bs>>>(
                    g, in, gh.m[0], gh.p[0], U, gu.m[0], A, (float)base.kappa, e);
              return;
            }
          }
          wilson_boundary_kernel<R, DAG, CLOVER><<<grid_for(n, kDslashThreads), kDslashThreads, 0, bs>>>(
              g, dv, in, gh, U, gu, A, kappa, e, list, n);
        },
        pairs);
  }
  template <int P, int DAG, class G, class Epi>
  int launch_g(lmb_ctx *ctx, const DistView &dv, const Field<P, 12> &in, const GhostSpinors<P, 12> &gh, const G &U,
               const GhostLinks<G> &gu, const Epi &epi, cudaStream_t st) const {
    if (base.op == LMB_OP_WILSON_CLOVER)
      return launch_cl<P, DAG, true>(ctx, dv, in, gh, U, gu, clover_view<P>(ctx->clover, ctx->g.V), epi, st);
    return launch_cl<P, DAG, false>(ctx, dv, in, gh, U, gu, NoClover{ctx->g.V}, epi, st);
  }
  template <int P, int DAG, class Epi>
  int launch(lmb_ctx *ctx, const Field<P, 12> &in, const Epi &epi, cudaStream_t st) const {
    const DistView dv = dist_view(ctx, 1);
    GhostSpinors<P, 12> gh{};
    int rc = dist_exchange(ctx, in, dv, gh, st);
    if (rc) return rc;
    const LinkSet &ls = ctx->links[LMB_LINKS_THIN];
    if (ls.recon(P))
      return launch_g<P, DAG>(ctx, dv, in, gh, gauge12_view<P>(ls, ctx->g.V),
                              ghost_views<Gauge12<P>, P>(ctx, LMB_LINKS_THIN, dv, true), epi, st);
    return launch_g<P, DAG>(ctx, dv, in, gh, gauge_view<P>(ls, ctx->g.V),
                            ghost_views<Gauge<P>, P>(ctx, LMB_LINKS_THIN, dv, false), epi, st);
  }
  int link_reals(const lmb_ctx *ctx, int prec) const { return base.link_reals(ctx, prec); }
  bool links_finite(const lmb_ctx *ctx) const { return base.links_finite(ctx); }
};

// the Naik links of a pair launch, or the fat (thin) ones standing in for the
// unused slot of plain staggered
template <int P, class GL> const Gauge<P> &naik_links(const Gauge<P> &X, const GL &Lk) {
  if constexpr (std::is_same<GL, Gauge<P>>::value) return Lk;
  else return X;
}

struct DistStaggeredPolicy {
  static constexpr int NC = 3;
  StaggeredPolicy base;
  int depth() const { return base.naik ? 3 : 1; }
  int prepare(lmb_ctx *ctx, int prec, cudaStream_t st) const {
    int rc = base.prepare(ctx, prec, st);
    if (rc) return rc;
    if (base.naik) {
      rc = dist_link_ghosts(ctx, LMB_LINKS_FAT, 3, prec, false, st);
      if (rc) return rc;
      return dist_link_ghosts(ctx, LMB_LINKS_LONG, 3, prec, false, st);
    }
    return dist_link_ghosts(ctx, LMB_LINKS_THIN, 1, prec, true, st);
  }
  template <int P, int DAG, bool NAIK, class GF, class GL, class Epi>
  int launch_links(lmb_ctx *ctx, const DistView &dv, const Field<P, 3> &in, const GhostSpinors<P, 3> &gh,
                   const GF &X, const GhostLinks<GF> &gx, const GL &Lk, const GhostLinks<GL> &gl, const Epi &epi,
                   cudaStream_t st) const {
    typedef typename Real<P>::type R;
    const Geom g = ctx->g;
    const R mass = (R)base.mass;
    const R fc = (R)(DAG ? -0.5 : 0.5);
    const R lc = (R)(DAG ? (1.0 + base.eps) / 48.0 : -(1.0 + base.eps) / 48.0);
    const SiteRange slab = t_slab(g, dv);
    // any other split with an even x extent, the t-phase mode and every block
    // extent >= 3, 18-real links: the interior on the x-adjacent pair stencil
    // (pairs with both sites interior)
    constexpr bool pair_ok = std::is_same<GF, Gauge<P>>::value && (!NAIK || std::is_same<GL, Gauge<P>>::value) &&
                             (P != PREC_DOUBLE || PairSiteAcc<Epi>::value);
    bool pairs = false;
    if constexpr (pair_ok)
      pairs = slab.hi <= slab.lo && ctx->pair_sites && ctx->adj_sites && g.L[0] % 2 == 0 &&
              phase_mode_of(g.phase_mask) == PH_T && g.L[0] >= 3 && g.L[1] >= 3 && g.L[2] >= 3 && g.L[3] >= 3;
    return dist_stencil(
        ctx, depth(), epi, st,
        [&](const Epi &e) {
          if (slab.hi > slab.lo) {  // split along t only: the single-lattice kernels on the slab
            base.template launch_range<P, DAG>(ctx, in, e, st, slab);
            return;
          }
          if constexpr (pair_ok) {
            if (pairs) {
              // one block at least: a reducing epilogue writes its (zero) block total
              const unsigned grid = std::max(1u, (unsigned)grid_for(dv.npairs, kStagThreads));
              const Gauge<P> &L2 = naik_links(X, Lk);  // plain staggered: X in the unused slot
              if constexpr (P == PREC_DOUBLE)
                staggered_adj_d_interior_kernel<NAIK><<<grid, kStagThreads, 0, st>>>(g, dv, in, X, L2, mass, fc, lc,
                                                                                    e);
              else
                staggered_adj_interior_kernel<NAIK, P><<<grid, kStagThreads, 0, st>>>(
                    g, dv, in, X, L2, (float)mass, (float)fc, (float)lc, e);
              return;
            }
          }
          staggered_interior_kernel<R, NAIK, PH_ANY>
              <<<std::max(1u, grid_for(dv.nsites, kStagThreads)), kStagThreads, 0, st>>>(
              g, dv, in, X, Lk, mass, fc, lc, e);
        },
        [&](const Epi &e, const int *list, int n, cudaStream_t bs) {
          staggered_boundary_kernel<R, NAIK><<<grid_for(n, kStagThreads), kStagThreads, 0, bs>>>(
              g, dv, in, gh, X, gx, Lk, gl, mass, fc, lc, e, list, n);
        },
        pairs);
  }
  template <int P, int DAG, class Epi>
  int launch(lmb_ctx *ctx, const Field<P, 3> &in, const Epi &epi, cudaStream_t st) const {
    const DistView dv = dist_view(ctx, depth());
    GhostSpinors<P, 3> gh{};
    int rc = dist_exchange(ctx, in, dv, gh, st);
    if (rc) return rc;
    if (base.naik) {
      const Gauge<P> X = gauge_view<P>(ctx->links[LMB_LINKS_FAT], ctx->g.V);
      const Gauge<P> Lk = gauge_view<P>(ctx->links[LMB_LINKS_LONG], ctx->g.V);
      return launch_links<P, DAG, true>(ctx, dv, in, gh, X, ghost_views<Gauge<P>, P>(ctx, LMB_LINKS_FAT, dv, false),
                                        Lk, ghost_views<Gauge<P>, P>(ctx, LMB_LINKS_LONG, dv, false), epi, st);
    }
    const LinkSet &ls = ctx->links[LMB_LINKS_THIN];
    const GhostLinks<NoLinks> none{};
    if (ls.recon(P))
      return launch_links<P, DAG, false>(ctx, dv, in, gh, gauge12_view<P>(ls, ctx->g.V),
                                         ghost_views<Gauge12<P>, P>(ctx, LMB_LINKS_THIN, dv, true),
                                         NoLinks{ctx->g.V}, none, epi, st);
    return launch_links<P, DAG, false>(ctx, dv, in, gh, gauge_view<P>(ls, ctx->g.V),
                                       ghost_views<Gauge<P>, P>(ctx, LMB_LINKS_THIN, dv, false), NoLinks{ctx->g.V},
                                       none, epi, st);
  }
  int link_reals(const lmb_ctx *ctx, int prec) const { return base.link_reals(ctx, prec); }
  bool links_finite(const lmb_ctx *ctx) const { return base.links_finite(ctx); }
};

inline double *op_local_sums(const lmb_ctx *ctx, const DistWilsonPolicy &) { return ctx->dist->sums; }
inline double *op_local_sums(const lmb_ctx *ctx, const DistStaggeredPolicy &) { return ctx->dist->sums; }
inline int op_allreduce_sums(lmb_ctx *ctx, const DistWilsonPolicy &, cudaStream_t st) {
  return dist_allreduce_sums(ctx, st);
}
inline int op_allreduce_sums(lmb_ctx *ctx, const DistStaggeredPolicy &, cudaStream_t st) {
  return dist_allreduce_sums(ctx, st);
}

// instantiated once per precision in lmb_dist_d.cu, lmb_dist_s.cu, lmb_dist_h.cu
LMB_OP_INSTANCES(extern, DistWilsonPolicy)
LMB_OP_INSTANCES(extern, DistStaggeredPolicy)

}  // namespace lmb
