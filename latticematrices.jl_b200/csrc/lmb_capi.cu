// lmb_capi.cu -- extern "C" entry points of liblmb200.so (declared in
// include/lmb200.h) and the host drivers behind them.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <type_traits>
#include <vector>

#include "lmb_context.cuh"
#include "lmb_random.cuh"
#include "lmb_hisq_smear.cuh"
#include "lmb_batch.cuh"
#include "lmb_hisq_force.cuh"
#include "lmb_clover_force.cuh"
#include "lmb_domainwall.cuh"
#include "lmb_evenodd.cuh"
#include "lmb_halo.cuh"

using namespace lmb;

namespace {

cudaStream_t as_stream(void *s) { return (cudaStream_t)s; }

bool ctx_ok(lmb_ctx *ctx) { return ctx != nullptr; }

// ---------------------------------------------------------------------------
// link caches
// ---------------------------------------------------------------------------
int ensure_link_precision(lmb_ctx *ctx, LinkSet &ls, int prec, cudaStream_t st, bool allow_recon = true) {
  const int64_t n = 36 * ctx->g.V;
  const int64_t V = ctx->g.V;
  if (allow_recon && ls.recon(prec)) {
    double2 *d = nullptr;
    float4 *f = nullptr;
    int4 *h = nullptr;
    if (prec == PREC_DOUBLE && ls.d12_version != ls.version) {
      if (!ls.d12) LMB_CUDA(ctx, cudaMalloc(&ls.d12, sizeof(double2) * 24 * V));
      d = ls.d12;
      ls.d12_version = ls.version;
    }
    if (prec == PREC_SINGLE && ls.f12_version != ls.version) {
      if (!ls.f12) LMB_CUDA(ctx, cudaMalloc(&ls.f12, sizeof(float4) * 12 * V));
      f = ls.f12;
      ls.f12_version = ls.version;
    }
    if (prec == PREC_HALF && ls.h12_version != ls.version) {
      if (!ls.h12) LMB_CUDA(ctx, cudaMalloc(&ls.h12, sizeof(int4) * 6 * V));
      h = ls.h12;
      ls.h12_version = ls.version;
    }
    if (d || f || h) {
      links_to_recon12_kernel<<<grid_for(V, 256), 256, 0, st>>>(d, f, h, ls.d, V);
      LMB_CHECK_LAUNCH(ctx);
    }
    return LMB_OK;
  }
  if (prec == PREC_SINGLE && ls.f_version != ls.version) {
    if (!ls.f) LMB_CUDA(ctx, cudaMalloc(&ls.f, sizeof(float2) * n));
    links_to_single_kernel<<<grid_for(V, 256), 256, 0, st>>>((float4 *)ls.f, ls.d, V);
    LMB_CHECK_LAUNCH(ctx);
    ls.f_version = ls.version;
  }
  if (prec == PREC_HALF && ls.h_version != ls.version) {
    if (!ls.h) LMB_CUDA(ctx, cudaMalloc(&ls.h, sizeof(int) * n));
    links_to_half_kernel<<<grid_for(n, 256), 256, 0, st>>>(ls.h, ls.d, n, pow2_exponent(ls.scale));
    LMB_CHECK_LAUNCH(ctx);
    ls.h_version = ls.version;
  }
  return LMB_OK;
}

float device_absmax(lmb_ctx *ctx, const double2 *p, int64_t n, cudaStream_t st, int *rc) {
  unsigned *bits = (unsigned *)workspace(ctx, "absmax", sizeof(unsigned));
  if (!bits) { *rc = fail(ctx, LMB_ERR_CUDA, "out of device memory (absmax)"); return 1.f; }
  cudaMemsetAsync(bits, 0, sizeof(unsigned), st);
  absmax_kernel<<<1184, 256, 0, st>>>(p, n, bits);
  unsigned h = 0;
  cudaMemcpyAsync(&h, bits, sizeof(unsigned), cudaMemcpyDeviceToHost, st);
  if (cudaStreamSynchronize(st) != cudaSuccess) { *rc = fail(ctx, LMB_ERR_CUDA, "absmax sync"); return 1.f; }
  float f;
  std::memcpy(&f, &h, sizeof f);
  *rc = LMB_OK;
  return f;
}

template <int P> Gauge12<P> gauge12_view(const LinkSet &ls, int64_t V);
template <> Gauge12<PREC_DOUBLE> gauge12_view<PREC_DOUBLE>(const LinkSet &ls, int64_t V) { return {ls.d12, V, 1.f}; }
template <> Gauge12<PREC_SINGLE> gauge12_view<PREC_SINGLE>(const LinkSet &ls, int64_t V) { return {ls.f12, V, 1.f}; }
template <> Gauge12<PREC_HALF> gauge12_view<PREC_HALF>(const LinkSet &ls, int64_t V) { return {ls.h12, V, 1.f}; }

template <int P> Gauge<P> gauge_view(const LinkSet &ls, int64_t V);
template <> Gauge<PREC_DOUBLE> gauge_view<PREC_DOUBLE>(const LinkSet &ls, int64_t V) { return {ls.d, V, ls.scale}; }
template <> Gauge<PREC_SINGLE> gauge_view<PREC_SINGLE>(const LinkSet &ls, int64_t V) {
  return {(const float4 *)ls.f, V, ls.scale};
}
template <> Gauge<PREC_HALF> gauge_view<PREC_HALF>(const LinkSet &ls, int64_t V) {
  return {ls.h, V, base_of_exponent(pow2_exponent(ls.scale))};
}

// ---------------------------------------------------------------------------
// clover cache
// ---------------------------------------------------------------------------
int ensure_field_strength(lmb_ctx *ctx, cudaStream_t st) {
  CloverCache &cc = ctx->clover;
  const LinkSet &ls = ctx->links[LMB_LINKS_THIN];
  if (cc.F_valid && cc.F_links_version == ls.version) return LMB_OK;
  const int64_t V = ctx->g.V;
  if (!cc.F) LMB_CUDA(ctx, cudaMalloc(&cc.F, sizeof(double2) * 54 * V));
  clover_field_strength_kernel<<<grid_for(6 * V, 128), 128, 0, st>>>(cc.F, ls.d, ctx->g);
  LMB_CHECK_LAUNCH(ctx);
  cc.F_valid = true;
  cc.F_links_version = ls.version;
  return LMB_OK;
}

int clover_convert(lmb_ctx *ctx, CloverCache &cc, int prec, cudaStream_t st);

int ensure_clover(lmb_ctx *ctx, double coef, int prec, cudaStream_t st) {
  CloverCache &cc = ctx->clover;
  const LinkSet &ls = ctx->links[LMB_LINKS_THIN];
  const int64_t V = ctx->g.V;
  int rc = ensure_field_strength(ctx, st);
  if (rc) return rc;
  if (!cc.d_valid || cc.links_version != ls.version || cc.coef != coef) {
    if (!cc.d) LMB_CUDA(ctx, cudaMalloc(&cc.d, sizeof(double2) * 36 * V));
    clover_blocks_double_kernel<<<grid_for(V, 128), 128, 0, st>>>(cc.d, cc.F, ctx->g, coef);
    LMB_CHECK_LAUNCH(ctx);
    cc.d_valid = true;
    cc.links_version = ls.version;
    cc.coef = coef;
    cc.d_version++;
  }
  return clover_convert(ctx, cc, prec, st);
}

// FP32 / int16 copies of a cache's FP64 blocks, rebuilt when those change
int clover_convert(lmb_ctx *ctx, CloverCache &cc, int prec, cudaStream_t st) {
  const int64_t V = ctx->g.V;
  int rc = LMB_OK;
  if (prec == PREC_SINGLE && cc.f_version != cc.d_version) {
    if (!cc.f) LMB_CUDA(ctx, cudaMalloc(&cc.f, sizeof(float4) * 18 * V));
    clover_to_single_kernel<<<grid_for(V, 256), 256, 0, st>>>(cc.f, cc.d, V);
    LMB_CHECK_LAUNCH(ctx);
    cc.f_version = cc.d_version;
  }
  if (prec == PREC_HALF && cc.h_version != cc.d_version) {
    if (!cc.h) LMB_CUDA(ctx, cudaMalloc(&cc.h, sizeof(int4) * 8 * V));
    if (!cc.ht) LMB_CUDA(ctx, cudaMalloc(&cc.ht, sizeof(int2) * 2 * V));
    const float amax = device_absmax(ctx, cc.d, 36 * V, st, &rc);
    if (rc) return rc;
    const int kexp = pow2_exponent(amax);
    cc.scale = base_of_exponent(kexp);
    clover_to_half_kernel<<<grid_for(V, 256), 256, 0, st>>>(cc.h, cc.ht, cc.d, V, kexp);
    LMB_CHECK_LAUNCH(ctx);
    cc.h_version = cc.d_version;
  }
  return LMB_OK;
}

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

template <int P> Clover<P> clover_view(const CloverCache &cc, int64_t V);
template <> Clover<PREC_DOUBLE> clover_view<PREC_DOUBLE>(const CloverCache &cc, int64_t V) { return {cc.d, V, cc.scale}; }
template <> Clover<PREC_SINGLE> clover_view<PREC_SINGLE>(const CloverCache &cc, int64_t V) { return {cc.f, V, cc.scale}; }
template <> Clover<PREC_HALF> clover_view<PREC_HALF>(const CloverCache &cc, int64_t V) {
  Clover<PREC_HALF> c;
  c.data = cc.h;
  c.tail = cc.ht;
  c.V = V;
  c.scale = cc.scale;
  return c;
}

// ---------------------------------------------------------------------------
// stencil launch
// ---------------------------------------------------------------------------
template <int PS, int PG, bool CLOVER, int PHM, class G, class Epi>
void launch_wilson_phm(lmb_ctx *ctx, const Field<PS, 12> &in, const G &U, int dagger, double kappa,
                       const Epi &epi, cudaStream_t st) {
  typedef typename Real<PS>::type R;
  const Geom &g = ctx->g;
  if constexpr (PS == PREC_HALF && std::is_same<G, Gauge12<PREC_HALF>>::value) {
    if (ctx->pair_sites && ctx->adj_sites && g.L[0] % 2 == 0) {
      const unsigned grid2 = grid_for(g.V / 2, kDslashThreads);
      if constexpr (CLOVER) {
        const Clover<PG> A = clover_view<PG>(ctx->clover, g.V);
        if (dagger)
          wilson_half_adj_kernel<1, true, PHM><<<grid2, kDslashThreads, 0, st>>>(g, in, U, A, (float)kappa, epi);
        else
          wilson_half_adj_kernel<0, true, PHM><<<grid2, kDslashThreads, 0, st>>>(g, in, U, A, (float)kappa, epi);
      } else {
        const NoClover A{g.V};
        if (dagger)
          wilson_half_adj_kernel<1, false, PHM><<<grid2, kDslashThreads, 0, st>>>(g, in, U, A, (float)kappa, epi);
        else
          wilson_half_adj_kernel<0, false, PHM><<<grid2, kDslashThreads, 0, st>>>(g, in, U, A, (float)kappa, epi);
      }
      return;
    }
  }
  if constexpr (PS != PREC_DOUBLE) {
    if (ctx->pair_sites && g.L[3] % 2 == 0) {
      const unsigned grid2 = grid_for(g.V / 2, kDslashThreads);
      if constexpr (CLOVER) {
        const Clover<PG> A = clover_view<PG>(ctx->clover, g.V);
        if (dagger)
          wilson_dslash_pair_kernel<1, true, PHM><<<grid2, kDslashThreads, 0, st>>>(g, in, U, A, (float)kappa, epi);
        else
          wilson_dslash_pair_kernel<0, true, PHM><<<grid2, kDslashThreads, 0, st>>>(g, in, U, A, (float)kappa, epi);
      } else {
        const NoClover A{g.V};
        if (dagger)
          wilson_dslash_pair_kernel<1, false, PHM><<<grid2, kDslashThreads, 0, st>>>(g, in, U, A, (float)kappa, epi);
        else
          wilson_dslash_pair_kernel<0, false, PHM><<<grid2, kDslashThreads, 0, st>>>(g, in, U, A, (float)kappa, epi);
      }
      return;
    }
  }
  const unsigned grid = grid_for(g.V, kDslashThreads);
  if constexpr (CLOVER) {
    const Clover<PG> A = clover_view<PG>(ctx->clover, g.V);
    if (dagger)
      wilson_dslash_kernel<R, 1, true, PHM><<<grid, kDslashThreads, 0, st>>>(g, in, U, A, (R)kappa, epi);
    else
      wilson_dslash_kernel<R, 0, true, PHM><<<grid, kDslashThreads, 0, st>>>(g, in, U, A, (R)kappa, epi);
  } else {
    const NoClover A{g.V};
    if (dagger)
      wilson_dslash_kernel<R, 1, false, PHM><<<grid, kDslashThreads, 0, st>>>(g, in, U, A, (R)kappa, epi);
    else
      wilson_dslash_kernel<R, 0, false, PHM><<<grid, kDslashThreads, 0, st>>>(g, in, U, A, (R)kappa, epi);
  }
}

template <int PS, int PG, bool CLOVER, class G, class Epi>
int launch_wilson_g(lmb_ctx *ctx, const Field<PS, 12> &in, const G &U, int dagger, double kappa, const Epi &epi,
                    cudaStream_t st) {
  if (phase_mode_of(ctx->g.phase_mask) == PH_T)
    launch_wilson_phm<PS, PG, CLOVER, PH_T>(ctx, in, U, dagger, kappa, epi, st);
  else
    launch_wilson_phm<PS, PG, CLOVER, PH_ANY>(ctx, in, U, dagger, kappa, epi, st);
  LMB_CHECK_LAUNCH(ctx);
  return LMB_OK;
}

template <int PS, int PG, bool CLOVER, class Epi>
int launch_wilson(lmb_ctx *ctx, const Field<PS, 12> &in, int dagger, double kappa, const Epi &epi,
                  cudaStream_t st) {
  const LinkSet &ls = ctx->links[LMB_LINKS_THIN];
  if (ls.recon(PG))
    return launch_wilson_g<PS, PG, CLOVER>(ctx, in, gauge12_view<PG>(ls, ctx->g.V), dagger, kappa, epi, st);
  return launch_wilson_g<PS, PG, CLOVER>(ctx, in, gauge_view<PG>(ls, ctx->g.V), dagger, kappa, epi, st);
}

int check_prec(lmb_ctx *ctx, int prec) {
  if (prec < PREC_DOUBLE || prec > PREC_HALF) return fail(ctx, LMB_ERR_ARG, "unknown precision %d", prec);
  return LMB_OK;
}

// ---------------------------------------------------------------------------
// operator policies: what to prepare and how to launch one stencil
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
  template <int P, class Epi>
  int launch(lmb_ctx *ctx, const Field<P, 12> &in, int dagger, const Epi &epi, cudaStream_t st) const {
    if (op == LMB_OP_WILSON_CLOVER) return launch_wilson<P, P, true>(ctx, in, dagger, kappa, epi, st);
    return launch_wilson<P, P, false>(ctx, in, dagger, kappa, epi, st);
  }
  int link_reals(const lmb_ctx *ctx, int prec) const { return ctx->links[LMB_LINKS_THIN].recon(prec) ? 12 : 18; }
};

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
  template <int P, int PHM, class Epi>
  void launch_phm(lmb_ctx *ctx, const Field<P, 3> &in, int dagger, const Epi &epi, cudaStream_t st) const {
    typedef typename Real<P>::type R;
    const Geom &g = ctx->g;
    const unsigned grid = grid_for(g.V, kStagThreads);
    const R fc = (R)(dagger ? -0.5 : 0.5);
    const R lc = (R)(dagger ? (1.0 + eps) / 48.0 : -(1.0 + eps) / 48.0);
    if constexpr (P == PREC_SINGLE && PHM == PH_T) {
      // x-adjacent two-site kernel: even x extent, 18-real FP32 links
      const LinkSet &thin = ctx->links[LMB_LINKS_THIN];
      if (ctx->pair_sites && ctx->adj_sites && g.L[0] % 2 == 0 && (naik || !thin.recon(P))) {
        const unsigned grid2 = grid_for(g.V / 2, kStagThreads);
        if (naik) {
          const Gauge<P> X = gauge_view<P>(ctx->links[LMB_LINKS_FAT], g.V);
          const Gauge<P> Lk = gauge_view<P>(ctx->links[LMB_LINKS_LONG], g.V);
          staggered_adj_kernel<true><<<grid2, kStagThreads, 0, st>>>(g, in, X, Lk, mass, fc, lc, epi);
        } else {
          const Gauge<P> X = gauge_view<P>(thin, g.V);
          staggered_adj_kernel<false><<<grid2, kStagThreads, 0, st>>>(g, in, X, X, mass, fc, lc, epi);
        }
        return;
      }
    }
    if (naik) {
      const Gauge<P> X = gauge_view<P>(ctx->links[LMB_LINKS_FAT], g.V);
      const Gauge<P> Lk = gauge_view<P>(ctx->links[LMB_LINKS_LONG], g.V);
      staggered_dslash_kernel<R, true, PHM><<<grid, kStagThreads, 0, st>>>(g, in, X, Lk, (R)mass, fc, lc, epi);
    } else {
      const LinkSet &ls = ctx->links[LMB_LINKS_THIN];
      const NoLinks none{g.V};
      if (ls.recon(P))
        staggered_dslash_kernel<R, false, PHM><<<grid, kStagThreads, 0, st>>>(g, in, gauge12_view<P>(ls, g.V),
                                                                               none, (R)mass, fc, lc, epi);
      else
        staggered_dslash_kernel<R, false, PHM><<<grid, kStagThreads, 0, st>>>(g, in, gauge_view<P>(ls, g.V),
                                                                               none, (R)mass, fc, lc, epi);
    }
  }
  template <int P, class Epi>
  int launch(lmb_ctx *ctx, const Field<P, 3> &in, int dagger, const Epi &epi, cudaStream_t st) const {
    // PH_T needs at most one edge crossing per hop: every extent >= 3.  The
    // FP64 HISQ stencils measured faster on B200 with the branch form (PH_ANY).
    const int *L = ctx->g.L;
    if (P != PREC_DOUBLE && phase_mode_of(ctx->g.phase_mask) == PH_T && L[0] >= 3 && L[1] >= 3 && L[2] >= 3 &&
        L[3] >= 3)
      launch_phm<P, PH_T>(ctx, in, dagger, epi, st);
    else
      launch_phm<P, PH_ANY>(ctx, in, dagger, epi, st);
    LMB_CHECK_LAUNCH(ctx);
    return LMB_OK;
  }
  int link_reals(const lmb_ctx *ctx, int prec) const {
    return (!naik && ctx->links[LMB_LINKS_THIN].recon(prec)) ? 12 : 18;
  }
};

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
  template <int P, class G, class Epi>
  int launch_g(lmb_ctx *ctx, const Field<P, 12> &in, const G &U, int dagger, const Epi &epi, cudaStream_t st) const {
    typedef typename Real<P>::type R;
    const int64_t V4 = ctx->g.V, V5 = V4 * ctx->dw_L5;
    Field<P, 12> tmp;
    if (!make_field(ctx, P == PREC_DOUBLE ? "dw_tmp_d" : (P == PREC_SINGLE ? "dw_tmp_s" : "dw_tmp_h"), tmp, V5))
      return fail(ctx, LMB_ERR_CUDA, "out of device memory (domain-wall workspace)");
    const DWParams d = params(ctx);
    const unsigned grid = grid_for(V5, kDslashThreads);
    if (one_pass(ctx)) {
      if (!dagger) {
        dw_forward_kernel<R><<<grid, kDslashThreads, 0, st>>>(ctx->g, in, U, d, epi);
      } else {
        const int npts = kDslashThreads / d.L5;
        dw_adjoint_kernel<R><<<grid_for(V4, npts), kDslashThreads, 0, st>>>(ctx->g, in, U, d, npts, epi);
      }
      LMB_CHECK_LAUNCH(ctx);
      return LMB_OK;
    }
    if (!dagger) {
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
  template <int P, class Epi>
  int launch(lmb_ctx *ctx, const Field<P, 12> &in, int dagger, const Epi &epi, cudaStream_t st) const {
    const LinkSet &ls = ctx->links[LMB_LINKS_THIN];
    if (ls.recon(P)) return launch_g<P>(ctx, in, gauge12_view<P>(ls, ctx->g.V), dagger, epi, st);
    return launch_g<P>(ctx, in, gauge_view<P>(ls, ctx->g.V), dagger, epi, st);
  }
  int link_reals(const lmb_ctx *ctx, int prec) const { return ctx->links[LMB_LINKS_THIN].recon(prec) ? 12 : 18; }
};

template <int PS, int NC>
int pack_in(lmb_ctx *ctx, Field<PS, NC> &f, const void *src, cudaStream_t st) {
  const unsigned grid = grid_for(ctx->g.V, 256);
  if (ctx->dtype == LMB_DTYPE_C128)
    pack_field_kernel<double2, PS, NC><<<grid, 256, 0, st>>>(f, (const double2 *)src, ctx->g, ctx->pd);
  else
    pack_field_kernel<float2, PS, NC><<<grid, 256, 0, st>>>(f, (const float2 *)src, ctx->g, ctx->pd);
  LMB_CHECK_LAUNCH(ctx);
  return LMB_OK;
}

template <int PS, int NC>
int unpack_out(lmb_ctx *ctx, void *dst, const Field<PS, NC> &f, cudaStream_t st) {
  const unsigned grid = grid_for(ctx->g.V, 256);
  if (ctx->dtype == LMB_DTYPE_C128)
    unpack_field_kernel<double2, PS, NC><<<grid, 256, 0, st>>>((double2 *)dst, f, ctx->g, ctx->pd);
  else
    unpack_field_kernel<float2, PS, NC><<<grid, 256, 0, st>>>((float2 *)dst, f, ctx->g, ctx->pd);
  LMB_CHECK_LAUNCH(ctx);
  return LMB_OK;
}

// operator hooks with the 4D defaults: field volume, pack, unpack
template <class Op> int64_t op_volume(const lmb_ctx *ctx, const Op &) { return ctx->g.V; }
// reduction partials a CG stencil launch of the operator needs (one per block)
template <class Op> int64_t op_max_blocks(const lmb_ctx *ctx, const Op &op) {
  return grid_for(op_volume(ctx, op), kDslashThreads);
}
template <class Op, int PS, int NC>
int op_pack_in(lmb_ctx *ctx, const Op &, Field<PS, NC> &f, const void *src, cudaStream_t st) {
  return pack_in(ctx, f, src, st);
}
template <class Op, int PS, int NC>
int op_unpack_out(lmb_ctx *ctx, const Op &, void *dst, const Field<PS, NC> &f, cudaStream_t st) {
  return unpack_out(ctx, dst, f, st);
}

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

// parity-ordered copy (eo_permute_kernel) of `nplanes` planes of T at byte
// offset `off` of buffer `name`, rebuilt when the source version, the volume
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

template <int P> Gauge<P> eo_gauge_view(lmb_ctx *ctx);
template <> Gauge<PREC_DOUBLE> eo_gauge_view<PREC_DOUBLE>(lmb_ctx *ctx) {
  return {(const double2 *)eo_buffer(ctx, "eo_U_d"), ctx->g.V, ctx->links[LMB_LINKS_THIN].scale};
}
template <> Gauge<PREC_SINGLE> eo_gauge_view<PREC_SINGLE>(lmb_ctx *ctx) {
  return {(const float4 *)eo_buffer(ctx, "eo_U_s"), ctx->g.V, ctx->links[LMB_LINKS_THIN].scale};
}
template <> Gauge<PREC_HALF> eo_gauge_view<PREC_HALF>(lmb_ctx *ctx) {
  return {(const int *)eo_buffer(ctx, "eo_U_h"), ctx->g.V,
          base_of_exponent(pow2_exponent(ctx->links[LMB_LINKS_THIN].scale))};
}
template <int P> Gauge12<P> eo_gauge12_view(lmb_ctx *ctx);
template <> Gauge12<PREC_DOUBLE> eo_gauge12_view<PREC_DOUBLE>(lmb_ctx *ctx) {
  return {(const double2 *)eo_buffer(ctx, "eo_U_d"), ctx->g.V, 1.f};
}
template <> Gauge12<PREC_SINGLE> eo_gauge12_view<PREC_SINGLE>(lmb_ctx *ctx) {
  return {(const float4 *)eo_buffer(ctx, "eo_U_s"), ctx->g.V, 1.f};
}
template <> Gauge12<PREC_HALF> eo_gauge12_view<PREC_HALF>(lmb_ctx *ctx) {
  return {(const int4 *)eo_buffer(ctx, "eo_U_h"), ctx->g.V, 1.f};
}
template <int P> Clover<P> eo_clover_view(lmb_ctx *ctx, int inverse);
template <> Clover<PREC_DOUBLE> eo_clover_view<PREC_DOUBLE>(lmb_ctx *ctx, int inverse) {
  return {(const double2 *)eo_buffer(ctx, inverse ? "eo_Ai_d" : "eo_A_d"), ctx->g.V, 1.f};
}
template <> Clover<PREC_SINGLE> eo_clover_view<PREC_SINGLE>(lmb_ctx *ctx, int inverse) {
  return {(const float4 *)eo_buffer(ctx, inverse ? "eo_Ai_s" : "eo_A_s"), ctx->g.V, 1.f};
}
template <> Clover<PREC_HALF> eo_clover_view<PREC_HALF>(lmb_ctx *ctx, int inverse) {
  Clover<PREC_HALF> c;
  const char *buf = eo_buffer(ctx, inverse ? "eo_Ai_h" : "eo_A_h");
  c.data = (const int4 *)buf;
  c.tail = buf ? (const int2 *)(buf + sizeof(int4) * 8 * ctx->g.V) : nullptr;
  c.V = ctx->g.V;
  c.scale = (inverse ? ctx->clover_inv : ctx->clover).scale;
  return c;
}

// even/odd Schur operator Dh = A_ee - k^2 H_eo A_oo^-1 H_oe on the V/2 even
// sites (checkerboard order), as the CG driver sees it: launch(dagger = 0)
// applies Dh^+ and launch(dagger = 1) applies Dh, so the CG solves
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
  template <int P, class G, class Epi>
  int launch_g(lmb_ctx *ctx, const Field<P, 12> &in, const G &U, int dagger, const Epi &epi, cudaStream_t st) const {
    Field<P, 12> t;
    if (!make_field(ctx, P == PREC_DOUBLE ? "eo_t_d" : (P == PREC_SINGLE ? "eo_t_s" : "eo_t_h"), t, ctx->g.V / 2))
      return fail(ctx, LMB_ERR_CUDA, "out of device memory (even/odd workspace)");
    if (clover) {
      if (dagger) launch_cl<P, true, 0>(ctx, in, t, U, epi, st);
      else launch_cl<P, true, 1>(ctx, in, t, U, epi, st);
    } else {
      if (dagger) launch_cl<P, false, 0>(ctx, in, t, U, epi, st);
      else launch_cl<P, false, 1>(ctx, in, t, U, epi, st);
    }
    LMB_CHECK_LAUNCH(ctx);
    return LMB_OK;
  }
  template <int P, class Epi>
  int launch(lmb_ctx *ctx, const Field<P, 12> &in, int dagger, const Epi &epi, cudaStream_t st) const {
    if (ctx->links[LMB_LINKS_THIN].recon(P)) return launch_g<P>(ctx, in, eo_gauge12_view<P>(ctx), dagger, epi, st);
    return launch_g<P>(ctx, in, eo_gauge_view<P>(ctx), dagger, epi, st);
  }
  int link_reals(const lmb_ctx *ctx, int prec) const { return ctx->links[LMB_LINKS_THIN].recon(prec) ? 12 : 18; }
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

template <int PS, class Op>
int apply_generic(lmb_ctx *ctx, const Op &op, void *out, const void *in, int dagger, cudaStream_t st) {
  constexpr int NC = Op::NC;
  const int64_t V = op_volume(ctx, op);
  Field<PS, NC> fin, fout;
  if (!make_field(ctx, "apply_in", fin, V) || !make_field(ctx, "apply_out", fout, V))
    return fail(ctx, LMB_ERR_CUDA, "out of device memory (apply workspaces)");
  int rc = op_pack_in(ctx, op, fin, in, st);
  if (rc) return rc;
  EpiStore<PS, NC> epi{fout, nullptr};
  rc = op.template launch<PS>(ctx, fin, dagger, epi, st);
  if (rc) return rc;
  return op_unpack_out(ctx, op, out, fout, st);
}

template <class Op>
int apply_dispatch(lmb_ctx *ctx, const Op &op, void *out, const void *in, int dagger, int prec, void *stream) {
  if (!ctx_ok(ctx)) return LMB_ERR_ARG;
  if (!out || !in) return fail(ctx, LMB_ERR_ARG, "null field pointer");
  if (out == in) return fail(ctx, LMB_ERR_ARG, "mul! requires distinct result and input fields");
  cudaStream_t st = as_stream(stream);
  int rc = op.prepare(ctx, prec, st);
  if (rc) return rc;
  switch (prec) {
    case PREC_DOUBLE: return apply_generic<PREC_DOUBLE>(ctx, op, out, in, dagger, st);
    case PREC_SINGLE: return apply_generic<PREC_SINGLE>(ctx, op, out, in, dagger, st);
    default: return apply_generic<PREC_HALF>(ctx, op, out, in, dagger, st);
  }
}

// ---------------------------------------------------------------------------
// CG driver
// ---------------------------------------------------------------------------
struct EventPool {
  std::vector<cudaEvent_t> ev;
  void ensure(size_t n) {
    while (ev.size() < n) {
      cudaEvent_t e;
      cudaEventCreate(&e);
      ev.push_back(e);
    }
  }
  ~EventPool() {
    for (auto e : ev) cudaEventDestroy(e);
  }
};

int read_state(lmb_ctx *ctx, cudaStream_t st) {
  LMB_CUDA(ctx, cudaMemcpyAsync(ctx->st_host, ctx->st_dev, sizeof(CGState), cudaMemcpyDeviceToHost, st));
  LMB_CUDA(ctx, cudaStreamSynchronize(st));
  return LMB_OK;
}

// K3: p = r + beta p; FP32 / int16 Wilson fields of an even volume use the
// two-site kernel (256-bit accesses)
template <int PS, int NC>
void launch_p_update(lmb_ctx *ctx, Field<PS, NC> &p, const Field<PS, NC> &r, int64_t V, cudaStream_t st) {
  if constexpr (PS != PREC_DOUBLE && NC == 12) {
    if (ctx->pair_sites && ctx->adj_sites && V % 2 == 0) {
      cg_p_update_adj_kernel<PS><<<grid_for(V / 2, kBlasThreads), kBlasThreads, 0, st>>>(p, r, ctx->st_dev, V);
      return;
    }
  }
  cg_p_update_kernel<PS, NC><<<grid_for(V, kBlasThreads), kBlasThreads, 0, st>>>(p, r, ctx->st_dev, V);
}

// PS: precision of the iterated fields (DOUBLE = plain FP64 CG), PX: of x_low
template <int PS, int PX, class Op>
int cg_run(lmb_ctx *ctx, const lmb_cg_params *prm, const Op &op, void *x_pad, const void *b_pad,
           lmb_cg_result *res, cudaStream_t st) {
  constexpr bool mixed = PS != PREC_DOUBLE;
  constexpr int NC = Op::NC;
  const int64_t V = op_volume(ctx, op);
  int rc;
  long long nl = 0;  // liblmb200 kernels launched by this solve
  Field<PREC_DOUBLE, NC> b64, x64, r64, t64;
  if (!make_field(ctx, "cg_b", b64, V) || !make_field(ctx, "cg_x", x64, V) || !make_field(ctx, "cg_r", r64, V) ||
      !make_field(ctx, "cg_t", t64, V))
    return fail(ctx, LMB_ERR_CUDA, "out of device memory (CG FP64 fields)");
  Field<PS, NC> p, rl, tl;
  Field<PX, NC> xl;
  if (!make_field(ctx, "cg_p", p, V)) return fail(ctx, LMB_ERR_CUDA, "out of device memory (CG p)");
  if constexpr (mixed) {
    if (!make_field(ctx, "cg_rl", rl, V) || !make_field(ctx, "cg_tl", tl, V) || !make_field(ctx, "cg_xl", xl, V))
      return fail(ctx, LMB_ERR_CUDA, "out of device memory (CG low-precision fields)");
  } else {
    rl = *(Field<PS, NC> *)&r64;
    tl = *(Field<PS, NC> *)&t64;
    xl = *(Field<PX, NC> *)&x64;
  }
  const unsigned dgrid = grid_for(V, kDslashThreads), bgrid = grid_for(V, kBlasThreads);
  const int64_t ogrid = op_max_blocks(ctx, op);
  int64_t pgrid = dgrid > bgrid ? dgrid : bgrid;
  if (ogrid > pgrid) pgrid = ogrid;
  if (!ensure_partials(ctx, pgrid, 2))
    return fail(ctx, LMB_ERR_CUDA, "out of device memory (reduction partials)");
  rc = op.prepare(ctx, PREC_DOUBLE, st);
  if (rc) return rc;
  if (mixed) {
    rc = op.prepare(ctx, PS, st);
    if (rc) return rc;
  }

  // initial state
  CGState init{};
  init.delta2 = mixed ? prm->delta * prm->delta : 0.0;
  init.maxiter = prm->maxiter;
  init.status = ST_RUNNING;
  LMB_CUDA(ctx, cudaMemcpyAsync(ctx->st_dev, &init, sizeof init, cudaMemcpyHostToDevice, st));
  rc = op_pack_in(ctx, op, b64, b_pad, st);
  if (rc) return rc;
  rc = op_pack_in(ctx, op, x64, x_pad, st);
  if (rc) return rc;
  nl += 2;
  if constexpr (mixed) {
    LMB_CUDA(ctx, cudaMemsetAsync(xl.data, 0, Field<PX, NC>::bytes(V), st));
    if (xl.norm) LMB_CUDA(ctx, cudaMemsetAsync(xl.norm, 0, Field<PX, NC>::norm_bytes(V), st));
  }
  norm_bx_kernel<NC><<<bgrid, kBlasThreads, 0, st>>>(b64, x64, ctx->st_dev, V, prm->rtol, prm->atol,
                                                      ctx->partials, ctx->counter);
  LMB_CHECK_LAUNCH(ctx);
  nl++;
  rc = read_state(ctx, st);
  if (rc) return rc;
  const bool zero_guess = ctx->st_host->xx == 0.0;
  // r = b - D'D x (FP64)
  auto true_residual = [&](int mode) -> int {
    EpiStore<PREC_DOUBLE, NC> e1{t64, nullptr};
    int r2 = op.template launch<PREC_DOUBLE>(ctx, x64, 0, e1, st);
    if (r2) return r2;
    nl += 2;
    EpiTrueResidual<PS, NC> e2{b64, r64, rl, mixed ? 1 : 0, mode, ctx->st_dev, ctx->partials, ctx->counter};
    return op.template launch<PREC_DOUBLE>(ctx, t64, 1, e2, st);
  };
  if (zero_guess) {
    // b - D'D 0 = b exactly: one pass instead of two FP64 stencils
    residual_of_zero_kernel<PS, NC><<<dgrid, kDslashThreads, 0, st>>>(b64, r64, rl, mixed ? 1 : 0, 0, ctx->st_dev,
                                                                      V, ctx->partials, ctx->counter);
    LMB_CHECK_LAUNCH(ctx);
    nl++;
  } else {
    rc = true_residual(0);
    if (rc) return rc;
  }
  convert_kernel<PS, PS, NC><<<bgrid, kBlasThreads, 0, st>>>(p, rl, V);
  LMB_CHECK_LAUNCH(ctx);
  nl++;
  rc = read_state(ctx, st);
  if (rc) return rc;
  CGState *hs = ctx->st_host;
  if (!std::isfinite(hs->bb)) hs->status = ST_BREAKDOWN;
  if (hs->status == ST_RUNNING && prm->maxiter == 0) hs->status = ST_MAXITER;
  if (hs->status != ST_RUNNING)
    LMB_CUDA(ctx, cudaMemcpyAsync(ctx->st_dev, hs, sizeof(CGState), cudaMemcpyHostToDevice, st));

  const int k = prm->check_interval > 0 ? prm->check_interval : 8;
  EventPool pool;
  if (prm->profile) pool.ensure(4 * (size_t)k);
  double k1_ms = 0, k2_ms = 0;
  int k1_n = 0, k2_n = 0;

  EpiStoreNorm<PS, NC> epi1{tl, ctx->st_dev, ctx->partials, ctx->counter};
  EpiCGUpdate<PS, PX, NC> epi2{p, rl, xl, ctx->st_dev, ctx->partials, ctx->counter};
  while (hs->status == ST_RUNNING) {
    const int it0 = hs->iter;
    for (int i = 0; i < k; i++) {
      if (prm->profile) cudaEventRecord(pool.ev[4 * i], st);
      rc = op.template launch<PS>(ctx, p, 0, epi1, st);
      if (rc) return rc;
      nl++;
      if (prm->profile) cudaEventRecord(pool.ev[4 * i + 1], st);
      rc = op.template launch<PS>(ctx, tl, 1, epi2, st);
      if (rc) return rc;
      nl++;
      if (prm->profile) cudaEventRecord(pool.ev[4 * i + 2], st);
      launch_p_update<PS, NC>(ctx, p, rl, V, st);
      LMB_CHECK_LAUNCH(ctx);
      nl++;
      if (prm->profile) cudaEventRecord(pool.ev[4 * i + 3], st);
    }
    rc = read_state(ctx, st);
    if (rc) return rc;
    if (prm->profile) {
      const int real = hs->iter - it0 + (hs->status == ST_RELIABLE ? 1 : 0);
      for (int i = 0; i < real && i < k; i++) {
        float a = 0, b = 0;
        cudaEventElapsedTime(&a, pool.ev[4 * i], pool.ev[4 * i + 1]);
        cudaEventElapsedTime(&b, pool.ev[4 * i + 1], pool.ev[4 * i + 2]);
        k1_ms += a;
        k2_ms += b;
        k1_n++;
        k2_n++;
      }
    }
    if (hs->status == ST_RELIABLE) {
      if constexpr (mixed) {
        fold_kernel<PX, NC><<<bgrid, kBlasThreads, 0, st>>>(x64, xl, V);
        LMB_CHECK_LAUNCH(ctx);
        nl++;
        // resume: the true-residual kernel runs regardless of the pause
        rc = true_residual(1);
        if (rc) return rc;
        launch_p_update<PS, NC>(ctx, p, rl, V, st);
        LMB_CHECK_LAUNCH(ctx);
        nl++;
        rc = read_state(ctx, st);
        if (rc) return rc;
      }
    }
  }
  if constexpr (mixed) {
    fold_kernel<PX, NC><<<bgrid, kBlasThreads, 0, st>>>(x64, xl, V);
    LMB_CHECK_LAUNCH(ctx);
    nl++;
  }
  const int status = hs->status;
  CGState final_state = *hs;
  // true residual for the report (does not change the outcome)
  if (!mixed || status != ST_CONVERGED) {
    rc = true_residual(2);
    if (rc) return rc;
    rc = read_state(ctx, st);
    if (rc) return rc;
  }
  const double rr_true = ctx->st_host->rr_true;
  rc = op_unpack_out(ctx, op, x_pad, x64, st);
  if (rc) return rc;
  nl++;
  LMB_CUDA(ctx, cudaStreamSynchronize(st));

  const double bn = std::sqrt(final_state.bb);
  double rn;
  if (status == ST_BREAKDOWN) rn = NAN;
  else rn = mixed ? std::sqrt(final_state.rr_true) : std::sqrt(final_state.rr);
  if (mixed && status != ST_CONVERGED && status != ST_BREAKDOWN) rn = std::sqrt(rr_true);
  res->converged = status == ST_CONVERGED;
  res->iterations = final_state.iter;
  res->residual_norm = rn;
  res->relative_residual = bn == 0.0 ? (rn == 0.0 ? 0.0 : INFINITY) : rn / bn;
  switch (status) {
    case ST_CONVERGED: res->reason = LMB_CG_CONVERGED; break;
    case ST_MAXITER: res->reason = LMB_CG_MAXIMUM_ITERATIONS; break;
    case ST_NONPOSITIVE: res->reason = LMB_CG_NONPOSITIVE_CURVATURE; break;
    default: res->reason = LMB_CG_NUMERICAL_BREAKDOWN; break;
  }
  res->reliable_updates = final_state.reliable_updates;
  res->true_residual_norm = std::sqrt(rr_true);
  res->dslash_ms = k1_ms;
  res->update_ms = k2_ms;
  res->dslash_launches = k1_n;
  res->update_launches = k2_n;
  res->kernel_launches = nl;
  res->link_reals = op.link_reals(ctx, PS);
  return LMB_OK;
}

template <class Op>
int cg_dispatch(lmb_ctx *ctx, const lmb_cg_params *prm, const Op &op, void *x, const void *b,
                lmb_cg_result *res, cudaStream_t st) {
  switch (prm->precision) {
    case PREC_DOUBLE: return cg_run<PREC_DOUBLE, PREC_DOUBLE>(ctx, prm, op, x, b, res, st);
    case PREC_SINGLE: return cg_run<PREC_SINGLE, PREC_SINGLE>(ctx, prm, op, x, b, res, st);
    case PREC_HALF: return cg_run<PREC_HALF, PREC_SINGLE>(ctx, prm, op, x, b, res, st);
    default: return fail(ctx, LMB_ERR_ARG, "unknown precision %d", prm->precision);
  }
}

template <int NC>
__global__ void __launch_bounds__(256)
    dot_kernel(const void *a, const void *b, int c64, Geom g, Padded pd, double *partials, unsigned *counter,
               double *out) {
  const int s = blockIdx.x * 256 + threadIdx.x;
  double v[2] = {0.0, 0.0}, tot[2];
  if (s < g.V) {
    int c[4];
    site_coords(g, s, c);
    const int64_t off = padded_site(pd, c) * NC;
    for (int k = 0; k < NC; k++) {
      double ar, ai, br, bi;
      if (c64) {
        const float2 x = ((const float2 *)a)[off + k], y = ((const float2 *)b)[off + k];
        ar = x.x; ai = x.y; br = y.x; bi = y.y;
      } else {
        const double2 x = ((const double2 *)a)[off + k], y = ((const double2 *)b)[off + k];
        ar = x.x; ai = x.y; br = y.x; bi = y.y;
      }
      v[0] += ar * br + ai * bi;
      v[1] += ar * bi - ai * br;
    }
  }
  if (grid_reduce<256, 2>(v, partials, counter, tot) && threadIdx.x == 0) {
    out[0] = tot[0];
    out[1] = tot[1];
  }
}

// ---------------------------------------------------------------------------
// HISQ smearing drivers (all FP64 on 36-plane link arrays)
// ---------------------------------------------------------------------------
int pack_links_to(lmb_ctx *ctx, double2 *dst, const void *const U[4], cudaStream_t st) {
  const unsigned grid = grid_for(ctx->g.V, 256);
  if (ctx->dtype == LMB_DTYPE_C128)
    pack_links_kernel<double2><<<grid, 256, 0, st>>>(dst, (const double2 *)U[0], (const double2 *)U[1],
                                                      (const double2 *)U[2], (const double2 *)U[3], ctx->g, ctx->pd);
  else
    pack_links_kernel<float2><<<grid, 256, 0, st>>>(dst, (const float2 *)U[0], (const float2 *)U[1],
                                                     (const float2 *)U[2], (const float2 *)U[3], ctx->g, ctx->pd);
  LMB_CHECK_LAUNCH(ctx);
  return LMB_OK;
}

int unpack_links_from(lmb_ctx *ctx, void *const U[4], const double2 *src, cudaStream_t st) {
  const unsigned grid = grid_for(ctx->g.V, 256);
  if (ctx->dtype == LMB_DTYPE_C128)
    unpack_links_kernel<double2><<<grid, 256, 0, st>>>((double2 *)U[0], (double2 *)U[1], (double2 *)U[2],
                                                        (double2 *)U[3], src, ctx->g, ctx->pd);
  else
    unpack_links_kernel<float2><<<grid, 256, 0, st>>>((float2 *)U[0], (float2 *)U[1], (float2 *)U[2],
                                                       (float2 *)U[3], src, ctx->g, ctx->pd);
  LMB_CHECK_LAUNCH(ctx);
  return LMB_OK;
}

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

int check_links_arg(lmb_ctx *ctx, const void *const U[4], const char *what) {
  if (!U) return fail(ctx, LMB_ERR_ARG, "null %s array", what);
  for (int mu = 0; mu < 4; mu++)
    if (!U[mu]) return fail(ctx, LMB_ERR_ARG, "%s[%d] is null", what, mu + 1);
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
// batched CG driver
// ---------------------------------------------------------------------------
struct BatchRun {
  std::vector<BatchGroup> groups;
  BatchGroup *d_groups = nullptr;
  int ntasks = 0;
  int nb = 1, nt = 128;
};

template <int NT, int NB, int ROLE>
void launch_batch_k(const BatchRun &br, CGState *states, cudaStream_t st, int grid) {
  batch_wilson_kernel<NT, NB, ROLE><<<grid, NT, 0, st>>>(br.d_groups, (int)br.groups.size(), br.ntasks, states);
}
template <int NT, int NB, int ROLE>
void launch_batch_64(const BatchRun &br, CGState *states, cudaStream_t st, int grid) {
  batch_wilson64_kernel<NT, NB, ROLE><<<grid, NT, 0, st>>>(br.d_groups, (int)br.groups.size(), br.ntasks, states);
}
template <int NT, int NB>
void launch_batch_p(const BatchRun &br, CGState *states, cudaStream_t st, int grid) {
  batch_p_update_kernel<NT, NB><<<grid, NT, 0, st>>>(br.d_groups, (int)br.groups.size(), br.ntasks, states);
}

// resident blocks of the persistent launch: SMs x blocks per SM (per device)
template <int NT, int NB>
int batch_grid() {
  static int cached[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev >= 0 && dev < 64 && cached[dev]) return cached[dev];
  int per_sm = 0, sms = 148;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batch_wilson_kernel<NT, NB, ROLE_K2>, NT, 0);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int g = (per_sm > 0 ? per_sm : 1) * sms;
  if (dev >= 0 && dev < 64) cached[dev] = g;
  return g;
}

// dispatch one stage for the run's (NT, NB)
int batch_stage(lmb_ctx *ctx, const BatchRun &br, CGState *states, int stage, cudaStream_t st) {
#define LMB_BATCH_CASE(NT_, NB_)                                                          \
  if (br.nt == NT_ && br.nb == NB_) {                                                     \
    const int grid = std::min(br.ntasks, batch_grid<NT_, NB_>());                        \
    switch (stage) {                                                                      \
      case 0: launch_batch_k<NT_, NB_, ROLE_K1>(br, states, st, grid); break;             \
      case 1: launch_batch_k<NT_, NB_, ROLE_K2>(br, states, st, grid); break;             \
      case 2: launch_batch_p<NT_, NB_>(br, states, st, grid); break;                      \
      case 3: launch_batch_64<NT_, NB_, ROLE_D64>(br, states, st, grid); break;           \
      default: launch_batch_64<NT_, NB_, ROLE_TRUE>(br, states, st, grid); break;         \
    }                                                                                     \
    LMB_CHECK_LAUNCH(ctx);                                                                \
    return LMB_OK;                                                                        \
  }
  LMB_BATCH_CASE(64, 1) LMB_BATCH_CASE(64, 2) LMB_BATCH_CASE(64, 4)
  LMB_BATCH_CASE(128, 1) LMB_BATCH_CASE(128, 2) LMB_BATCH_CASE(128, 4)
  LMB_BATCH_CASE(256, 1) LMB_BATCH_CASE(256, 2) LMB_BATCH_CASE(256, 4)
#undef LMB_BATCH_CASE
  return fail(ctx, LMB_ERR_UNSUPPORTED, "batched tile %d x rhs block %d not built", br.nt, br.nb);
}

struct BatchMember {
  int lattice, rhs;
  Geom g;
  Padded pd;
  Field<PREC_DOUBLE, 12> b64, x64, r64, t64;
  Field<PREC_SINGLE, 12> p, t, r, xl;
};

int build_run(lmb_ctx *ctx, BatchRun &br, int nb, int nt, const std::vector<BatchMember> &m,
              const std::vector<int> &member_lattice_start, const std::vector<int> &nrhs,
              const std::vector<lmb_batch_links *> &links, const std::vector<double> &kappa,
              const std::string &tag) {
  br.nb = nb;
  br.nt = nt;
  br.groups.clear();
  int task = 0;
  size_t partial_words = 0;
  for (size_t l = 0; l < nrhs.size(); l++) {
    for (int r0 = 0; r0 < nrhs[l]; r0 += nb) {
      BatchGroup G{};
      const BatchMember &m0 = m[member_lattice_start[l] + r0];
      G.g = m0.g;
      G.U = links[l]->f12;
      G.U64 = links[l]->d12;
      G.nact = std::min(nb, nrhs[l] - r0);
      G.first_task = task;
      G.ntasks = (int)((G.g.V + nt - 1) / nt);
      G.state0 = member_lattice_start[l] + r0;
      G.kappa = kappa[l];
      for (int r = 0; r < G.nact; r++) {
        const BatchMember &mm = m[G.state0 + r];
        G.p[r] = mm.p.data;
        G.t[r] = mm.t.data;
        G.r[r] = mm.r.data;
        G.xl[r] = mm.xl.data;
        G.b64[r] = mm.b64.data;
        G.x64[r] = mm.x64.data;
        G.r64[r] = mm.r64.data;
        G.t64[r] = mm.t64.data;
      }
      task += G.ntasks;
      partial_words += (size_t)G.ntasks * nb;
      br.groups.push_back(G);
    }
  }
  br.ntasks = task;
  double *partials = (double *)workspace(ctx, "batch_partials_" + tag, sizeof(double) * partial_words);
  unsigned *counters = (unsigned *)workspace(ctx, "batch_counters_" + tag, sizeof(unsigned) * br.groups.size());
  br.d_groups = (BatchGroup *)workspace(ctx, "batch_groups_" + tag, sizeof(BatchGroup) * br.groups.size());
  if (!partials || !counters || !br.d_groups) return fail(ctx, LMB_ERR_CUDA, "out of device memory (batch tables)");
  LMB_CUDA(ctx, cudaMemset(counters, 0, sizeof(unsigned) * br.groups.size()));
  size_t off = 0;
  for (size_t i = 0; i < br.groups.size(); i++) {
    br.groups[i].partials = partials + off;
    br.groups[i].counter = counters + i;
    off += (size_t)br.groups[i].ntasks * nb;
  }
  return LMB_OK;
}

int upload_groups(lmb_ctx *ctx, BatchRun &br, cudaStream_t st) {
  LMB_CUDA(ctx, cudaMemcpyAsync(br.d_groups, br.groups.data(), sizeof(BatchGroup) * br.groups.size(),
                                cudaMemcpyHostToDevice, st));
  return LMB_OK;
}

int batch_links_for(lmb_ctx *ctx, const lmb_batch_lattice &lat, const Geom &g, const Padded &pd,
                    lmb_batch_links **out, cudaStream_t st) {
  for (auto &bl : ctx->batch_links) {
    bool same = bl.V == g.V;
    for (int mu = 0; mu < 4 && same; mu++) same = bl.ptr[mu] == lat.U[mu] && bl.epoch[mu] == lat.epoch[mu];
    if (same) {
      *out = &bl;
      return LMB_OK;
    }
  }
  ctx->batch_links.emplace_back();
  lmb_batch_links &bl = ctx->batch_links.back();
  const int64_t V = g.V;
  double2 *d = (double2 *)workspace(ctx, "batch_pack", sizeof(double2) * 36 * V);
  if (!d) return fail(ctx, LMB_ERR_CUDA, "out of device memory (batched links)");
  pack_links_kernel<double2><<<grid_for(V, 256), 256, 0, st>>>(
      d, (const double2 *)lat.U[0], (const double2 *)lat.U[1], (const double2 *)lat.U[2],
      (const double2 *)lat.U[3], g, pd);
  LMB_CHECK_LAUNCH(ctx);
  unsigned *bits = (unsigned *)workspace(ctx, "su3dev", sizeof(unsigned));
  if (!bits) return fail(ctx, LMB_ERR_CUDA, "out of device memory (su3 check)");
  LMB_CUDA(ctx, cudaMemsetAsync(bits, 0, sizeof(unsigned), st));
  su3_deviation_kernel<<<1184, 256, 0, st>>>(d, V, bits);
  unsigned hb = 0;
  LMB_CUDA(ctx, cudaMemcpyAsync(&hb, bits, sizeof hb, cudaMemcpyDeviceToHost, st));
  LMB_CUDA(ctx, cudaStreamSynchronize(st));
  float dev;
  std::memcpy(&dev, &hb, sizeof dev);
  if (!(dev <= 1e-12f)) {
    ctx->batch_links.pop_back();
    return fail(ctx, LMB_ERR_UNSUPPORTED, "batched CG needs SU(3) links (deviation %.3g)", (double)dev);
  }
  LMB_CUDA(ctx, cudaMalloc(&bl.d12, sizeof(double2) * 24 * V));
  LMB_CUDA(ctx, cudaMalloc(&bl.f12, sizeof(float4) * 12 * V));
  links_to_recon12_kernel<<<grid_for(V, 256), 256, 0, st>>>(bl.d12, bl.f12, nullptr, d, V);
  LMB_CHECK_LAUNCH(ctx);
  for (int mu = 0; mu < 4; mu++) {
    bl.ptr[mu] = lat.U[mu];
    bl.epoch[mu] = lat.epoch[mu];
  }
  bl.V = V;
  *out = &bl;
  return LMB_OK;
}

int cg_batched(lmb_ctx *ctx, const lmb_cg_params *prm, int nlat, const lmb_batch_lattice *lats,
               lmb_cg_result *res, lmb_batch_tuning *tuning, cudaStream_t st) {
  // geometry and links per lattice
  std::vector<Geom> geoms(nlat);
  std::vector<Padded> pads(nlat);
  std::vector<lmb_batch_links *> links(nlat);
  std::vector<int> nrhs(nlat), start(nlat);
  std::vector<double> kappa(nlat);
  std::string sig;
  int total = 0;
  for (int l = 0; l < nlat; l++) {
    const lmb_batch_lattice &lat = lats[l];
    if (lat.nrhs <= 0 || !lat.x || !lat.b) return fail(ctx, LMB_ERR_ARG, "lattice %d has no right-hand sides", l);
    Geom g{};
    int64_t V = 1;
    int stride = 1;
    for (int mu = 0; mu < 4; mu++) {
      if (lat.L[mu] <= 0 || lat.nw < 0 || lat.nw > lat.L[mu]) return fail(ctx, LMB_ERR_ARG, "bad geometry of lattice %d", l);
      const double re = lat.phase_re[mu], im = lat.phase_im[mu], n = re * re + im * im;
      if (n == 0.0) return fail(ctx, LMB_ERR_ARG, "boundary phases must be nonzero because negative wraps use inv(phase)");
      g.L[mu] = lat.L[mu];
      g.stride[mu] = stride;
      stride *= lat.L[mu];
      V *= lat.L[mu];
      g.ph_fwd[mu][0] = re;
      g.ph_fwd[mu][1] = im;
      g.ph_bwd[mu][0] = re / n;
      g.ph_bwd[mu][1] = -im / n;
      if (!(re == 1.0 && im == 0.0)) g.phase_mask |= 1 << mu;
      pads[l].P[mu] = lat.L[mu] + 2 * lat.nw;
    }
    g.V = V;
    pads[l].nw = lat.nw;
    geoms[l] = g;
    for (int mu = 0; mu < 4; mu++)
      if (!lat.U[mu]) return fail(ctx, LMB_ERR_ARG, "gauge link U[%d] of lattice %d is null", mu + 1, l);
    int rc = batch_links_for(ctx, lat, g, pads[l], &links[l], st);
    if (rc) return rc;
    nrhs[l] = lat.nrhs;
    start[l] = total;
    total += lat.nrhs;
    kappa[l] = lat.kappa;
    char buf[96];
    snprintf(buf, sizeof buf, "%dx%dx%dx%d:%d;", lat.L[0], lat.L[1], lat.L[2], lat.L[3], lat.nrhs);
    sig += buf;
  }
  // fields of every member
  std::vector<BatchMember> m(total);
  for (int l = 0; l < nlat; l++)
    for (int r = 0; r < nrhs[l]; r++) {
      BatchMember &mm = m[start[l] + r];
      mm.lattice = l;
      mm.rhs = r;
      mm.g = geoms[l];
      mm.pd = pads[l];
      const std::string k = std::to_string(start[l] + r);
      // member fields sized by its own lattice (workspace grows on demand)
      const int64_t V = geoms[l].V;
      auto mk64 = [&](const std::string &n, Field<PREC_DOUBLE, 12> &f) {
        f.V = V;
        f.norm = nullptr;
        f.data = (double2 *)workspace(ctx, n, Field<PREC_DOUBLE, 12>::bytes(V));
        return f.data != nullptr;
      };
      auto mk32 = [&](const std::string &n, Field<PREC_SINGLE, 12> &f) {
        f.V = V;
        f.norm = nullptr;
        f.data = (float4 *)workspace(ctx, n, Field<PREC_SINGLE, 12>::bytes(V));
        return f.data != nullptr;
      };
      if (!mk64("bt_b" + k, mm.b64) || !mk64("bt_x" + k, mm.x64) || !mk64("bt_r" + k, mm.r64) ||
          !mk64("bt_t" + k, mm.t64) || !mk32("bt_p" + k, mm.p) || !mk32("bt_tl" + k, mm.t) ||
          !mk32("bt_rl" + k, mm.r) || !mk32("bt_xl" + k, mm.xl))
        return fail(ctx, LMB_ERR_CUDA, "out of device memory (batched fields)");
    }
  CGState *states = (CGState *)workspace(ctx, "bt_states", sizeof(CGState) * total);
  if (!states) return fail(ctx, LMB_ERR_CUDA, "out of device memory (batched states)");
  std::vector<CGState> init(total);
  for (auto &s0 : init) {
    s0 = CGState{};
    s0.delta2 = prm->delta * prm->delta;
    s0.maxiter = prm->maxiter;
    s0.status = ST_RUNNING;
  }
  int rc;
  // ---- pack b and x of every member; p = b gives the tuning passes real data
  for (int i = 0; i < total; i++) {
    BatchMember &mm = m[i];
    const lmb_batch_lattice &lat = lats[mm.lattice];
    const unsigned grid = grid_for(mm.g.V, 256);
    pack_field_kernel<double2, PREC_DOUBLE, 12><<<grid, 256, 0, st>>>(mm.b64, (const double2 *)lat.b[mm.rhs], mm.g, mm.pd);
    pack_field_kernel<double2, PREC_DOUBLE, 12><<<grid, 256, 0, st>>>(mm.x64, (const double2 *)lat.x[mm.rhs], mm.g, mm.pd);
    convert_kernel<PREC_SINGLE, PREC_DOUBLE, 12><<<grid_for(mm.g.V, kBlasThreads), kBlasThreads, 0, st>>>(
        mm.p, mm.b64, mm.g.V);
    LMB_CHECK_LAUNCH(ctx);
  }
  // ---- autotune (RHS block, threads) on the stencil stages, once per shape set
  lmb_batch_tune tune;
  auto it = ctx->batch_tune.find(sig);
  if (it != ctx->batch_tune.end()) {
    tune = it->second;
  } else {
    double best = 1e30;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    std::vector<CGState> dummy(total);
    for (auto &d : dummy) {
      d = CGState{};
      d.status = ST_RUNNING;
      d.alpha = 0.0;
      d.rr = 1.0;
      d.maxrr = 1e300;
      d.delta2 = 0.0;
      d.maxiter = 1 << 30;
      d.tol2 = -1.0;
    }
    const int nbs[3] = {1, 2, 4}, nts[3] = {64, 128, 256};
    for (int a = 0; a < 3; a++)
      for (int b = 0; b < 3; b++) {
        BatchRun br;
        if ((rc = build_run(ctx, br, nbs[a], nts[b], m, start, nrhs, links, kappa, "tune"))) return rc;
        if ((rc = upload_groups(ctx, br, st))) return rc;
        LMB_CUDA(ctx, cudaMemcpyAsync(states, dummy.data(), sizeof(CGState) * total, cudaMemcpyHostToDevice, st));
        for (int w = 0; w < 2; w++) {
          if ((rc = batch_stage(ctx, br, states, 0, st))) return rc;
          if ((rc = batch_stage(ctx, br, states, 1, st))) return rc;
        }
        cudaEventRecord(e0, st);
        for (int w = 0; w < 3; w++) {
          if ((rc = batch_stage(ctx, br, states, 0, st))) return rc;
          if ((rc = batch_stage(ctx, br, states, 1, st))) return rc;
        }
        cudaEventRecord(e1, st);
        LMB_CUDA(ctx, cudaEventSynchronize(e1));
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best) {
          best = ms;
          tune.nb = nbs[a];
          tune.nt = nts[b];
          tune.ms = ms / 3.0;
        }
      }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    ctx->batch_tune[sig] = tune;
  }
  BatchRun br;
  if ((rc = build_run(ctx, br, tune.nb, tune.nt, m, start, nrhs, links, kappa, "run"))) return rc;
  if ((rc = upload_groups(ctx, br, st))) return rc;
  LMB_CUDA(ctx, cudaMemcpyAsync(states, init.data(), sizeof(CGState) * total, cudaMemcpyHostToDevice, st));
  // ---- per-member setup: pack b and x, x_low = 0, |b|
  if (!ensure_partials(ctx, grid_for(1 << 24, kBlasThreads), 1))
    return fail(ctx, LMB_ERR_CUDA, "out of device memory (reduction partials)");
  for (int i = 0; i < total; i++) {
    BatchMember &mm = m[i];
    LMB_CUDA(ctx, cudaMemsetAsync(mm.xl.data, 0, Field<PREC_SINGLE, 12>::bytes(mm.g.V), st));
    norm_b_kernel<12><<<grid_for(mm.g.V, kBlasThreads), kBlasThreads, 0, st>>>(
        mm.b64, states + i, mm.g.V, prm->rtol, prm->atol, ctx->partials, ctx->counter);
    LMB_CHECK_LAUNCH(ctx);
  }
  // ---- r = b - D'D x for all members, p = r
  auto true_pass = [&](const std::vector<unsigned> &masks, int mode) -> int {
    for (size_t gi = 0; gi < br.groups.size(); gi++) {
      br.groups[gi].mask = masks[gi];
      br.groups[gi].mode = mode;
    }
    int r2 = upload_groups(ctx, br, st);
    if (r2) return r2;
    if ((r2 = batch_stage(ctx, br, states, 3, st))) return r2;
    return batch_stage(ctx, br, states, 4, st);
  };
  std::vector<unsigned> all_mask(br.groups.size()), none_mask(br.groups.size(), 0u);
  for (size_t gi = 0; gi < br.groups.size(); gi++) all_mask[gi] = (1u << br.groups[gi].nact) - 1u;
  if ((rc = true_pass(all_mask, 0))) return rc;
  for (int i = 0; i < total; i++) {
    convert_kernel<PREC_SINGLE, PREC_SINGLE, 12><<<grid_for(m[i].g.V, kBlasThreads), kBlasThreads, 0, st>>>(
        m[i].p, m[i].r, m[i].g.V);
  }
  LMB_CHECK_LAUNCH(ctx);
  std::vector<CGState> hs(total);
  auto read_all = [&]() -> int {
    LMB_CUDA(ctx, cudaMemcpyAsync(hs.data(), states, sizeof(CGState) * total, cudaMemcpyDeviceToHost, st));
    LMB_CUDA(ctx, cudaStreamSynchronize(st));
    return LMB_OK;
  };
  if ((rc = read_all())) return rc;
  bool fix = false;
  for (auto &x : hs) {
    if (!std::isfinite(x.bb)) { x.status = ST_BREAKDOWN; fix = true; }
    if (x.status == ST_RUNNING && prm->maxiter == 0) { x.status = ST_MAXITER; fix = true; }
  }
  if (fix) LMB_CUDA(ctx, cudaMemcpyAsync(states, hs.data(), sizeof(CGState) * total, cudaMemcpyHostToDevice, st));
  // ---- one iteration as a CUDA graph
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaStream_t cs;
  LMB_CUDA(ctx, cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
  LMB_CUDA(ctx, cudaStreamSynchronize(st));
  LMB_CUDA(ctx, cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
  int crc = batch_stage(ctx, br, states, 0, cs);
  if (!crc) crc = batch_stage(ctx, br, states, 1, cs);
  if (!crc) crc = batch_stage(ctx, br, states, 2, cs);
  cudaError_t ge = cudaStreamEndCapture(cs, &graph);
  if (crc || ge != cudaSuccess) {
    cudaStreamDestroy(cs);
    return crc ? crc : fail(ctx, LMB_ERR_CUDA, "graph capture: %s", cudaGetErrorString(ge));
  }
  ge = cudaGraphInstantiate(&exec, graph, 0);
  if (ge != cudaSuccess) {
    cudaGraphDestroy(graph);
    cudaStreamDestroy(cs);
    return fail(ctx, LMB_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(ge));
  }
  const int k = prm->check_interval > 0 ? prm->check_interval : 8;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  double graph_ms = 0;
  long long graph_iters = 0;
  auto cleanup = [&]() {
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaGraphExecDestroy(exec);
    cudaGraphDestroy(graph);
    cudaStreamDestroy(cs);
  };
  auto any_running = [&]() {
    for (auto &x : hs)
      if (x.status == ST_RUNNING || x.status == ST_RELIABLE) return true;
    return false;
  };
  while (any_running()) {
    cudaEventRecord(e0, st);
    for (int i = 0; i < k; i++) {
      cudaError_t le = cudaGraphLaunch(exec, st);
      if (le != cudaSuccess) {
        cleanup();
        return fail(ctx, LMB_ERR_CUDA, "graph launch: %s", cudaGetErrorString(le));
      }
    }
    cudaEventRecord(e1, st);
    if ((rc = read_all())) { cleanup(); return rc; }
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    graph_ms += ms;
    graph_iters += k;
    // reliable updates for the paused members
    std::vector<unsigned> masks(br.groups.size(), 0u);
    bool anyrel = false;
    for (size_t gi = 0; gi < br.groups.size(); gi++)
      for (int r = 0; r < br.groups[gi].nact; r++)
        if (hs[br.groups[gi].state0 + r].status == ST_RELIABLE) {
          masks[gi] |= 1u << r;
          anyrel = true;
          BatchMember &mm = m[br.groups[gi].state0 + r];
          fold_kernel<PREC_SINGLE, 12><<<grid_for(mm.g.V, kBlasThreads), kBlasThreads, 0, st>>>(mm.x64, mm.xl, mm.g.V);
        }
    if (anyrel) {
      if ((rc = true_pass(masks, 1))) { cleanup(); return rc; }
      for (size_t gi = 0; gi < br.groups.size(); gi++)
        for (int r = 0; r < br.groups[gi].nact; r++)
          if ((masks[gi] >> r) & 1) {
            BatchMember &mm = m[br.groups[gi].state0 + r];
            cg_p_update_kernel<PREC_SINGLE, 12><<<grid_for(mm.g.V, kBlasThreads), kBlasThreads, 0, st>>>(
                mm.p, mm.r, states + br.groups[gi].state0 + r, mm.g.V);
          }
      LMB_CHECK_LAUNCH(ctx);
      if ((rc = read_all())) { cleanup(); return rc; }
    }
  }
  // ---- finish: fold, report true residuals, unpack
  for (int i = 0; i < total; i++)
    fold_kernel<PREC_SINGLE, 12><<<grid_for(m[i].g.V, kBlasThreads), kBlasThreads, 0, st>>>(m[i].x64, m[i].xl, m[i].g.V);
  std::vector<CGState> fin = hs;
  if ((rc = true_pass(all_mask, 2))) { cleanup(); return rc; }
  if ((rc = read_all())) { cleanup(); return rc; }
  for (int i = 0; i < total; i++) {
    const BatchMember &mm = m[i];
    const lmb_batch_lattice &lat = lats[mm.lattice];
    unpack_field_kernel<double2, PREC_DOUBLE, 12><<<grid_for(mm.g.V, 256), 256, 0, st>>>(
        (double2 *)lat.x[mm.rhs], mm.x64, mm.g, mm.pd);
  }
  LMB_CHECK_LAUNCH(ctx);
  LMB_CUDA(ctx, cudaStreamSynchronize(st));
  for (int i = 0; i < total; i++) {
    const CGState &f = fin[i];
    const double bn = std::sqrt(f.bb);
    const double rt = std::sqrt(hs[i].rr_true);
    const double rn = f.status == ST_BREAKDOWN ? NAN : (f.status == ST_CONVERGED ? std::sqrt(f.rr_true) : rt);
    lmb_cg_result &o = res[i];
    std::memset(&o, 0, sizeof o);
    o.converged = f.status == ST_CONVERGED;
    o.iterations = f.iter;
    o.residual_norm = rn;
    o.relative_residual = bn == 0.0 ? (rn == 0.0 ? 0.0 : INFINITY) : rn / bn;
    o.reason = f.status == ST_CONVERGED ? LMB_CG_CONVERGED
               : f.status == ST_MAXITER ? LMB_CG_MAXIMUM_ITERATIONS
               : f.status == ST_NONPOSITIVE ? LMB_CG_NONPOSITIVE_CURVATURE
                                             : LMB_CG_NUMERICAL_BREAKDOWN;
    o.reliable_updates = f.reliable_updates;
    o.true_residual_norm = rt;
    o.link_reals = 12;
  }
  if (tuning) {
    tuning->rhs_block = tune.nb;
    tuning->threads = tune.nt;
    tuning->ms_per_iteration = graph_iters ? graph_ms / graph_iters : 0.0;
    tuning->graph_iterations = (int)graph_iters;
  }
  cleanup();
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

}  // namespace

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

int lmb_version(void) { return 100; }

lmb_ctx *lmb_create(int device) {
  if (cudaSetDevice(device) != cudaSuccess) return nullptr;
  lmb_ctx *ctx = new lmb_ctx();
  ctx->device = device;
  if (const char *ps = getenv("LMB_PAIR_SITES")) ctx->pair_sites = atoi(ps) != 0;
  if (const char *as = getenv("LMB_ADJ_SITES")) ctx->adj_sites = atoi(as) != 0;
  if (const char *dw = getenv("LMB_DW_TWO_PASS")) ctx->dw_two_pass = atoi(dw) != 0;
  if (cudaMalloc(&ctx->counter, sizeof(unsigned)) != cudaSuccess ||
      cudaMemset(ctx->counter, 0, sizeof(unsigned)) != cudaSuccess ||
      cudaMalloc(&ctx->st_dev, sizeof(CGState)) != cudaSuccess ||
      cudaMallocHost(&ctx->st_host, sizeof(CGState)) != cudaSuccess ||
      cudaMallocHost(&ctx->dot_host, 2 * sizeof(double)) != cudaSuccess) {
    lmb_destroy(ctx);
    return nullptr;
  }
  return ctx;
}

void lmb_destroy(lmb_ctx *ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  for (auto &kv : ctx->buffers) cudaFree(kv.second.first);
  for (auto &bl : ctx->batch_links) {
    cudaFree(bl.d12);
    cudaFree(bl.f12);
  }
  for (auto &ls : ctx->links) {
    cudaFree(ls.d);
    cudaFree(ls.f);
    cudaFree(ls.h);
    cudaFree(ls.d12);
    cudaFree(ls.f12);
    cudaFree(ls.h12);
  }
  cudaFree(ctx->clover.F);
  cudaFree(ctx->clover.d);
  cudaFree(ctx->dw_coef);
  cudaFree(ctx->clover.f);
  cudaFree(ctx->clover.h);
  cudaFree(ctx->clover.ht);
  cudaFree(ctx->clover_inv.d);
  cudaFree(ctx->clover_inv.f);
  cudaFree(ctx->clover_inv.h);
  cudaFree(ctx->clover_inv.ht);
  cudaFree(ctx->partials);
  cudaFree(ctx->counter);
  cudaFree(ctx->st_dev);
  if (ctx->st_host) cudaFreeHost(ctx->st_host);
  if (ctx->dot_host) cudaFreeHost(ctx->dot_host);
  delete ctx;
}

const char *lmb_last_error(const lmb_ctx *ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int lmb_set_geometry(lmb_ctx *ctx, const int L[4], int nw, const double phase_re[4], const double phase_im[4],
                     const int coords[4], int dtype) {
  if (!ctx_ok(ctx)) return LMB_ERR_ARG;
  if (!L || !phase_re || !phase_im) return fail(ctx, LMB_ERR_ARG, "null geometry argument");
  if (nw < 0) return fail(ctx, LMB_ERR_ARG, "nw must be non-negative, got %d", nw);
  if (dtype != LMB_DTYPE_C128 && dtype != LMB_DTYPE_C64) return fail(ctx, LMB_ERR_ARG, "unknown dtype %d", dtype);
  int64_t V = 1;
  for (int mu = 0; mu < 4; mu++) {
    if (L[mu] <= 0) return fail(ctx, LMB_ERR_ARG, "global lattice sizes must be positive, got %d", L[mu]);
    if (nw > L[mu])
      return fail(ctx, LMB_ERR_ARG, "halo width nw=%d exceeds local lattice size %d in dimension %d", nw, L[mu],
                  mu + 1);
    const double re = phase_re[mu], im = phase_im[mu];
    if (re == 0.0 && im == 0.0)
      return fail(ctx, LMB_ERR_ARG, "boundary phases must be nonzero because negative wraps use inv(phase)");
    V *= L[mu];
  }
  if (V > (int64_t)0x7fffffff / 4) return fail(ctx, LMB_ERR_ARG, "local volume too large for one GPU context");
  Geom g{};
  int stride = 1;
  for (int mu = 0; mu < 4; mu++) {
    g.L[mu] = L[mu];
    g.stride[mu] = stride;
    stride *= L[mu];
    const double re = phase_re[mu], im = phase_im[mu], n = re * re + im * im;
    g.ph_fwd[mu][0] = re;
    g.ph_fwd[mu][1] = im;
    g.ph_bwd[mu][0] = re / n;
    g.ph_bwd[mu][1] = -im / n;
    if (!(re == 1.0 && im == 0.0)) g.phase_mask |= 1 << mu;
    g.eta_off[mu] = coords ? coords[mu] * L[mu] : 0;
  }
  g.V = V;
  const bool changed = !ctx->geom_set || std::memcmp(&g, &ctx->g, sizeof g) != 0 || ctx->pd.nw != nw ||
                       ctx->dtype != dtype;
  ctx->g = g;
  ctx->pd.nw = nw;
  for (int mu = 0; mu < 4; mu++) ctx->pd.P[mu] = L[mu] + 2 * nw;
  ctx->dtype = dtype;
  ctx->geom_set = true;
  if (changed) {
    for (auto &ls : ctx->links) ls.valid = false;
    ctx->smear.valid = false;
  }
  return LMB_OK;
}

int lmb_links_upload(lmb_ctx *ctx, int which, const void *const U[4], const uint64_t epoch[4], void *stream) {
  if (!ctx_ok(ctx)) return LMB_ERR_ARG;
  if (!ctx->geom_set) return fail(ctx, LMB_ERR_STATE, "lmb_set_geometry has not been called");
  if (which < 0 || which > 2) return fail(ctx, LMB_ERR_ARG, "unknown link set %d", which);
  if (!U) return fail(ctx, LMB_ERR_ARG, "null link array");
  for (int mu = 0; mu < 4; mu++)
    if (!U[mu]) return fail(ctx, LMB_ERR_ARG, "gauge link U[%d] is null", mu + 1);
  LinkSet &ls = ctx->links[which];
  if (which != LMB_LINKS_THIN) ctx->smear.valid = false;
  bool same = ls.valid;
  for (int mu = 0; mu < 4 && same; mu++)
    same = ls.ptr[mu] == U[mu] && epoch && ls.epoch[mu] == epoch[mu];
  if (same) return LMB_OK;
  cudaStream_t st = as_stream(stream);
  const int64_t V = ctx->g.V;
  if (!ls.d) LMB_CUDA(ctx, cudaMalloc(&ls.d, sizeof(double2) * 36 * V));
  if (ctx->dtype == LMB_DTYPE_C128)
    pack_links_kernel<double2><<<grid_for(V, 256), 256, 0, st>>>(
        ls.d, (const double2 *)U[0], (const double2 *)U[1], (const double2 *)U[2], (const double2 *)U[3], ctx->g,
        ctx->pd);
  else
    pack_links_kernel<float2><<<grid_for(V, 256), 256, 0, st>>>(ls.d, (const float2 *)U[0], (const float2 *)U[1],
                                                                (const float2 *)U[2], (const float2 *)U[3],
                                                                ctx->g, ctx->pd);
  LMB_CHECK_LAUNCH(ctx);
  int rc;
  ls.scale = device_absmax(ctx, ls.d, 36 * V, st, &rc);
  if (rc) return rc;
  {
    unsigned *bits = (unsigned *)workspace(ctx, "su3dev", sizeof(unsigned));
    if (!bits) return fail(ctx, LMB_ERR_CUDA, "out of device memory (su3 check)");
    LMB_CUDA(ctx, cudaMemsetAsync(bits, 0, sizeof(unsigned), st));
    su3_deviation_kernel<<<1184, 256, 0, st>>>(ls.d, V, bits);
    LMB_CHECK_LAUNCH(ctx);
    unsigned hb = 0;
    LMB_CUDA(ctx, cudaMemcpyAsync(&hb, bits, sizeof hb, cudaMemcpyDeviceToHost, st));
    LMB_CUDA(ctx, cudaStreamSynchronize(st));
    float dev;
    std::memcpy(&dev, &hb, sizeof dev);
    ls.su3_dev = dev;
  }
  for (int mu = 0; mu < 4; mu++) {
    ls.ptr[mu] = U[mu];
    ls.epoch[mu] = epoch ? epoch[mu] : 0;
  }
  ls.valid = true;
  ls.version++;
  return LMB_OK;
}

int lmb_wilson_apply(lmb_ctx *ctx, void *out, const void *in, double kappa, int dagger, int precision,
                     void *stream) {
  return apply_dispatch(ctx, WilsonPolicy{LMB_OP_WILSON, kappa, 0.0}, out, in, dagger, precision, stream);
}

int lmb_wilson_clover_apply(lmb_ctx *ctx, void *out, const void *in, double kappa, double csw, int dagger,
                            int precision, void *stream) {
  return apply_dispatch(ctx, WilsonPolicy{LMB_OP_WILSON_CLOVER, kappa, csw}, out, in, dagger, precision, stream);
}

int lmb_staggered_apply(lmb_ctx *ctx, void *out, const void *in, double mass, int dagger, int precision,
                        void *stream) {
  if (ctx && !std::isfinite(mass)) return fail(ctx, LMB_ERR_ARG, "mass must be finite");
  return apply_dispatch(ctx, StaggeredPolicy{false, mass, 0.0}, out, in, dagger, precision, stream);
}

int lmb_hisq_apply(lmb_ctx *ctx, void *out, const void *in, double mass, double naik_epsilon, int dagger,
                   int precision, void *stream) {
  if (ctx && !std::isfinite(mass)) return fail(ctx, LMB_ERR_ARG, "mass must be finite");
  if (ctx && !std::isfinite(naik_epsilon)) return fail(ctx, LMB_ERR_ARG, "naik_epsilon must be finite");
  return apply_dispatch(ctx, StaggeredPolicy{true, mass, naik_epsilon}, out, in, dagger, precision, stream);
}

int lmb_clover_field_strength(lmb_ctx *ctx, void *const F[6], void *stream) {
  if (!ctx_ok(ctx)) return LMB_ERR_ARG;
  if (!ctx->geom_set) return fail(ctx, LMB_ERR_STATE, "lmb_set_geometry has not been called");
  if (!ctx->links[LMB_LINKS_THIN].valid) return fail(ctx, LMB_ERR_STATE, "gauge links have not been uploaded");
  cudaStream_t st = as_stream(stream);
  int rc = ensure_field_strength(ctx, st);
  if (rc) return rc;
  for (int p = 0; p < 6; p++) {
    if (!F[p]) return fail(ctx, LMB_ERR_ARG, "null field-strength pointer %d", p);
    Field<PREC_DOUBLE, 9> f;
    f.data = ctx->clover.F + (size_t)p * 9 * ctx->g.V;
    f.norm = nullptr;
    f.V = ctx->g.V;
    rc = unpack_out(ctx, F[p], f, st);
    if (rc) return rc;
  }
  return LMB_OK;
}

int lmb_cg_ddagd(lmb_ctx *ctx, const lmb_cg_params *prm, void *x, const void *b, lmb_cg_result *res,
                 void *stream) {
  if (!ctx_ok(ctx)) return LMB_ERR_ARG;
  if (!prm || !res || !x || !b) return fail(ctx, LMB_ERR_ARG, "null argument");
  if (x == b) return fail(ctx, LMB_ERR_ARG, "CG fields x and b must not alias");
  if (!(prm->rtol >= 0)) return fail(ctx, LMB_ERR_ARG, "rtol must be nonnegative");
  if (!(prm->atol >= 0)) return fail(ctx, LMB_ERR_ARG, "atol must be nonnegative");
  if (!std::isfinite(prm->rtol)) return fail(ctx, LMB_ERR_ARG, "rtol must be finite");
  if (!std::isfinite(prm->atol)) return fail(ctx, LMB_ERR_ARG, "atol must be finite");
  if (prm->maxiter < 0) return fail(ctx, LMB_ERR_ARG, "maxiter must be nonnegative");
  if (prm->precision != PREC_DOUBLE && !(prm->delta > 0 && prm->delta < 1))
    return fail(ctx, LMB_ERR_ARG, "reliable-update delta must lie in (0, 1)");
  std::memset(res, 0, sizeof *res);
  cudaStream_t st = as_stream(stream);
  switch (prm->op) {
    case LMB_OP_WILSON:
    case LMB_OP_WILSON_CLOVER:
      return cg_dispatch(ctx, prm, WilsonPolicy{prm->op, prm->kappa, prm->csw}, x, b, res, st);
    case LMB_OP_STAGGERED:
      if (!std::isfinite(prm->mass)) return fail(ctx, LMB_ERR_ARG, "mass must be finite");
      return cg_dispatch(ctx, prm, StaggeredPolicy{false, prm->mass, 0.0}, x, b, res, st);
    case LMB_OP_HISQ:
      if (!std::isfinite(prm->mass)) return fail(ctx, LMB_ERR_ARG, "mass must be finite");
      return cg_dispatch(ctx, prm, StaggeredPolicy{true, prm->mass, prm->naik_epsilon}, x, b, res, st);
    case LMB_OP_DOMAINWALL:
      return cg_dispatch(ctx, prm, DWPolicy{}, x, b, res, st);
    default: return fail(ctx, LMB_ERR_ARG, "unknown operator %d", prm->op);
  }
}

int lmb_field_dot(lmb_ctx *ctx, const void *a, const void *b, int ncomp, double out[2], void *stream) {
  if (!ctx_ok(ctx)) return LMB_ERR_ARG;
  if (!ctx->geom_set) return fail(ctx, LMB_ERR_STATE, "lmb_set_geometry has not been called");
  if (!a || !b || !out) return fail(ctx, LMB_ERR_ARG, "null argument");
  cudaStream_t st = as_stream(stream);
  const unsigned grid = grid_for(ctx->g.V, 256);
  if (!ensure_partials(ctx, grid, 2)) return fail(ctx, LMB_ERR_CUDA, "out of device memory (partials)");
  double *dout = (double *)workspace(ctx, "dot_out", 2 * sizeof(double));
  if (!dout) return fail(ctx, LMB_ERR_CUDA, "out of device memory (dot)");
  const int c64 = ctx->dtype == LMB_DTYPE_C64;
  switch (ncomp) {
    case 1: dot_kernel<1><<<grid, 256, 0, st>>>(a, b, c64, ctx->g, ctx->pd, ctx->partials, ctx->counter, dout); break;
    case 3: dot_kernel<3><<<grid, 256, 0, st>>>(a, b, c64, ctx->g, ctx->pd, ctx->partials, ctx->counter, dout); break;
    case 9: dot_kernel<9><<<grid, 256, 0, st>>>(a, b, c64, ctx->g, ctx->pd, ctx->partials, ctx->counter, dout); break;
    case 12: dot_kernel<12><<<grid, 256, 0, st>>>(a, b, c64, ctx->g, ctx->pd, ctx->partials, ctx->counter, dout); break;
    default: return fail(ctx, LMB_ERR_UNSUPPORTED, "dot over %d components per site is not provided", ncomp);
  }
  LMB_CHECK_LAUNCH(ctx);
  LMB_CUDA(ctx, cudaMemcpyAsync(ctx->dot_host, dout, 2 * sizeof(double), cudaMemcpyDeviceToHost, st));
  LMB_CUDA(ctx, cudaStreamSynchronize(st));
  out[0] = ctx->dot_host[0];
  out[1] = ctx->dot_host[1];
  return LMB_OK;
}


int lmb_random_su3_links(lmb_ctx *ctx, void *const U[4], double amplitude, uint64_t seed, void *stream) {
  if (!ctx_ok(ctx)) return LMB_ERR_ARG;
  if (!ctx->geom_set) return fail(ctx, LMB_ERR_STATE, "lmb_set_geometry has not been called");
  if (!U) return fail(ctx, LMB_ERR_ARG, "null link array");
  for (int mu = 0; mu < 4; mu++)
    if (!U[mu]) return fail(ctx, LMB_ERR_ARG, "gauge link U[%d] is null", mu + 1);
  cudaStream_t st = as_stream(stream);
  const unsigned grid = grid_for(4 * ctx->g.V, 128);
  if (ctx->dtype == LMB_DTYPE_C128)
    random_su3_kernel<double2><<<grid, 128, 0, st>>>((double2 *)U[0], (double2 *)U[1], (double2 *)U[2],
                                                      (double2 *)U[3], ctx->g, ctx->pd, amplitude, seed);
  else
    random_su3_kernel<float2><<<grid, 128, 0, st>>>((float2 *)U[0], (float2 *)U[1], (float2 *)U[2],
                                                     (float2 *)U[3], ctx->g, ctx->pd, amplitude, seed);
  LMB_CHECK_LAUNCH(ctx);
  return LMB_OK;
}

int lmb_gaussian_field(lmb_ctx *ctx, void *out, int ncomp, uint64_t seed, void *stream) {
  if (!ctx_ok(ctx)) return LMB_ERR_ARG;
  if (!ctx->geom_set) return fail(ctx, LMB_ERR_STATE, "lmb_set_geometry has not been called");
  if (!out) return fail(ctx, LMB_ERR_ARG, "null field");
  if (ncomp <= 0) return fail(ctx, LMB_ERR_ARG, "ncomp must be positive");
  cudaStream_t st = as_stream(stream);
  const unsigned grid = grid_for(ctx->g.V, 256);
  if (ctx->dtype == LMB_DTYPE_C128)
    gaussian_field_kernel<double2><<<grid, 256, 0, st>>>((double2 *)out, ncomp, ctx->g, ctx->pd, seed);
  else
    gaussian_field_kernel<float2><<<grid, 256, 0, st>>>((float2 *)out, ncomp, ctx->g, ctx->pd, seed);
  LMB_CHECK_LAUNCH(ctx);
  return LMB_OK;
}


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


int lmb_cg_ddagd_batched(lmb_ctx *ctx, const lmb_cg_params *prm, int nlattices, const lmb_batch_lattice *lattices,
                         lmb_cg_result *results, lmb_batch_tuning *tuning, void *stream) {
  if (!ctx_ok(ctx)) return LMB_ERR_ARG;
  if (!prm || !lattices || !results || nlattices <= 0) return fail(ctx, LMB_ERR_ARG, "null or empty argument");
  if (prm->op != LMB_OP_WILSON) return fail(ctx, LMB_ERR_UNSUPPORTED, "batched CG is built for the Wilson operator");
  if (prm->precision != PREC_SINGLE)
    return fail(ctx, LMB_ERR_UNSUPPORTED, "batched CG runs FP32 inner iterations (LMB_PREC_SINGLE)");
  if (!(prm->rtol >= 0) || !std::isfinite(prm->rtol)) return fail(ctx, LMB_ERR_ARG, "rtol must be nonnegative");
  if (!(prm->atol >= 0) || !std::isfinite(prm->atol)) return fail(ctx, LMB_ERR_ARG, "atol must be nonnegative");
  if (prm->maxiter < 0) return fail(ctx, LMB_ERR_ARG, "maxiter must be nonnegative");
  if (!(prm->delta > 0 && prm->delta < 1)) return fail(ctx, LMB_ERR_ARG, "reliable-update delta must lie in (0, 1)");
  return cg_batched(ctx, prm, nlattices, lattices, results, tuning, as_stream(stream));
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
    rc = op.launch<PREC_DOUBLE>(ctx, y, 0, e, st);
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
  rc = full.launch<PREC_DOUBLE>(ctx, xf, 0, er, st);
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

int lmb_set_halo(void *field, int dtype, int ncomp, int D, const int *L, int nw, const double *phase_re,
                 const double *phase_im, void *stream) {
  if (!field || !L || !phase_re || !phase_im) return LMB_ERR_ARG;
  if ((dtype != LMB_DTYPE_C128 && dtype != LMB_DTYPE_C64) || ncomp <= 0 || (D != 4 && D != 5) || nw < 0)
    return LMB_ERR_ARG;
  HaloGeom h{};
  h.D = D;
  h.nw = nw;
  h.npad = 1;
  for (int d = 0; d < D; d++) {
    if (L[d] <= 0 || nw > L[d]) return LMB_ERR_ARG;
    const double re = phase_re[d], im = phase_im[d], m2 = re * re + im * im;
    if (!(m2 > 0) || !std::isfinite(m2)) return LMB_ERR_ARG;
    h.L[d] = L[d];
    h.P[d] = L[d] + 2 * nw;
    h.ph[d][0] = re;
    h.ph[d][1] = im;
    h.iph[d][0] = re / m2;
    h.iph[d][1] = -im / m2;
    h.npad *= h.P[d];
  }
  if (nw == 0) return LMB_OK;
  cudaStream_t st = as_stream(stream);
  const unsigned grid = grid_for(h.npad, 256);
  if (dtype == LMB_DTYPE_C128)
    set_halo_kernel<double2><<<grid, 256, 0, st>>>((double2 *)field, ncomp, h);
  else
    set_halo_kernel<float2><<<grid, 256, 0, st>>>((float2 *)field, ncomp, h);
  return cudaGetLastError() == cudaSuccess ? LMB_OK : LMB_ERR_CUDA;
}

int lmb_domainwall_set(lmb_ctx *ctx, int L5, double mass, double M, const double *a, const double *b,
                       const double *c, void *stream) {
  if (!ctx_ok(ctx)) return LMB_ERR_ARG;
  if (L5 <= 0) return fail(ctx, LMB_ERR_ARG, "L5 must be positive");
  if (!a || !b || !c) return fail(ctx, LMB_ERR_ARG, "null coefficient array");
  if (!std::isfinite(mass) || !std::isfinite(M)) return fail(ctx, LMB_ERR_ARG, "mass and M must be finite");
  std::vector<double> h(3 * (size_t)L5);
  for (int s = 0; s < L5; s++) {
    h[s] = a[s];
    h[L5 + s] = b[s];
    h[2 * L5 + s] = c[s];
  }
  for (double v : h)
    if (!std::isfinite(v)) return fail(ctx, LMB_ERR_ARG, "domain-wall coefficients must all be finite");
  if (ctx->dw_coef_cap < 3 * L5) {
    cudaFree(ctx->dw_coef);
    ctx->dw_coef = nullptr;
    ctx->dw_coef_cap = 0;
    LMB_CUDA(ctx, cudaMalloc(&ctx->dw_coef, sizeof(double) * 3 * L5));
    ctx->dw_coef_cap = 3 * L5;
  }
  // ordered on the stream after the kernels that read the previous values
  LMB_CUDA(ctx, cudaMemcpyAsync(ctx->dw_coef, h.data(), sizeof(double) * 3 * L5, cudaMemcpyHostToDevice,
                                as_stream(stream)));
  LMB_CUDA(ctx, cudaStreamSynchronize(as_stream(stream)));
  ctx->dw_L5 = L5;
  ctx->dw_mass = mass;
  ctx->dw_M = M;
  return LMB_OK;
}

int lmb_domainwall_apply(lmb_ctx *ctx, void *out, const void *in, int dagger, int precision, void *stream) {
  return apply_dispatch(ctx, DWPolicy{}, out, in, dagger, precision, stream);
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
