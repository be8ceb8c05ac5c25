// lmb_capi.cu -- extern "C" entry points of liblmb200.so (declared in
// include/lmb200.h): context, geometry, link upload and caches, operator
// application, the D^+D CG entry, inner product, seeded inputs, halo fill.
// The operator drivers are instantiated in their own translation units
// (lmb_wilson_*.cu, lmb_staggered_ops.cu, lmb_dw_ops.cu); the even/odd solve,
// batched CG and the smearing / force chains live in lmb_schur_ops.cu,
// lmb_batch_ops.cu and lmb_force_ops.cu.
#include "lmb_halo.cuh"
#include "lmb_hisq_smear.cuh"
#include "lmb_op_dist.cuh"
#include "lmb_op_dw.cuh"
#include "lmb_op_staggered.cuh"
#include "lmb_op_wilson.cuh"
#include "lmb_random.cuh"

using namespace lmb;

namespace lmb {

// ---------------------------------------------------------------------------
// link caches
// ---------------------------------------------------------------------------
int ensure_link_precision(lmb_ctx *ctx, LinkSet &ls, int prec, cudaStream_t st, bool allow_recon, int64_t Vset) {
  const int64_t V = Vset >= 0 ? Vset : ctx->g.V;
  const int64_t n = 36 * V;
  if (prec != PREC_DOUBLE && !ls.finite())
    return fail(ctx, LMB_ERR_ARG, "gauge links hold a non-finite entry (or one beyond FP32 range): "
                "FP32 and int16 storage need finite links");
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

// The link sets and clover caches are sized by the volume they were built
// for: free them (the next use rebuilds them) when that volume goes away.
// Version counters keep counting across a release, so nothing keyed by an
// old version (parity-ordered copies, derived caches) can match again.
void release_site_caches(lmb_ctx *ctx) {
  for (auto &ls : ctx->links) {
    cudaFree(ls.d);
    cudaFree(ls.f);
    cudaFree(ls.h);
    cudaFree(ls.d12);
    cudaFree(ls.f12);
    cudaFree(ls.h12);
    const uint64_t version = ls.version + 1;
    ls = LinkSet{};
    ls.version = version;
  }
  for (CloverCache *cc : {&ctx->clover, &ctx->clover_inv}) {
    cudaFree(cc->F);
    cudaFree(cc->d);
    cudaFree(cc->f);
    cudaFree(cc->h);
    cudaFree(cc->ht);
    const uint64_t dv = cc->d_version + 1;
    *cc = CloverCache{};
    cc->d_version = dv;
  }
  ctx->smear.valid = false;
}

int resident_blocks_per_sm(const void *kern) {
  static std::mutex mu;
  static std::map<const void *, int> cache;
  std::lock_guard<std::mutex> lock(mu);
  auto it = cache.find(kern);
  if (it != cache.end()) return it->second;
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kern, kDslashThreads, 0) != cudaSuccess || n < 1) n = 1;
  cache[kern] = n;
  return n;
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

// ---------------------------------------------------------------------------
// clover cache
// ---------------------------------------------------------------------------
int ensure_field_strength(lmb_ctx *ctx, cudaStream_t st) {
  CloverCache &cc = ctx->clover;
  const LinkSet &ls = ctx->links[LMB_LINKS_THIN];
  if (cc.F_valid && cc.F_links_version == ls.version) return LMB_OK;
  const int64_t V = ctx->g.V;
  if (!cc.F) LMB_CUDA(ctx, cudaMalloc(&cc.F, sizeof(double2) * 54 * V));
  if (ctx->dist && ctx->dist->split) {
    // a block of a process grid: the leaves reach the neighbours' links
    const int rc = dist_field_strength(ctx, st);
    if (rc) return rc;
  } else {
    clover_field_strength_kernel<<<grid_for(6 * V, 128), 128, 0, st>>>(cc.F, ls.d, ctx->g);
    LMB_CHECK_LAUNCH(ctx);
  }
  cc.F_valid = true;
  cc.F_links_version = ls.version;
  return LMB_OK;
}

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

int read_state(lmb_ctx *ctx, cudaStream_t st) {
  LMB_CUDA(ctx, cudaMemcpyAsync(ctx->st_host, ctx->st_dev, sizeof(CGState), cudaMemcpyDeviceToHost, st));
  LMB_CUDA(ctx, cudaStreamSynchronize(st));
  return LMB_OK;
}

// K3: p = r + beta p; FP32 / int16 Wilson fields of an even volume use the
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

int check_links_arg(lmb_ctx *ctx, const void *const U[4], const char *what) {
  if (!U) return fail(ctx, LMB_ERR_ARG, "null %s array", what);
  for (int mu = 0; mu < 4; mu++)
    if (!U[mu]) return fail(ctx, LMB_ERR_ARG, "%s[%d] is null", what, mu + 1);
  return LMB_OK;
}


// the operator of a whole lattice, or of a block of a process grid
template <class Fn>
int with_wilson(const lmb_ctx *ctx, const WilsonPolicy &op, Fn fn) {
  if (ctx && ctx->dist) return fn(DistWilsonPolicy{op});
  return fn(op);
}
template <class Fn>
int with_staggered(const lmb_ctx *ctx, const StaggeredPolicy &op, Fn fn) {
  if (ctx && ctx->dist) return fn(DistStaggeredPolicy{op});
  return fn(op);
}

}  // namespace lmb

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
  if (const char *pe = getenv("LMB_PERSISTENT")) ctx->persistent = atoi(pe) != 0;
  if (const char *bf = getenv("LMB_BATCH_FAMILY")) ctx->batch_family = atoi(bf);
  if (cudaDeviceGetAttribute(&ctx->sm_count, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) {
    delete ctx;
    return nullptr;
  }
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
  release_site_caches(ctx);
  dist_release(ctx);
  cudaFree(ctx->dw_coef);
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
  if (V != ctx->cache_V) {  // caches built for another volume
    release_site_caches(ctx);
    ctx->cache_V = V;
  }
  if (changed && ctx->dist) {  // boundary lists and link ghosts follow the block
    for (auto &kv : ctx->dist->boundary) cudaFree(kv.second.first);
    ctx->dist->boundary.clear();
    for (auto &v : ctx->dist->ghost_of_version) v = ~0ull;
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
  return with_wilson(ctx, WilsonPolicy{LMB_OP_WILSON, kappa, 0.0},
                     [&](const auto &op) { return apply_dispatch(ctx, op, out, in, dagger, precision, stream); });
}

int lmb_wilson_clover_apply(lmb_ctx *ctx, void *out, const void *in, double kappa, double csw, int dagger,
                            int precision, void *stream) {
  return with_wilson(ctx, WilsonPolicy{LMB_OP_WILSON_CLOVER, kappa, csw},
                     [&](const auto &op) { return apply_dispatch(ctx, op, out, in, dagger, precision, stream); });
}

int lmb_staggered_apply(lmb_ctx *ctx, void *out, const void *in, double mass, int dagger, int precision,
                        void *stream) {
  if (ctx && !std::isfinite(mass)) return fail(ctx, LMB_ERR_ARG, "mass must be finite");
  return with_staggered(ctx, StaggeredPolicy{false, mass, 0.0},
                        [&](const auto &op) { return apply_dispatch(ctx, op, out, in, dagger, precision, stream); });
}

int lmb_hisq_apply(lmb_ctx *ctx, void *out, const void *in, double mass, double naik_epsilon, int dagger,
                   int precision, void *stream) {
  if (ctx && !std::isfinite(mass)) return fail(ctx, LMB_ERR_ARG, "mass must be finite");
  if (ctx && !std::isfinite(naik_epsilon)) return fail(ctx, LMB_ERR_ARG, "naik_epsilon must be finite");
  return with_staggered(ctx, StaggeredPolicy{true, mass, naik_epsilon},
                        [&](const auto &op) { return apply_dispatch(ctx, op, out, in, dagger, precision, stream); });
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
  auto cg = [&](const auto &op) { return cg_dispatch(ctx, prm, op, x, b, res, st); };
  switch (prm->op) {
    case LMB_OP_WILSON:
    case LMB_OP_WILSON_CLOVER:
      return with_wilson(ctx, WilsonPolicy{prm->op, prm->kappa, prm->csw}, cg);
    case LMB_OP_STAGGERED:
      if (!std::isfinite(prm->mass)) return fail(ctx, LMB_ERR_ARG, "mass must be finite");
      return with_staggered(ctx, StaggeredPolicy{false, prm->mass, 0.0}, cg);
    case LMB_OP_HISQ:
      if (!std::isfinite(prm->mass)) return fail(ctx, LMB_ERR_ARG, "mass must be finite");
      return with_staggered(ctx, StaggeredPolicy{true, prm->mass, prm->naik_epsilon}, cg);
    case LMB_OP_DOMAINWALL:
      if (ctx->dist) return fail(ctx, LMB_ERR_UNSUPPORTED, "the domain-wall operator takes one rank per lattice");
      return cg_dispatch(ctx, prm, DWPolicy{}, x, b, res, st);
    default: return fail(ctx, LMB_ERR_ARG, "unknown operator %d", prm->op);
  }
}

int lmb_operator_timing(lmb_ctx *ctx, const lmb_cg_params *prm, const void *in, int napply, int dagger,
                        double *ms_per_apply, void *stream) {
  if (!ctx_ok(ctx)) return LMB_ERR_ARG;
  if (!prm || !in || !ms_per_apply) return fail(ctx, LMB_ERR_ARG, "null argument");
  const int prec = prm->precision;
  auto timing = [&](const auto &op) {
    return time_dispatch(ctx, op, in, napply, dagger, prec, ms_per_apply, stream);
  };
  switch (prm->op) {
    case LMB_OP_WILSON:
    case LMB_OP_WILSON_CLOVER:
      return with_wilson(ctx, WilsonPolicy{prm->op, prm->kappa, prm->csw}, timing);
    case LMB_OP_STAGGERED:
      return with_staggered(ctx, StaggeredPolicy{false, prm->mass, 0.0}, timing);
    case LMB_OP_HISQ:
      return with_staggered(ctx, StaggeredPolicy{true, prm->mass, prm->naik_epsilon}, timing);
    case LMB_OP_DOMAINWALL:
      return time_dispatch(ctx, DWPolicy{}, in, napply, dagger, prec, ms_per_apply, stream);
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
  if (ctx && ctx->dist) return fail(ctx, LMB_ERR_UNSUPPORTED, "the domain-wall operator takes one rank per lattice");
  return apply_dispatch(ctx, DWPolicy{}, out, in, dagger, precision, stream);
}


}  // extern "C"
