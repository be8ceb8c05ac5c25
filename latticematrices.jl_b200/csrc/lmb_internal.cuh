// lmb_internal.cuh -- host-side helpers shared by the translation units of
// liblmb200.so: stream and argument checks, the views of the link and clover
// caches the kernels take, and the cache builders (defined in lmb_capi.cu and
// lmb_schur_ops.cu).
#pragma once
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <type_traits>
#include <vector>

#include "lmb_context.cuh"

namespace lmb {

inline cudaStream_t as_stream(void *s) { return (cudaStream_t)s; }

inline bool ctx_ok(lmb_ctx *ctx) { return ctx != nullptr; }

// blocks of kernel `kern` (kDslashThreads threads, no dynamic shared memory)
// resident on the whole device at once: the grid of a persistent launch.
// The per-SM figure depends only on the kernel and the architecture, so it
// is looked up once per kernel (lmb_capi.cu).
int resident_blocks_per_sm(const void *kern);
template <class K>
unsigned resident_grid(const lmb_ctx *ctx, K kern) {
  return (unsigned)(resident_blocks_per_sm((const void *)kern) * (ctx->sm_count > 0 ? ctx->sm_count : 1));
}

inline int check_prec(lmb_ctx *ctx, int prec) {
  if (prec < PREC_DOUBLE || prec > PREC_HALF) return fail(ctx, LMB_ERR_ARG, "unknown precision %d", prec);
  return LMB_OK;
}

// link and clover caches (lmb_capi.cu)
// Vset: volume of the set (default: the context's)
int ensure_link_precision(lmb_ctx *ctx, LinkSet &ls, int prec, cudaStream_t st, bool allow_recon = true,
                          int64_t Vset = -1);
float device_absmax(lmb_ctx *ctx, const double2 *p, int64_t n, cudaStream_t st, int *rc);
int ensure_field_strength(lmb_ctx *ctx, cudaStream_t st);
int ensure_clover(lmb_ctx *ctx, double coef, int prec, cudaStream_t st);
int clover_convert(lmb_ctx *ctx, CloverCache &cc, int prec, cudaStream_t st);
int read_state(lmb_ctx *ctx, cudaStream_t st);
int pack_links_to(lmb_ctx *ctx, double2 *dst, const void *const U[4], cudaStream_t st);
int unpack_links_from(lmb_ctx *ctx, void *const U[4], const double2 *src, cudaStream_t st);
int check_links_arg(lmb_ctx *ctx, const void *const U[4], const char *what);
void release_site_caches(lmb_ctx *ctx);
// F_mu_nu of a process-grid block from the caller's halo-filled links (lmb_dist_ops.cu)
int dist_field_strength(lmb_ctx *ctx, cudaStream_t st);
// even/odd caches (lmb_schur_ops.cu)
int ensure_clover_inverse(lmb_ctx *ctx, int prec, cudaStream_t st);
int ensure_eo_copies(lmb_ctx *ctx, int prec, bool clover, cudaStream_t st);
const char *eo_buffer(lmb_ctx *ctx, const std::string &name);

template <int P> Gauge12<P> gauge12_view(const LinkSet &ls, int64_t V);
template <> inline Gauge12<PREC_DOUBLE> gauge12_view<PREC_DOUBLE>(const LinkSet &ls, int64_t V) { return {ls.d12, V, 1.f}; }
template <> inline Gauge12<PREC_SINGLE> gauge12_view<PREC_SINGLE>(const LinkSet &ls, int64_t V) { return {ls.f12, V, 1.f}; }
template <> inline Gauge12<PREC_HALF> gauge12_view<PREC_HALF>(const LinkSet &ls, int64_t V) { return {ls.h12, V, 1.f}; }

template <int P> Gauge<P> gauge_view(const LinkSet &ls, int64_t V);
template <> inline Gauge<PREC_DOUBLE> gauge_view<PREC_DOUBLE>(const LinkSet &ls, int64_t V) { return {ls.d, V, ls.scale}; }
template <> inline Gauge<PREC_SINGLE> gauge_view<PREC_SINGLE>(const LinkSet &ls, int64_t V) {
  return {(const float4 *)ls.f, V, ls.scale};
}
template <> inline Gauge<PREC_HALF> gauge_view<PREC_HALF>(const LinkSet &ls, int64_t V) {
  return {ls.h, V, base_of_exponent(pow2_exponent(ls.scale))};
}

template <int P> Clover<P> clover_view(const CloverCache &cc, int64_t V);
template <> inline Clover<PREC_DOUBLE> clover_view<PREC_DOUBLE>(const CloverCache &cc, int64_t V) { return {cc.d, V, cc.scale}; }
template <> inline Clover<PREC_SINGLE> clover_view<PREC_SINGLE>(const CloverCache &cc, int64_t V) { return {cc.f, V, cc.scale}; }
template <> inline Clover<PREC_HALF> clover_view<PREC_HALF>(const CloverCache &cc, int64_t V) {
  Clover<PREC_HALF> c;
  c.data = cc.h;
  c.tail = cc.ht;
  c.V = V;
  c.scale = cc.scale;
  return c;
}

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


}  // namespace lmb
