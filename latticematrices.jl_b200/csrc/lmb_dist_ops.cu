// lmb_dist_ops.cu -- the sharded path's host side: process grid and NCCL
// communicator of a context (lmb_set_process_grid), ghost links and boundary
// lists, the all-reduce of the partial sums and F_mu_nu of a block.  The
// operator drivers are instantiated per precision in lmb_dist_{d,s,h}.cu.
#include <algorithm>
#include <dlfcn.h>

#include "lmb_op_dist.cuh"

using namespace lmb;

namespace lmb {

const NcclApi &nccl_api() {
  static NcclApi api;
  static std::once_flag once;
  std::call_once(once, [] {
    void *h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_GLOBAL);
    if (!h) h = dlopen("libnccl.so", RTLD_NOW | RTLD_GLOBAL);
    if (!h) {
      api.error = std::string("NCCL is not available: ") + dlerror();
      return;
    }
    bool ok = true;
    auto sym = [&](const char *name) {
      void *p = dlsym(h, name);
      if (!p) ok = false;
      return p;
    };
    api.GetUniqueId = (decltype(api.GetUniqueId))sym("ncclGetUniqueId");
    api.CommInitRank = (decltype(api.CommInitRank))sym("ncclCommInitRank");
    api.CommDestroy = (decltype(api.CommDestroy))sym("ncclCommDestroy");
    api.Send = (decltype(api.Send))sym("ncclSend");
    api.Recv = (decltype(api.Recv))sym("ncclRecv");
    api.GroupStart = (decltype(api.GroupStart))sym("ncclGroupStart");
    api.GroupEnd = (decltype(api.GroupEnd))sym("ncclGroupEnd");
    api.AllReduce = (decltype(api.AllReduce))sym("ncclAllReduce");
    api.GetErrorString = (decltype(api.GetErrorString))sym("ncclGetErrorString");
    api.loaded = ok;
    if (!ok) api.error = "NCCL library lacks a required entry point";
  });
  return api;
}

DistView dist_view(const lmb_ctx *ctx, int depth) {
  DistView dv{};
  dv.split = ctx->dist ? ctx->dist->split : 0u;
  dv.depth = depth;
  const Geom &g = ctx->g;
  for (int mu = 0; mu < 4; mu++) {
    dv.face[mu] = (int)(g.V / g.L[mu]);
    int stride = 1;
    for (int nu = 0; nu < 4; nu++) {
      if (nu == mu) {
        dv.fstr[mu][nu] = 0;
        continue;
      }
      dv.fstr[mu][nu] = stride;
      stride *= g.L[nu];
    }
  }
  int64_t np = 1;
  for (int mu = 0; mu < 4; mu++) {
    const int lo = ((dv.split >> mu) & 1) ? depth : 0, hi = g.L[mu] - lo;
    dv.plo[mu] = mu == 0 ? (lo + 1) / 2 : lo;
    dv.pn[mu] = std::max(0, mu == 0 ? hi / 2 - dv.plo[0] : hi - lo);
    np *= dv.pn[mu];
  }
  dv.npairs = (int)np;
  int64_t ns = 1;
  for (int mu = 0; mu < 4; mu++) {
    const int lo = ((dv.split >> mu) & 1) ? depth : 0;
    dv.slo[mu] = lo;
    dv.sn[mu] = std::max(0, g.L[mu] - 2 * lo);
    ns *= dv.sn[mu];
  }
  dv.nsites = (int)ns;
  return dv;
}

int dist_boundary(lmb_ctx *ctx, int depth, bool pairs, const int **list, int *n) {
  lmb_dist *d = ctx->dist;
  const int key = 2 * depth + (pairs ? 1 : 0);
  auto it = d->boundary.find(key);
  if (it == d->boundary.end()) {
    const Geom &g = ctx->g;
    auto on_boundary = [&](const int *c) {
      for (int mu = 0; mu < 4; mu++)
        if (((d->split >> mu) & 1) && (c[mu] < depth || c[mu] >= g.L[mu] - depth)) return true;
      return false;
    };
    std::vector<int> sites;
    for (int64_t s = 0; s < g.V; s++) {
      int64_t q = s;
      int c[4];
      for (int mu = 0; mu < 4; mu++) {
        c[mu] = (int)(q % g.L[mu]);
        q /= g.L[mu];
      }
      bool b = on_boundary(c);
      if (!b && pairs) {
        int cp[4] = {c[0] ^ 1, c[1], c[2], c[3]};
        b = cp[0] < g.L[0] && on_boundary(cp);
      }
      if (b) sites.push_back((int)s);
    }
    int *dev = nullptr;
    if (!sites.empty()) {
      LMB_CUDA(ctx, cudaMalloc(&dev, sizeof(int) * sites.size()));
      LMB_CUDA(ctx, cudaMemcpy(dev, sites.data(), sizeof(int) * sites.size(), cudaMemcpyHostToDevice));
    }
    it = d->boundary.emplace(key, std::make_pair(dev, (int)sites.size())).first;
  }
  *list = it->second.first;
  *n = it->second.second;
  return LMB_OK;
}

int dist_link_ghosts(lmb_ctx *ctx, int which, int depth, int prec, bool allow_recon, cudaStream_t st) {
  lmb_dist *d = ctx->dist;
  const LinkSet &ls = ctx->links[which];
  if (ls.version != d->ghost_of_version[which] || depth > d->ghost_depth[which]) {
    if (ctx->pd.nw < depth)
      return fail(ctx, LMB_ERR_ARG, "a split lattice needs halo width nw >= %d for its link ghosts, got %d", depth,
                  ctx->pd.nw);
    for (int mu = 0; mu < 4; mu++)
      if (!ls.ptr[mu]) return fail(ctx, LMB_ERR_STATE, "link ghosts need the caller's padded links");
    const DistView dv = dist_view(ctx, depth);
    for (int mu = 0; mu < 4; mu++) {
      LinkSet &gs = d->ghost[which][mu];
      cudaFree(gs.d);
      cudaFree(gs.f);
      cudaFree(gs.h);
      cudaFree(gs.d12);
      cudaFree(gs.f12);
      cudaFree(gs.h12);
      const uint64_t version = gs.version + 1;
      gs = LinkSet{};
      gs.version = version;
      if (!((d->split >> mu) & 1)) continue;
      const int64_t Vg = (int64_t)depth * dv.face[mu];
      LMB_CUDA(ctx, cudaMalloc(&gs.d, sizeof(double2) * 36 * Vg));
      LMB_CUDA(ctx, cudaMemsetAsync(gs.d, 0, sizeof(double2) * 36 * Vg, st));
      const unsigned grid = grid_for(Vg, 256);
      if (ctx->dtype == LMB_DTYPE_C128)
        pack_link_ghost_kernel<double2><<<grid, 256, 0, st>>>(gs.d, (const double2 *)ls.ptr[mu], ctx->g, ctx->pd,
                                                               dv, mu);
      else
        pack_link_ghost_kernel<float2><<<grid, 256, 0, st>>>(gs.d, (const float2 *)ls.ptr[mu], ctx->g, ctx->pd, dv,
                                                              mu);
      LMB_CHECK_LAUNCH(ctx);
      int rc = LMB_OK;
      gs.scale = device_absmax(ctx, gs.d, 36 * Vg, st, &rc);
      if (rc) return rc;
      gs.su3_dev = ls.su3_dev;  // the same field: reconstruct-12 exactly when the block does
      gs.valid = true;
    }
    d->ghost_of_version[which] = ls.version;
    d->ghost_depth[which] = depth;
  }
  const DistView dv = dist_view(ctx, d->ghost_depth[which]);
  for (int mu = 0; mu < 4; mu++) {
    if (!((d->split >> mu) & 1)) continue;
    const int rc = ensure_link_precision(ctx, d->ghost[which][mu], prec, st, allow_recon,
                                         (int64_t)d->ghost_depth[which] * dv.face[mu]);
    if (rc) return rc;
  }
  return LMB_OK;
}

int dist_allreduce_sums(lmb_ctx *ctx, cudaStream_t st) {
  const NcclApi &nc = nccl_api();
  const ncclResult_t r = nc.AllReduce(ctx->dist->sums, ctx->dist->sums, 2, ncclFloat64, ncclSum, ctx->dist->comm, st);
  if (r != ncclSuccess) return fail(ctx, LMB_ERR_CUDA, "NCCL all-reduce: %s", nc.GetErrorString(r));
  return LMB_OK;
}

void dist_release(lmb_ctx *ctx) {
  lmb_dist *d = ctx->dist;
  if (!d) return;
  if (d->comm) nccl_api().CommDestroy(d->comm);
  if (d->comm_stream) cudaStreamDestroy(d->comm_stream);
  if (d->bnd_stream) cudaStreamDestroy(d->bnd_stream);
  if (d->ev_packed) cudaEventDestroy(d->ev_packed);
  if (d->ev_comm) cudaEventDestroy(d->ev_comm);
  if (d->ev_bnd) cudaEventDestroy(d->ev_bnd);
  cudaFree(d->bcounter);
  cudaFree(d->sums);
  for (auto &kv : d->boundary) cudaFree(kv.second.first);
  for (auto &set : d->ghost)
    for (auto &gs : set) {
      cudaFree(gs.d);
      cudaFree(gs.f);
      cudaFree(gs.h);
      cudaFree(gs.d12);
      cudaFree(gs.f12);
      cudaFree(gs.h12);
    }
  delete d;
  ctx->dist = nullptr;
}

// F_mu_nu of a block: the padded block of the caller's links (halo filled by
// the caller's exchange, corners included) is a lattice of the padded
// extents; the single-lattice kernel computes F on it, and the core sites,
// whose leaves reach one site into the halo, are exact.
int dist_field_strength(lmb_ctx *ctx, cudaStream_t st) {
  const LinkSet &ls = ctx->links[LMB_LINKS_THIN];
  if (ctx->pd.nw < 1) return fail(ctx, LMB_ERR_ARG, "the clover term of a split lattice needs nw >= 1");
  for (int mu = 0; mu < 4; mu++)
    if (!ls.ptr[mu]) return fail(ctx, LMB_ERR_STATE, "the clover term of a split lattice needs the padded links");
  Geom gp{};
  int64_t Vp = 1;
  for (int mu = 0; mu < 4; mu++) {
    gp.L[mu] = ctx->pd.P[mu];
    gp.stride[mu] = (int)Vp;
    Vp *= ctx->pd.P[mu];
    gp.ph_fwd[mu][0] = gp.ph_bwd[mu][0] = 1.0;
  }
  gp.V = Vp;
  double2 *Up = (double2 *)workspace(ctx, "dist_block_links", sizeof(double2) * 36 * Vp);
  double2 *Fp = (double2 *)workspace(ctx, "dist_block_F", sizeof(double2) * 54 * Vp);
  if (!Up || !Fp) return fail(ctx, LMB_ERR_CUDA, "out of device memory (block field strength)");
  const unsigned grid = grid_for(Vp, 256);
  if (ctx->dtype == LMB_DTYPE_C128)
    padded_block_links_kernel<double2><<<grid, 256, 0, st>>>(Up, (const double2 *)ls.ptr[0],
                                                              (const double2 *)ls.ptr[1], (const double2 *)ls.ptr[2],
                                                              (const double2 *)ls.ptr[3], Vp);
  else
    padded_block_links_kernel<float2><<<grid, 256, 0, st>>>(Up, (const float2 *)ls.ptr[0], (const float2 *)ls.ptr[1],
                                                             (const float2 *)ls.ptr[2], (const float2 *)ls.ptr[3], Vp);
  clover_field_strength_kernel<<<grid_for(6 * Vp, 128), 128, 0, st>>>(Fp, Up, gp);
  core_of_padded_kernel<<<grid_for(ctx->g.V, 256), 256, 0, st>>>(ctx->clover.F, Fp, ctx->g, ctx->pd, Vp);
  LMB_CHECK_LAUNCH(ctx);
  return LMB_OK;
}

}  // namespace lmb

extern "C" {

int lmb_nccl_unique_id(void *id) {
  if (!id) return LMB_ERR_ARG;
  const NcclApi &nc = nccl_api();
  if (!nc.loaded) return LMB_ERR_UNSUPPORTED;
  ncclUniqueId u;
  if (nc.GetUniqueId(&u) != ncclSuccess) return LMB_ERR_CUDA;
  std::memcpy(id, u.internal, NCCL_UNIQUE_ID_BYTES);
  return LMB_OK;
}

int lmb_set_process_grid(lmb_ctx *ctx, const void *nccl_id, int nranks, int rank, const int dims[4],
                         const int coords[4], unsigned split_mask, const int nb_minus[4], const int nb_plus[4]) {
  if (!ctx_ok(ctx)) return LMB_ERR_ARG;
  dist_release(ctx);
  // F_mu_nu and the clover blocks depend on which dimensions are split:
  // the next upload rebuilds every link-derived cache
  for (auto &ls : ctx->links) ls.valid = false;
  ctx->smear.valid = false;
  if (!nccl_id) return LMB_OK;  // back to one lattice per context
  if (!dims || !coords || !nb_minus || !nb_plus) return fail(ctx, LMB_ERR_ARG, "null process-grid argument");
  if (nranks < 1 || rank < 0 || rank >= nranks) return fail(ctx, LMB_ERR_ARG, "bad rank %d of %d", rank, nranks);
  if (split_mask > 15u) return fail(ctx, LMB_ERR_ARG, "split mask %u names a dimension beyond 4", split_mask);
  int prod = 1;
  for (int mu = 0; mu < 4; mu++) {
    if (dims[mu] < 1 || coords[mu] < 0 || coords[mu] >= dims[mu])
      return fail(ctx, LMB_ERR_ARG, "bad grid coordinate %d of %d in dimension %d", coords[mu], dims[mu], mu + 1);
    if (dims[mu] > 1 && !((split_mask >> mu) & 1))
      return fail(ctx, LMB_ERR_ARG, "dimension %d spans %d ranks and must be split", mu + 1, dims[mu]);
    if (nb_minus[mu] < 0 || nb_minus[mu] >= nranks || nb_plus[mu] < 0 || nb_plus[mu] >= nranks)
      return fail(ctx, LMB_ERR_ARG, "neighbour rank out of range in dimension %d", mu + 1);
    prod *= dims[mu];
  }
  if (prod != nranks) return fail(ctx, LMB_ERR_ARG, "process grid holds %d ranks, communicator %d", prod, nranks);
  const NcclApi &nc = nccl_api();
  if (!nc.loaded) return fail(ctx, LMB_ERR_UNSUPPORTED, "%s", nc.error.c_str());
  if (cudaSetDevice(ctx->device) != cudaSuccess) return fail(ctx, LMB_ERR_CUDA, "cudaSetDevice");
  lmb_dist *d = new lmb_dist();
  ctx->dist = d;
  d->nranks = nranks;
  d->rank = rank;
  d->split = split_mask;
  for (int mu = 0; mu < 4; mu++) {
    d->dims[mu] = dims[mu];
    d->coords[mu] = coords[mu];
    d->nb_minus[mu] = nb_minus[mu];
    d->nb_plus[mu] = nb_plus[mu];
  }
  ncclUniqueId u;
  std::memcpy(u.internal, nccl_id, NCCL_UNIQUE_ID_BYTES);
  ncclResult_t r = nc.CommInitRank(&d->comm, nranks, u, rank);
  if (r != ncclSuccess) {
    d->comm = nullptr;
    dist_release(ctx);
    return fail(ctx, LMB_ERR_CUDA, "ncclCommInitRank: %s", nc.GetErrorString(r));
  }
  int prio_low = 0, prio_high = 0;
  cudaDeviceGetStreamPriorityRange(&prio_low, &prio_high);
  if (cudaStreamCreateWithFlags(&d->comm_stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithPriority(&d->bnd_stream, cudaStreamNonBlocking, prio_high) != cudaSuccess ||
      cudaEventCreateWithFlags(&d->ev_packed, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&d->ev_comm, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&d->ev_bnd, cudaEventDisableTiming) != cudaSuccess ||
      cudaMalloc(&d->bcounter, sizeof(unsigned)) != cudaSuccess ||
      cudaMemset(d->bcounter, 0, sizeof(unsigned)) != cudaSuccess ||
      cudaMalloc(&d->sums, 2 * sizeof(double)) != cudaSuccess) {
    dist_release(ctx);
    return fail(ctx, LMB_ERR_CUDA, "process-grid resources");
  }
  return LMB_OK;
}

}  // extern "C"
