// lmb_context.cuh -- the lmb_ctx object behind the C ABI: geometry, link and
// clover caches, named workspaces and error reporting.
#pragma once
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>
#include <deque>
#include <map>
#include <string>
#include <vector>

#include "../../include/lmb200.h"
#include "lmb_pack.cuh"
#include "lmb_solver.cuh"

namespace lmb {

struct LinkSet {
  const void *ptr[4] = {nullptr, nullptr, nullptr, nullptr};
  uint64_t epoch[4] = {0, 0, 0, 0};
  bool valid = false;
  uint64_t version = 0;  // bumps on every repack
  double2 *d = nullptr;  // 36 planes
  float2 *f = nullptr;
  int *h = nullptr;
  float scale = 1.f;     // max |element| (for int16); +Inf for a non-finite entry
  uint64_t f_version = ~0ull, h_version = ~0ull;
  // SU(3) links store two rows (reconstruct-12); chosen per precision by the
  // measured deviation max(|U U^+ - 1|, |det U - 1|) at upload
  double su3_dev = 1.0;
  double2 *d12 = nullptr;
  float4 *f12 = nullptr;
  int4 *h12 = nullptr;
  uint64_t d12_version = ~0ull, f12_version = ~0ull, h12_version = ~0ull;
  bool recon(int prec) const { return prec == PREC_DOUBLE ? su3_dev <= 1e-14 : su3_dev <= 1e-6; }
  // every entry finite and within FP32 range (the low-precision copies hold it)
  bool finite() const { return scale <= 3.0e38f; }
};

struct CloverCache {
  uint64_t links_version = ~0ull;
  double coef = 0.0;
  bool F_valid = false;
  uint64_t F_links_version = ~0ull;
  double2 *F = nullptr;  // 54 planes
  double2 *d = nullptr;  // 36 planes
  float4 *f = nullptr;
  int4 *h = nullptr;
  int2 *ht = nullptr;
  float scale = 1.f;
  bool d_valid = false;
  uint64_t f_version = ~0ull, h_version = ~0ull, d_version = 0;
  uint64_t src_version = ~0ull;  // inverse blocks: d_version of the blocks inverted
};

}  // namespace lmb

struct lmb_smear_key {
  const void *ptr[4] = {nullptr, nullptr, nullptr, nullptr};
  uint64_t epoch[4] = {0, 0, 0, 0};
  double naik_epsilon = 0.0;
  bool valid = false;
};

struct lmb_batch_links {
  const void *ptr[4] = {nullptr, nullptr, nullptr, nullptr};
  uint64_t epoch[4] = {0, 0, 0, 0};
  int64_t V = 0;
  double2 *d12 = nullptr;  // FP64 reconstruct-12
  float4 *f12 = nullptr;   // FP32 reconstruct-12
  int4 *h12 = nullptr;     // int16 reconstruct-12
};

struct lmb_batch_tune {
  int nb = 0, nt = 0;
  // 0: links in registers, NB <= 4; 1: links in shared memory, NB up to 16;
  // 2: int16 x-adjacent pairs, tasks (tile, member) sharing links through L2
  int family = 0;
  double ms = 0;
};

struct lmb_dist;  // process grid, NCCL communicator, ghost buffers (lmb_dist_host.cuh)

struct lmb_ctx {
  int device = 0;
  lmb_dist *dist = nullptr;  // set by lmb_set_process_grid
  std::deque<lmb_batch_links> batch_links;  // deque: element addresses stay valid on growth
  std::map<std::string, lmb_batch_tune> batch_tune;
  lmb_smear_key smear;  // thin links the HISQ fat/long link sets were built from
  bool geom_set = false;
  lmb::Geom g{};
  lmb::Padded pd{};
  int dtype = LMB_DTYPE_C128;
  // FP32 / int16 Wilson stencils with two sites per thread (packed FP32);
  // LMB_PAIR_SITES=0 in the environment selects one site per thread
  bool pair_sites = true;
  // int16 Wilson stencils with reconstruct-12 links and an even x extent:
  // the two sites of a thread are x-neighbours, read with 256-bit loads
  // (environment LMB_ADJ_SITES=0: sites s and s + V/2)
  bool adj_sites = true;
  // int16 K1 / K2 stencils as persistent kernels (one block per resident
  // slot walking the tiles, one reduction per block); LMB_PERSISTENT=0 in
  // the environment: one block per tile
  bool persistent = true;
  // batched CG kernel family the autotuner may pick: -1 either, 0 links in
  // registers, 1 links in shared memory (environment LMB_BATCH_FAMILY)
  int batch_family = -1;
  int sm_count = 0;
  lmb::LinkSet links[3];
  // domain-wall operator (lmb_domainwall_set): L5 slices of the 4D geometry,
  // mass, M and the coefficients a, b, c (3 L5 doubles, device memory)
  int dw_L5 = 0;
  double dw_mass = 0.0, dw_M = 0.0;
  double *dw_coef = nullptr;
  int dw_coef_cap = 0;
  // LMB_DW_TWO_PASS=1 in the environment: domain-wall applications in two
  // passes (a local pass and a stencil pass) at every L5, instead of one
  bool dw_two_pass = false;
  lmb::CloverCache clover;
  lmb::CloverCache clover_inv;  // A^-1 blocks (even/odd solve)
  int64_t cache_V = 0;          // volume the link sets and clover caches are sized for
  // parity-ordered copies of link / clover storage for the even/odd solve:
  // workspace name -> (source version, volume, buffer) they were built for
  struct EoTag {
    uint64_t version;
    int64_t V;
    void *ptr;
  };
  std::map<std::string, EoTag> eo_tags;
  std::map<std::string, std::pair<void *, size_t>> buffers;
  double *partials = nullptr;
  size_t partials_cap = 0;
  unsigned *counter = nullptr;
  lmb::CGState *st_dev = nullptr;
  lmb::CGState *st_host = nullptr;  // pinned
  double *dot_host = nullptr;       // pinned
  std::string err;
};

namespace lmb {

inline int fail(lmb_ctx *ctx, int code, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  if (ctx) ctx->err = buf;
  return code;
}

#define LMB_CUDA(ctx, call)                                                              \
  do {                                                                                   \
    cudaError_t e_ = (call);                                                             \
    if (e_ != cudaSuccess)                                                               \
      return ::lmb::fail(ctx, LMB_ERR_CUDA, "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), \
                         __FILE__, __LINE__);                                            \
  } while (0)

#define LMB_CHECK_LAUNCH(ctx)                                                             \
  do {                                                                                    \
    cudaError_t e_ = cudaGetLastError();                                                  \
    if (e_ != cudaSuccess)                                                                \
      return ::lmb::fail(ctx, LMB_ERR_CUDA, "kernel launch: %s (%s:%d)", cudaGetErrorString(e_), \
                         __FILE__, __LINE__);                                             \
  } while (0)

// named workspace, grown on demand (never shrinks until lmb_destroy)
inline void *workspace(lmb_ctx *ctx, const std::string &name, size_t bytes) {
  auto it = ctx->buffers.find(name);
  if (it != ctx->buffers.end() && it->second.second >= bytes) return it->second.first;
  if (it != ctx->buffers.end()) {
    cudaFree(it->second.first);
    ctx->buffers.erase(it);
  }
  void *p = nullptr;
  if (cudaMalloc(&p, bytes) != cudaSuccess) return nullptr;
  ctx->buffers[name] = {p, bytes};
  return p;
}

inline bool ensure_partials(lmb_ctx *ctx, size_t blocks, int nval) {
  const size_t need = blocks * (size_t)nval;
  if (ctx->partials_cap >= need) return true;
  if (ctx->partials) cudaFree(ctx->partials);
  ctx->partials = nullptr;
  ctx->partials_cap = 0;
  if (cudaMalloc(&ctx->partials, need * sizeof(double)) != cudaSuccess) return false;
  ctx->partials_cap = need;
  return true;
}

// a field of V sites (default: the context's 4D volume)
template <int P, int NC>
inline bool make_field(lmb_ctx *ctx, const std::string &name, Field<P, NC> &f, int64_t V = -1) {
  if (V < 0) V = ctx->g.V;
  f.V = V;
  const size_t nb = Field<P, NC>::bytes(V), mb = Field<P, NC>::norm_bytes(V);
  void *p = workspace(ctx, name, nb + mb + 256);
  if (!p) return false;
  f.data = (decltype(f.data))p;
  f.norm = mb ? (float *)((char *)p + ((nb + 255) / 256) * 256) : nullptr;
  return true;
}

inline unsigned grid_for(int64_t n, int threads) { return (unsigned)((n + threads - 1) / threads); }

}  // namespace lmb
