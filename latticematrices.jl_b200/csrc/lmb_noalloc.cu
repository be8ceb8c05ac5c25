// lmb_noalloc.cu -- lmb_field_dot_noalloc: the field inner product with no
// device allocation at all.
//
// Who needs it: callers that must not call cudaMalloc -- callers whose
// device memory is owned by a pool allocator (CUDA.jl, PyTorch) running close
// to the device limit, where a stray cudaMalloc can fail or force the pool to
// release cached blocks; host plugins whose embedding application forbids
// allocations outside its own allocator; and latency-sensitive loops, where
// cudaMalloc may synchronise the device.  Such
// a caller cannot create an lmb_ctx either (its workspaces are allocated),
// so this entry point takes the geometry directly and needs no context.
//
// Scratch: the per-block partial sums and the last-block counter live in
// one file-scope `static __device__` array of kScratchBytes (1 MiB + 256 B),
// held on every GPU where this file's module is loaded until the process
// exits.  It holds one partial pair per 256-site block, so one call handles
// at most kMaxSites = 16,777,216 lattice sites (48^3 x 96 = 10.6M fits);
// larger volumes are rejected with LMB_ERR_ARG.  The array keeps the previous
// call's contents; the counter is cleared on the caller's stream before every
// launch, and every partial the kernel reads was written by the same launch.
// All calls on a device share this one array: calls whose kernels overlap on
// the GPU (different streams, no ordering between them) race and may return
// wrong sums; calls on one stream, or otherwise ordered, are safe.
//
// Module loading: with CUDA's lazy loading (the default), this file's module
// -- its kernels and the array -- is placed on a device only when the first
// call on that device looks up the array's address.  That load takes device
// memory, so make one call per device at initialisation, before a pool
// allocator has taken the free memory and outside any stream capture.
// Later calls look the address up again (a host-side table lookup that
// allocates nothing), so a device reset or a recreated primary context,
// after which the module is loaded afresh and the array may move, never
// leaves a stale address behind.
#include "../../include/lmb200.h"
#include "lmb_common.cuh"

namespace {

constexpr int kDotThreads = 256;
constexpr int64_t kMaxSites = 16777216;                      // 2^24
constexpr int64_t kMaxBlocks = kMaxSites / kDotThreads;      // 65536
constexpr size_t kCounterBytes = 256;                        // counter slot
constexpr size_t kScratchBytes = kCounterBytes + sizeof(double) * 2 * kMaxBlocks;

static __device__ __align__(256) unsigned char g_dot_scratch[kScratchBytes];

// halo-padded site offset (column-major (.., X+2nw, Y+2nw, Z+2nw, T+2nw))
struct PaddedGeom {
  int P[4];
  int nw;
};
__device__ __forceinline__ int64_t padded_offset(const PaddedGeom &pd, const int c[4]) {
  return (c[0] + pd.nw) +
         (int64_t)pd.P[0] * ((c[1] + pd.nw) + (int64_t)pd.P[1] * ((c[2] + pd.nw) + (int64_t)pd.P[2] * (c[3] + pd.nw)));
}

// Device address of g_dot_scratch on the current device.  In host code
// `g_dot_scratch` names a host-side shadow, not device memory, so the kernel
// is always given the looked-up address.
int scratch_for_current_device(void **out) {
  void *p = nullptr;
  if (cudaGetSymbolAddress(&p, g_dot_scratch) != cudaSuccess || !p) return LMB_ERR_CUDA;
  *out = p;
  return LMB_OK;
}

template <int NC, typename T>
__global__ void __launch_bounds__(kDotThreads)
    dot_noalloc_kernel(const T *a, const T *b, lmb::Geom g, PaddedGeom pd, unsigned char *scratch,
                       double *out) {
  unsigned *counter = (unsigned *)scratch;
  double *partials = (double *)(scratch + kCounterBytes);
  const int s = blockIdx.x * kDotThreads + threadIdx.x;
  double v[2] = {0.0, 0.0}, tot[2];
  if (s < g.V) {
    int c[4];
    lmb::site_coords(g, s, c);
    const int64_t off = padded_offset(pd, c) * NC;
    for (int k = 0; k < NC; k++) {
      const T x = a[off + k], y = b[off + k];
      v[0] += (double)x.x * (double)y.x + (double)x.y * (double)y.y;
      v[1] += (double)x.x * (double)y.y - (double)x.y * (double)y.x;
    }
  }
  if (lmb::grid_reduce<kDotThreads, 2>(v, partials, counter, tot) && threadIdx.x == 0) {
    out[0] = tot[0];
    out[1] = tot[1];
  }
}

template <typename T>
cudaError_t launch(int ncomp, const void *a, const void *b, const lmb::Geom &g, const PaddedGeom &pd,
                   unsigned char *scratch, double *out, cudaStream_t st, unsigned grid) {
  switch (ncomp) {
    case 1: dot_noalloc_kernel<1, T><<<grid, kDotThreads, 0, st>>>((const T *)a, (const T *)b, g, pd, scratch, out); break;
    case 3: dot_noalloc_kernel<3, T><<<grid, kDotThreads, 0, st>>>((const T *)a, (const T *)b, g, pd, scratch, out); break;
    case 9: dot_noalloc_kernel<9, T><<<grid, kDotThreads, 0, st>>>((const T *)a, (const T *)b, g, pd, scratch, out); break;
    case 12: dot_noalloc_kernel<12, T><<<grid, kDotThreads, 0, st>>>((const T *)a, (const T *)b, g, pd, scratch, out); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

}  // namespace

extern "C" int lmb_field_dot_noalloc(const void *a, const void *b, const int L[4], int nw, int dtype, int ncomp,
                                     double *out_device, void *stream) {
  if (!a || !b || !L || !out_device) return LMB_ERR_ARG;
  if (nw < 0 || (dtype != LMB_DTYPE_C128 && dtype != LMB_DTYPE_C64)) return LMB_ERR_ARG;
  if (ncomp != 1 && ncomp != 3 && ncomp != 9 && ncomp != 12) return LMB_ERR_UNSUPPORTED;
  lmb::Geom g{};
  PaddedGeom pd{};
  int64_t V = 1;
  for (int mu = 0; mu < 4; mu++) {
    if (L[mu] <= 0 || nw > L[mu]) return LMB_ERR_ARG;
    g.L[mu] = L[mu];
    g.stride[mu] = (int)V;
    V *= L[mu];
    if (V > kMaxSites) return LMB_ERR_ARG;  // beyond the static scratch
    pd.P[mu] = L[mu] + 2 * nw;
  }
  g.V = V;
  pd.nw = nw;
  void *scratch = nullptr;
  int rc = scratch_for_current_device(&scratch);
  if (rc != LMB_OK) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  // the last-block counter must start at zero
  if (cudaMemsetAsync(scratch, 0, kCounterBytes, st) != cudaSuccess) return LMB_ERR_CUDA;
  const unsigned grid = (unsigned)((V + kDotThreads - 1) / kDotThreads);
  cudaError_t e = dtype == LMB_DTYPE_C128
                      ? launch<double2>(ncomp, a, b, g, pd, (unsigned char *)scratch, out_device, st, grid)
                      : launch<float2>(ncomp, a, b, g, pd, (unsigned char *)scratch, out_device, st, grid);
  return e == cudaSuccess ? LMB_OK : LMB_ERR_CUDA;
}
