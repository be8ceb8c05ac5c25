// lmb_halo.cuh -- fill the halo of a padded single-rank field
// (set_halo! / exchange_dim_local!, LatticeMatrices_core.jl:550-567, 707-723).
//
// The reference fills the ghosts one dimension after another: in dimension d
// the minus ghost slab takes the plus face times 1/phase_d and the plus ghost
// slab the minus face times phase_d, each slab spanning the full padded
// extent of the other dimensions, so corners pick up the phases of every
// dimension they wrap in.  The result has a closed form that one kernel
// writes directly: a padded coordinate i (0-based, 0 <= i < L + 2 nw) in
// dimension d reads core coordinate c = (i - nw) mod L with wrap count
// w = floor((i - nw) / L) in {-1, 0, 1} (nw <= L), and the value is the
// core value times prod_d phase_d^w_d.
#pragma once
#include "lmb_common.cuh"

namespace lmb {

struct HaloGeom {
  int D;           // 4 or 5
  int L[5];        // core extents
  int P[5];        // padded extents L + 2 nw
  int nw;
  double ph[5][2];   // phase_d
  double iph[5][2];  // 1 / phase_d
  int64_t npad;      // prod P
};

template <typename T>
__global__ void __launch_bounds__(256) set_halo_kernel(T *A, const int ncomp, const HaloGeom h) {
  const int64_t p = (int64_t)blockIdx.x * 256 + threadIdx.x;
  if (p >= h.npad) return;
  int64_t rest = p, src = 0, stride = 1;
  bool halo = false;
  double fr = 1.0, fi = 0.0;
  for (int d = 0; d < h.D; d++) {
    const int i = (int)(rest % h.P[d]);
    rest /= h.P[d];
    int c = i - h.nw, w = 0;
    if (c < 0) {
      c += h.L[d];
      w = -1;
    } else if (c >= h.L[d]) {
      c -= h.L[d];
      w = 1;
    }
    if (w) {
      halo = true;
      const double *q = w > 0 ? h.ph[d] : h.iph[d];
      const double nr = fr * q[0] - fi * q[1], ni = fr * q[1] + fi * q[0];
      fr = nr;
      fi = ni;
    }
    src += (int64_t)(c + h.nw) * stride;
    stride *= h.P[d];
  }
  if (!halo) return;
  const T *s = A + src * ncomp;
  T *o = A + p * ncomp;
  for (int k = 0; k < ncomp; k++) {
    const T v = s[k];
    o[k].x = v.x * fr - v.y * fi;
    o[k].y = v.x * fi + v.y * fr;
  }
}

}  // namespace lmb
