// lmb_dist.cuh -- device side of the sharded (process-grid) operators.
//
// A rank holds the block of its Cartesian coordinates (the reference's
// LatticeMatrix PN block, LatticeMatrices_core.jl:350-358).  Along every
// exchanged ("split") dimension mu a stencil application
//   1. packs the rank's two faces of `depth` layers (1 for Wilson, 3 for the
//      HISQ Naik term) into send buffers -- the minus face multiplied by the
//      boundary phase when the rank holds global coordinate 0, the plus face by
//      1/phase when it holds the last one, the rule of exchange_dim!
//      (LatticeMatrices_core.jl:742-921) --
//   2. sends them to the two neighbours and receives their faces into ghost
//      buffers (NCCL, on a communication stream), while
//   3. an interior kernel computes every site whose neighbours are all local,
//   4. then a boundary kernel computes the remaining sites, reading the ghost
//      layers for hops that leave the block (no phase: the sender applied it).
// Dimensions that are not split wrap in-kernel with the phase, as on one GPU.
//
// Ghost layout: a ghost (or face) buffer of dimension mu is a Field of
// depth * F_mu sites in the storage format of the stencil's field (planes,
// int16 norms), F_mu = V / L_mu; element (layer j, face index f) sits at
// j * F_mu + f, f lexicographic (x fastest) over the three other dimensions.
// Minus ghost layer j holds x_mu = -1 - j, plus ghost layer j holds
// x_mu = L_mu + j.  Link ghosts hold U_mu (direction mu only) at
// x_mu = -1 - j, read from the halo the caller filled in the padded links.
#pragma once
#include "lmb_pack.cuh"
#include "lmb_solver.cuh"
#include "lmb_staggered.cuh"
#include "lmb_wilson.cuh"

namespace lmb {

struct DistView {
  unsigned split;   // bit mu: dimension mu exchanged with neighbours
  int depth;        // ghost layers
  int face[4];      // F_mu
  int fstr[4][4];   // stride of dimension nu in the face index of dimension mu (0 for nu == mu)
  // the box of x-adjacent pairs with both sites interior: pair index px (x =
  // 2 px) in [plo[0], plo[0] + pn[0]), coordinate mu >= 1 in [plo, plo + pn)
  int plo[4], pn[4];
  int npairs;
  // the box of interior sites: coordinate mu in [slo, slo + sn)
  int slo[4], sn[4];
  int nsites;
};

LMB_D int face_index(const DistView &dv, const int *c, int mu) {
  return dv.fstr[mu][0] * c[0] + dv.fstr[mu][1] * c[1] + dv.fstr[mu][2] * c[2] + dv.fstr[mu][3] * c[3];
}

template <int P, int NC>
struct GhostSpinors {
  Field<P, NC> m[4], p[4];
};
template <class G>
struct GhostLinks {
  G m[4];
};

// a site is interior when every hop of reach `depth` stays in the block
LMB_D bool dist_interior(const Geom &g, const DistView &dv, const int *c) {
#pragma unroll
  for (int mu = 0; mu < 4; mu++)
    if (((dv.split >> mu) & 1) && (c[mu] < dv.depth || c[mu] >= g.L[mu] - dv.depth)) return false;
  return true;
}

// the i-th site of the interior box (i < nsites) and its coordinates c
LMB_D int interior_site(const Geom &g, const DistView &dv, int i, int *c) {
  c[0] = dv.slo[0] + i % dv.sn[0];
  int q = i / dv.sn[0];
  c[1] = dv.slo[1] + q % dv.sn[1];
  q /= dv.sn[1];
  c[2] = dv.slo[2] + q % dv.sn[2];
  c[3] = dv.slo[3] + q / dv.sn[2];
  return c[0] + g.stride[1] * c[1] + g.stride[2] * c[2] + g.stride[3] * c[3];
}

// the interior of a block split along t only as one range of sites,
// t in [depth, L_t - depth); empty for any other split
inline SiteRange t_slab(const Geom &g, const DistView &dv) {
  if (dv.split != 8u || g.L[3] <= 2 * dv.depth) return SiteRange{0, 0};
  return SiteRange{dv.depth * g.stride[3], (int)g.V - dv.depth * g.stride[3]};
}

// spinor at distance d (|d| <= depth) along MU from site s: a split
// dimension reads a ghost layer past the block (*wrap = 0), any other
// dimension wraps periodically (*wrap = signed number of edge crossings)
template <int P, int NC, typename R>
LMB_D void load_nb(const Field<P, NC> &in, const GhostSpinors<P, NC> &gh, const Geom &g, const DistView &dv,
                   int s, const int *c, int MU, int d, Cx<R> *v, int *wrap) {
  const int L = g.L[MU];
  int x = c[MU] + d;
  if ((dv.split >> MU) & 1) {
    *wrap = 0;
    if (x >= 0 && x < L) {
      in.load(s + d * g.stride[MU], v);
    } else {
      const int f = face_index(dv, c, MU);
      if (x >= L) gh.p[MU].load((int64_t)(x - L) * dv.face[MU] + f, v);
      else gh.m[MU].load((int64_t)(-1 - x) * dv.face[MU] + f, v);
    }
    return;
  }
  int w = 0;
  while (x >= L) {
    x -= L;
    w++;
  }
  while (x < 0) {
    x += L;
    w--;
  }
  *wrap = w;
  in.load(s + (x - c[MU]) * g.stride[MU], v);
}

// link U_MU at site x + d MU, d <= 0 (backward hops)
template <class G, typename R>
LMB_D void load_link_nb(const G &U, const GhostLinks<G> &gu, const Geom &g, const DistView &dv, int s,
                        const int *c, int MU, int d, Cx<R> *u) {
  const int L = g.L[MU];
  int x = c[MU] + d;
  if (((dv.split >> MU) & 1) && x < 0) {
    gu.m[MU].load(MU, (int64_t)(-1 - x) * dv.face[MU] + face_index(dv, c, MU), u);
    return;
  }
  while (x < 0) x += L;
  U.load(MU, s + (x - c[MU]) * g.stride[MU], u);
}

// ---------------------------------------------------------------------------
// face packing, every split dimension in one launch (blockIdx.y = the n-th
// split dimension mu[n]): minus face (x_mu = j) -> send_m, plus face
// (x_mu = L-1-j) -> send_p, each multiplied by its phase factor (1 unless
// the rank holds the global edge)
// ---------------------------------------------------------------------------
template <int P, int NC>
struct FacePack {
  Field<P, NC> send_m[4], send_p[4];
  double2 ph_m[4], ph_p[4];
  int mu[4];
};

template <int P, int NC>
__global__ void __launch_bounds__(256)
    pack_faces_kernel(const Field<P, NC> in, const FacePack<P, NC> fp, const Geom g, const DistView dv) {
  typedef typename Real<P>::type R;
  const int n = blockIdx.y;
  const int mu = fp.mu[n];
  const int64_t F = dv.face[mu];
  const int64_t t = (int64_t)blockIdx.x * 256 + threadIdx.x;
  if (t >= dv.depth * F) return;
  const int layer = (int)(t / F);
  int f = (int)(t - layer * F);
  int c[4];
#pragma unroll
  for (int nu = 0; nu < 4; nu++) {
    if (nu == mu) continue;
    c[nu] = f % g.L[nu];
    f /= g.L[nu];
  }
  Cx<R> v[NC];
  c[mu] = layer;
  int s = c[0] + g.stride[1] * c[1] + g.stride[2] * c[2] + g.stride[3] * c[3];
  in.load(s, v);
  const double2 pm = fp.ph_m[n], pp = fp.ph_p[n];
  if (pm.x != 1.0 || pm.y != 0.0) {
    const Cx<R> ph((R)pm.x, (R)pm.y);
#pragma unroll
    for (int k = 0; k < NC; k++) v[k] = v[k] * ph;
  }
  fp.send_m[n].store(t, v);
  c[mu] = g.L[mu] - 1 - layer;
  s = c[0] + g.stride[1] * c[1] + g.stride[2] * c[2] + g.stride[3] * c[3];
  in.load(s, v);
  if (pp.x != 1.0 || pp.y != 0.0) {
    const Cx<R> ph((R)pp.x, (R)pp.y);
#pragma unroll
    for (int k = 0; k < NC; k++) v[k] = v[k] * ph;
  }
  fp.send_p[n].store(t, v);
}

// link ghost of dimension mu from the caller's padded links (halo filled):
// U_mu at x_mu = -1 - j into direction mu's 9 planes of a 36-plane buffer
template <typename T>
__global__ void __launch_bounds__(256)
    pack_link_ghost_kernel(double2 *dst, const T *Umu, const Geom g, const Padded pd, const DistView dv, int mu) {
  const int64_t F = dv.face[mu], Vg = dv.depth * F;
  const int64_t t = (int64_t)blockIdx.x * 256 + threadIdx.x;
  if (t >= Vg) return;
  const int layer = (int)(t / F);
  int f = (int)(t - layer * F);
  int c[4];
#pragma unroll
  for (int nu = 0; nu < 4; nu++) {
    if (nu == mu) continue;
    c[nu] = f % g.L[nu];
    f /= g.L[nu];
  }
  c[mu] = -1 - layer;
  const int64_t ps = padded_site(pd, c) * 9;
#pragma unroll
  for (int k = 0; k < 9; k++) {
    const T v = Umu[ps + k];
    dst[(mu * 9 + k) * Vg + t] = make_double2((double)v.x, (double)v.y);
  }
}

// ---------------------------------------------------------------------------
// Wilson / Wilson-clover, one site per thread
// ---------------------------------------------------------------------------
template <typename R, int DAG, int MU, int P, class G>
LMB_D void hop_dir_dist(const Geom &g, const DistView &dv, int s, const int *c, const Field<P, 12> &in,
                        const GhostSpinors<P, 12> &gh, const G &U, const GhostLinks<G> &gu, Cx<R> *acc) {
  constexpr int FPM = DAG ? +1 : -1;
  constexpr int BPM = -FPM;
  Cx<R> p[12], h[6], uh[6], u[9];
  int w;
  load_nb(in, gh, g, dv, s, c, MU, 1, p, &w);
  project<FPM, MU>(p, h);
  if (w && ((g.phase_mask >> MU) & 1)) scale_phase(h, 6, g.ph_fwd[MU]);
  U.load(MU, s, u);
  su3_mul_half(u, h, uh);
  reconstruct<FPM, MU>(acc, uh);
  load_nb(in, gh, g, dv, s, c, MU, -1, p, &w);
  project<BPM, MU>(p, h);
  if (w && ((g.phase_mask >> MU) & 1)) scale_phase(h, 6, g.ph_bwd[MU]);
  load_link_nb(U, gu, g, dv, s, c, MU, -1, u);
  su3_adj_mul_half(u, h, uh);
  reconstruct<BPM, MU>(acc, uh);
}

// interior sites (every neighbour local) with the single-lattice hops
template <typename R, int DAG, bool CLOVER, int PHM, int P, class G, class CL, class Epi>
__global__ void __launch_bounds__(kDslashThreads)
    wilson_interior_kernel(const Geom g, const DistView dv, const Field<P, 12> in, const G U, const CL A,
                           const R kappa, Epi epi) {
  if (epi.skip()) return;
  const int i = blockIdx.x * kDslashThreads + threadIdx.x;
  const bool active = i < dv.nsites;
  Cx<R> out[12];
  int c[4];
  const int s = active ? interior_site(g, dv, i, c) : 0;
  if (active) wilson_site_out<R, DAG, CLOVER, PHM>(g, s, c, in, U, A, kappa, out);
  epi(s, active, out);
}

// The interior of a block split in any dimension on the int16 x-adjacent
// pair stencil (x extent even): one thread per pair (s0 = 2i, s0 + 1), the
// pairs with both sites interior; the sites of the other pairs are in the
// boundary list built with their x partners (dist_boundary, pairs).  An
// interior site's hops stay inside the block or wrap in place along an
// unsplit dimension, as on a single lattice.
// site s0 (x even) of the i-th pair of the interior pair box (i < npairs):
// the interior kernels run one thread per interior pair, no thread idle
LMB_D int interior_pair_site(const Geom &g, const DistView &dv, int i) {
  const int px = dv.plo[0] + i % dv.pn[0];
  int q = i / dv.pn[0];
  const int y = dv.plo[1] + q % dv.pn[1];
  q /= dv.pn[1];
  const int z = dv.plo[2] + q % dv.pn[2];
  const int t = dv.plo[3] + q / dv.pn[2];
  return 2 * px + g.stride[1] * y + g.stride[2] * z + g.stride[3] * t;
}

template <int DAG, bool CLOVER, int PHM, class CL, class Epi>
__global__ void __launch_bounds__(kDslashThreads, LMB_PAIR_MINB)
    wilson_half_adj_interior_kernel(const Geom g, const DistView dv, const Field<PREC_HALF, 12> in,
                                    const Gauge12<PREC_HALF> U, const CL A, const float kappa, Epi epi) {
  if (epi.skip()) return;
  const int i = blockIdx.x * kDslashThreads + threadIdx.x;
  const bool active = i < dv.npairs;
  const int s0 = active ? interior_pair_site(g, dv, i) : 0;
  Cx2 out[12];
  if (active) half_adj_sites<DAG, CLOVER, PHM>(g, s0, in, U, A, kappa, out);
  epi.pair_adj(s0, active, out);
}

// The same for the staggered / HISQ stencils (PH_T mode, every extent of the
// block >= 3, 18-real links): FP32 / int16 storage on packed FP32, and FP64
// through the epilogue's site_acc / finish
template <bool NAIK, int PS, class Epi>
__global__ void __launch_bounds__(kStagThreads, LMB_PAIR_MINB)
    staggered_adj_interior_kernel(const Geom g, const DistView dv, const Field<PS, 3> in, const Gauge<PS> X,
                                  const Gauge<PS> Lk, const float mass, const float fc, const float lc, Epi epi) {
  if (epi.skip()) return;
  const int i = blockIdx.x * kStagThreads + threadIdx.x;
  const bool active = i < dv.npairs;
  const int s0 = active ? interior_pair_site(g, dv, i) : 0;
  Cx2 out[3];
  if (active) stag_adj_sites<NAIK, PS>(g, s0, in, X, Lk, mass, fc, lc, out);
  epi.pair_adj(s0, active, out);
}
template <bool NAIK, class Epi>
__global__ void __launch_bounds__(kStagThreads, StagD2MinBlocks<Epi>::value)
    staggered_adj_d_interior_kernel(const Geom g, const DistView dv, const Field<PREC_DOUBLE, 3> in,
                                    const Gauge<PREC_DOUBLE> X, const Gauge<PREC_DOUBLE> Lk, const double mass,
                                    const double fc, const double lc, Epi epi) {
  if (epi.skip()) return;
  double red[1] = {0.0};
  const int i = blockIdx.x * kStagThreads + threadIdx.x;
  const bool active = i < dv.npairs;
  const int s0 = active ? interior_pair_site(g, dv, i) : 0;
  Cd2 out[3];
  if (active) stag_adj_sites_d<NAIK>(g, s0, in, X, Lk, mass, fc, lc, out);
  Cx<double> o0[3], o1[3];
#pragma unroll
  for (int k = 0; k < 3; k++) {
    o0[k] = Cx<double>(out[k].re.x, out[k].im.x);
    o1[k] = Cx<double>(out[k].re.y, out[k].im.y);
  }
  epi.site_acc(s0, active, o0, red);
  epi.site_acc(s0 + 1, active, o1, red);
  epi.finish(red);
}

// the sites of `list` (the block's boundary), ghost-aware
template <typename R, int DAG, bool CLOVER, int P, class G, class CL, class Epi>
__global__ void __launch_bounds__(kDslashThreads)
    wilson_boundary_kernel(const Geom g, const DistView dv, const Field<P, 12> in, const GhostSpinors<P, 12> gh,
                           const G U, const GhostLinks<G> gu, const CL A, const R kappa, Epi epi, const int *list,
                           int n) {
  if (epi.skip()) return;
  const int i = blockIdx.x * kDslashThreads + threadIdx.x;
  const bool active = i < n;
  const int s = active ? list[i] : 0;
  Cx<R> out[12];
  if (active) {
    int c[4];
    site_coords(g, s, c);
    Cx<R> acc[12];
#pragma unroll
    for (int k = 0; k < 12; k++) acc[k] = Cx<R>(0, 0);
    hop_dir_dist<R, DAG, 0>(g, dv, s, c, in, gh, U, gu, acc);
    hop_dir_dist<R, DAG, 1>(g, dv, s, c, in, gh, U, gu, acc);
    hop_dir_dist<R, DAG, 2>(g, dv, s, c, in, gh, U, gu, acc);
    hop_dir_dist<R, DAG, 3>(g, dv, s, c, in, gh, U, gu, acc);
    wilson_site_finish<R, CLOVER>(s, in, A, kappa, acc, out);
  }
  epi(s, active, out);
}

// ---------------------------------------------------------------------------
// int16 boundary slabs of a block split along t only: the two x-adjacent
// sites of a thread lie in slab t = 0 (TB = 1: the backward t hop reads the
// minus ghost layer and the ghost link) or t = L_t - 1 (TB = 2: the forward
// t hop reads the plus ghost layer); the site's index within its slab is its
// face index.  The other seven hops are the single-lattice ones.
// ---------------------------------------------------------------------------
template <int DAG, int PHM, int TB>
LMB_D void hop_t_ghost(const Geom &g, int s0, const int *c0, const Field<PREC_HALF, 12> &in,
                       const Field<PREC_HALF, 12> &ghost, const Gauge12<PREC_HALF> &U,
                       const Gauge12<PREC_HALF> &Ughost, Cx2 *acc) {
  constexpr int FPM = DAG ? +1 : -1;
  constexpr int BPM = -FPM;
  const int f = s0 - c0[3] * g.stride[3];  // index within the slab = face index
  Cx2 p[12], h[6], uh[6], u[9];
  float2 nc2;
  {  // forward: t + 1
    if constexpr (TB == 2) load_adj_raw(ghost, f, p, nc2);  // the sender applied any phase
    else load_adj_raw(in, s0 + g.stride[3], p, nc2);
    project_raw<FPM, 3>(p, nc2, h);
    load_adj(U, 3, s0, u);
    su3_mul_half(u, h, uh);
    reconstruct<FPM, 3>(acc, uh);
  }
  {  // backward: t - 1
    if constexpr (TB == 1) {
      load_adj_raw(ghost, f, p, nc2);
      project_raw<BPM, 3>(p, nc2, h);
      load_adj(Ughost, 3, f, u);
    } else {
      load_adj_raw(in, s0 - g.stride[3], p, nc2);
      project_raw<BPM, 3>(p, nc2, h);
      load_adj(U, 3, s0 - g.stride[3], u);
    }
    su3_adj_mul_half(u, h, uh);
    reconstruct<BPM, 3>(acc, uh);
  }
  (void)PHM;
}

template <int DAG, bool CLOVER, int PHM, int TB, class CL>
LMB_D void half_tslab_sites(const Geom &g, int s0, const Field<PREC_HALF, 12> &in,
                            const Field<PREC_HALF, 12> &ghost, const Gauge12<PREC_HALF> &U,
                            const Gauge12<PREC_HALF> &Ughost, const CL &A, float kappa, Cx2 *out) {
  int c0[4], c1[4];
  site_coords(g, s0, c0);
  c1[0] = c0[0] + 1;
  c1[1] = c0[1];
  c1[2] = c0[2];
  c1[3] = c0[3];
#pragma unroll
  for (int k = 0; k < 12; k++) out[k] = cx2_zero();
  hop_adj<DAG, 0, PHM>(g, s0, c0, c1, in, U, out);
  hop_adj<DAG, 1, PHM>(g, s0, c0, c1, in, U, out);
  hop_adj<DAG, 2, PHM>(g, s0, c0, c1, in, U, out);
  hop_t_ghost<DAG, PHM, TB>(g, s0, c0, in, ghost, U, Ughost, out);
  Cx2 p[12];
  load_adj(in, s0, p);
  const float2 nk2 = f2(-kappa);
  if constexpr (CLOVER) {
#pragma unroll
    for (int k = 0; k < 12; k++) out[k] = Cx2(nk2 * out[k].re, nk2 * out[k].im);
    float2 a[36];
#pragma unroll
    for (int blk = 0; blk < 2; blk++) {
      load_adj(A, blk, s0, a);
      herm6_mul_acc(a, p + 6 * blk, out + 6 * blk);
    }
  } else {
#pragma unroll
    for (int k = 0; k < 12; k++) out[k] = Cx2(fma2(nk2, out[k].re, p[k].re), fma2(nk2, out[k].im, p[k].im));
  }
}

// Two int16 sites held in two fields or link sets (lane 0: the first at i0,
// lane 1: the second at i1), for the face pairs whose one site reads a ghost
LMB_D void load2_raw_ff(const Field<PREC_HALF, 12> &f0, int64_t i0, const Field<PREC_HALF, 12> &f1, int64_t i1,
                        Cx2 *v, float2 &nc2) {
  const float b0 = __ldg(f0.norm + i0), b1 = __ldg(f1.norm + i1);
  const unsigned y0 = __float_as_uint(b0) >> 16, y1 = __float_as_uint(b1) >> 16;
  nc2 = make_float2(-b0 * 2.0078125f, -b1 * 2.0078125f);
#pragma unroll
  for (int k = 0; k < 3; k++) {
    const int4 t0 = __ldg(f0.data + k * f0.V + i0), t1 = __ldg(f1.data + k * f1.V + i1);
    const int w0[4] = {t0.x, t0.y, t0.z, t0.w}, w1[4] = {t1.x, t1.y, t1.z, t1.w};
#pragma unroll
    for (int j = 0; j < 4; j++) v[4 * k + j] = raw_pair2(w0[j], w1[j], y0, y1);
  }
}
LMB_D void load2_gg(const Gauge12<PREC_HALF> &U0, int64_t i0, const Gauge12<PREC_HALF> &U1, int64_t i1, int mu,
                    Cx2 *u) {
  const int q0 = mu * 6, p0 = q0 >> 2, lane0 = q0 & 3;
  const int4 a0 = __ldg(U0.data + p0 * U0.V + i0), b0 = __ldg(U0.data + (p0 + 1) * U0.V + i0);
  const int4 a1 = __ldg(U1.data + p0 * U1.V + i1), b1 = __ldg(U1.data + (p0 + 1) * U1.V + i1);
  const int w0[8] = {a0.x, a0.y, a0.z, a0.w, b0.x, b0.y, b0.z, b0.w};
  const int w1[8] = {a1.x, a1.y, a1.z, a1.w, b1.x, b1.y, b1.z, b1.w};
  const float2 negc = f2(-257.0f);  // base 2^8
#pragma unroll
  for (int e = 0; e < 6; e++)
    u[(e / 3) + 3 * (e % 3)] = dec_pair2(w0[lane0 + e], w1[lane0 + e], 0x4380u, 0x4380u, negc);
  su3_third_row(u);
}

// x hop of a face pair of a block split along x alone (depth 1): XB = 1 the
// pair (0, 1), whose site 0 reads its x - 1 neighbour from the minus ghost
// layer and that neighbour's link from the link ghost; XB = 2 the pair
// (L_x - 2, L_x - 1), whose site L_x - 1 reads x + 1 from the plus ghost
// layer.  f = the row's face index; the sender applied any boundary phase.
template <int DAG, int XB>
LMB_D void hop_x_ghost(int s0, int f, const Field<PREC_HALF, 12> &in, const Field<PREC_HALF, 12> &ghost,
                       const Gauge12<PREC_HALF> &U, const Gauge12<PREC_HALF> &Ughost, Cx2 *acc) {
  constexpr int FPM = DAG ? +1 : -1;
  constexpr int BPM = -FPM;
  Cx2 p[12], h[6], uh[6], u[9];
  float2 nc2;
  {  // forward: x + 1
    if constexpr (XB == 2) load2_raw_ff(in, s0 + 1, ghost, f, p, nc2);
    else load2_raw(in, s0 + 1, s0 + 2, p, nc2);
    project_raw<FPM, 0>(p, nc2, h);
    load_adj(U, 0, s0, u);
    su3_mul_half(u, h, uh);
    reconstruct<FPM, 0>(acc, uh);
  }
  {  // backward: x - 1
    if constexpr (XB == 1) {
      load2_raw_ff(ghost, f, in, s0, p, nc2);
      project_raw<BPM, 0>(p, nc2, h);
      load2_gg(Ughost, f, U, s0, 0, u);
    } else {
      load2_raw(in, s0 - 1, s0, p, nc2);
      project_raw<BPM, 0>(p, nc2, h);
      load2(U, 0, s0 - 1, s0, u);
    }
    su3_adj_mul_half(u, h, uh);
    reconstruct<BPM, 0>(acc, uh);
  }
}

template <int DAG, bool CLOVER, int PHM, int XB, class CL>
LMB_D void half_xface_sites(const Geom &g, int s0, int f, const Field<PREC_HALF, 12> &in,
                            const Field<PREC_HALF, 12> &ghost, const Gauge12<PREC_HALF> &U,
                            const Gauge12<PREC_HALF> &Ughost, const CL &A, float kappa, Cx2 *out) {
  int c0[4], c1[4];
  site_coords(g, s0, c0);
  c1[0] = c0[0] + 1;
  c1[1] = c0[1];
  c1[2] = c0[2];
  c1[3] = c0[3];
#pragma unroll
  for (int k = 0; k < 12; k++) out[k] = cx2_zero();
  hop_x_ghost<DAG, XB>(s0, f, in, ghost, U, Ughost, out);
  hop_adj<DAG, 1, PHM>(g, s0, c0, c1, in, U, out);
  hop_adj<DAG, 2, PHM>(g, s0, c0, c1, in, U, out);
  hop_adj<DAG, 3, PHM>(g, s0, c0, c1, in, U, out);
  Cx2 p[12];
  load_adj(in, s0, p);
  const float2 nk2 = f2(-kappa);
  if constexpr (CLOVER) {
#pragma unroll
    for (int k = 0; k < 12; k++) out[k] = Cx2(nk2 * out[k].re, nk2 * out[k].im);
    float2 a[36];
#pragma unroll
    for (int blk = 0; blk < 2; blk++) {
      load_adj(A, blk, s0, a);
      herm6_mul_acc(a, p + 6 * blk, out + 6 * blk);
    }
  } else {
#pragma unroll
    for (int k = 0; k < 12; k++) out[k] = Cx2(fma2(nk2, out[k].re, p[k].re), fma2(nk2, out[k].im, p[k].im));
  }
}

// one thread per face pair of a block split along x alone, x extent even and
// >= 4: threads [0, F) the pairs (0, 1) of the F = L_y L_z L_t rows (face
// index = row), [F, 2F) the pairs (L_x - 2, L_x - 1)
template <int DAG, bool CLOVER, int PHM, class CL, class Epi>
__global__ void __launch_bounds__(kDslashThreads, LMB_PAIR_MINB)
    wilson_half_xface_kernel(const Geom g, const Field<PREC_HALF, 12> in, const Field<PREC_HALF, 12> ghm,
                             const Field<PREC_HALF, 12> ghp, const Gauge12<PREC_HALF> U,
                             const Gauge12<PREC_HALF> Ughost, const CL A, const float kappa, Epi epi) {
  if (epi.skip()) return;
  const int Lx = g.L[0], F = (int)(g.V / Lx);
  const int i = blockIdx.x * kDslashThreads + threadIdx.x;
  const bool active = i < 2 * F;
  const bool top = i >= F;
  const int f = top ? i - F : i;
  const int s0 = f * Lx + (top ? Lx - 2 : 0);
  Cx2 out[12];
  if (active) {
    if (top) half_xface_sites<DAG, CLOVER, PHM, 2>(g, s0, f, in, ghp, U, Ughost, A, kappa, out);
    else half_xface_sites<DAG, CLOVER, PHM, 1>(g, s0, f, in, ghm, U, Ughost, A, kappa, out);
  }
  epi.pair_adj(s0, active, out);
}

// one thread per x-adjacent pair of the two boundary slabs (pairs
// [0, F/2) in slab t = 0, [F/2, F) in slab t = L_t - 1; F = L_x L_y L_z)
template <int DAG, bool CLOVER, int PHM, class CL, class Epi>
__global__ void __launch_bounds__(kDslashThreads, LMB_PAIR_MINB)
    wilson_half_tslab_kernel(const Geom g, const Field<PREC_HALF, 12> in, const Field<PREC_HALF, 12> ghm,
                             const Field<PREC_HALF, 12> ghp, const Gauge12<PREC_HALF> U,
                             const Gauge12<PREC_HALF> Ughost, const CL A, const float kappa, Epi epi) {
  if (epi.skip()) return;
  const int F = g.stride[3], half = F >> 1;
  const int i = blockIdx.x * kDslashThreads + threadIdx.x;
  const bool active = i < F;
  const bool top = i >= half;
  const int s0 = top ? (int)g.V - F + 2 * (i - half) : 2 * i;
  Cx2 out[12];
  if (active) {
    if (top) half_tslab_sites<DAG, CLOVER, PHM, 2>(g, s0, in, ghp, U, Ughost, A, kappa, out);
    else half_tslab_sites<DAG, CLOVER, PHM, 1>(g, s0, in, ghm, U, Ughost, A, kappa, out);
  }
  epi.pair_adj(s0, active, out);
}

// ---------------------------------------------------------------------------
// staggered / HISQ, one site per thread
// ---------------------------------------------------------------------------
template <typename R, int MU, int D, int P, class G>
LMB_D void stag_hop_dist(const Geom &g, const DistView &dv, int s, const int *c, const Field<P, 3> &in,
                         const GhostSpinors<P, 3> &gh, const G &U, const GhostLinks<G> &gu, R eta, Cx<R> *acc) {
  Cx<R> v[3], u[9], o[3];
  int w;
  load_nb(in, gh, g, dv, s, c, MU, D, v, &w);
  apply_wraps(g, MU, w, v);
  U.load(MU, s, u);
  su3_mul_vec(u, v, o);
#pragma unroll
  for (int i = 0; i < 3; i++) acc[i] = acc[i] + eta * o[i];
  load_nb(in, gh, g, dv, s, c, MU, -D, v, &w);
  apply_wraps(g, MU, w, v);
  load_link_nb(U, gu, g, dv, s, c, MU, -D, u);
  su3_adj_mul_vec(u, v, o);
#pragma unroll
  for (int i = 0; i < 3; i++) acc[i] = acc[i] - eta * o[i];
}

template <typename R, bool NAIK, int PHM, int P, class GF, class GL, class Epi>
__global__ void __launch_bounds__(kStagThreads)
    staggered_interior_kernel(const Geom g, const DistView dv, const Field<P, 3> in, const GF X, const GL Lk,
                              const R mass, const R fc, const R lc, Epi epi) {
  if (epi.skip()) return;
  const int i = blockIdx.x * kStagThreads + threadIdx.x;
  const bool active = i < dv.nsites;
  Cx<R> out[3];
  int c[4];
  const int s = active ? interior_site(g, dv, i, c) : 0;
  if (active) stag_site<R, NAIK, PHM>(g, s, in, X, Lk, mass, fc, lc, out);
  epi(s, active, out);
}

template <typename R, bool NAIK, int P, class GF, class GL, class Epi>
__global__ void __launch_bounds__(kStagThreads)
    staggered_boundary_kernel(const Geom g, const DistView dv, const Field<P, 3> in, const GhostSpinors<P, 3> gh,
                              const GF X, const GhostLinks<GF> gx, const GL Lk, const GhostLinks<GL> gl,
                              const R mass, const R fc, const R lc, Epi epi, const int *list, int n) {
  if (epi.skip()) return;
  const int i = blockIdx.x * kStagThreads + threadIdx.x;
  const bool active = i < n;
  const int s = active ? list[i] : 0;
  Cx<R> out[3];
  if (active) {
    int c[4];
    site_coords(g, s, c);
    const int p0 = c[0] + g.eta_off[0], p1 = p0 + c[1] + g.eta_off[1], p2 = p1 + c[2] + g.eta_off[2];
    const R eta[4] = {(R)1, (p0 & 1) ? (R)-1 : (R)1, (p1 & 1) ? (R)-1 : (R)1, (p2 & 1) ? (R)-1 : (R)1};
    Cx<R> fat[3] = {Cx<R>(0, 0), Cx<R>(0, 0), Cx<R>(0, 0)};
    stag_hop_dist<R, 0, 1>(g, dv, s, c, in, gh, X, gx, eta[0], fat);
    stag_hop_dist<R, 1, 1>(g, dv, s, c, in, gh, X, gx, eta[1], fat);
    stag_hop_dist<R, 2, 1>(g, dv, s, c, in, gh, X, gx, eta[2], fat);
    stag_hop_dist<R, 3, 1>(g, dv, s, c, in, gh, X, gx, eta[3], fat);
    Cx<R> psi[3];
    in.load(s, psi);
    if constexpr (NAIK) {
      Cx<R> lng[3] = {Cx<R>(0, 0), Cx<R>(0, 0), Cx<R>(0, 0)};
      stag_hop_dist<R, 0, 3>(g, dv, s, c, in, gh, Lk, gl, eta[0], lng);
      stag_hop_dist<R, 1, 3>(g, dv, s, c, in, gh, Lk, gl, eta[1], lng);
      stag_hop_dist<R, 2, 3>(g, dv, s, c, in, gh, Lk, gl, eta[2], lng);
      stag_hop_dist<R, 3, 3>(g, dv, s, c, in, gh, Lk, gl, eta[3], lng);
#pragma unroll
      for (int k = 0; k < 3; k++) out[k] = mass * psi[k] + fc * fat[k] + lc * lng[k];
    } else {
#pragma unroll
      for (int k = 0; k < 3; k++) out[k] = mass * psi[k] + fc * fat[k];
    }
  }
  epi(s, active, out);
}

// the scalar step after the sum over the ranks: sums[0] + sums[1] are the
// interior and boundary kernels' totals
template <class Epi>
__global__ void dist_finalize_kernel(Epi epi, const double *sums) {
  if (epi.skip()) return;  // a paused solve skipped the stencils as well
  if (threadIdx.x == 0 && blockIdx.x == 0) epi.finalize(sums[0] + sums[1]);
}

// the whole padded block of the caller's links (halo filled) as 36 planes of
// a lattice of the padded extents (site order of the padded array)
template <typename T>
__global__ void __launch_bounds__(256)
    padded_block_links_kernel(double2 *dst, const T *U0, const T *U1, const T *U2, const T *U3, int64_t Vp) {
  const int64_t t = (int64_t)blockIdx.x * 256 + threadIdx.x;
  if (t >= Vp) return;
  const T *U[4] = {U0, U1, U2, U3};
#pragma unroll
  for (int mu = 0; mu < 4; mu++)
#pragma unroll
    for (int k = 0; k < 9; k++) {
      const T v = U[mu][t * 9 + k];
      dst[(mu * 9 + k) * Vp + t] = make_double2((double)v.x, (double)v.y);
    }
}

// core sites of 54 field-strength planes computed on the padded block
template <int = 0>
__global__ void __launch_bounds__(256)
    core_of_padded_kernel(double2 *F, const double2 *Fp, const Geom g, const Padded pd, int64_t Vp) {
  const int s = blockIdx.x * 256 + threadIdx.x;
  if (s >= g.V) return;
  int c[4];
  site_coords(g, s, c);
  const int64_t ps = padded_site(pd, c);
  for (int k = 0; k < 54; k++) F[k * g.V + s] = Fp[k * Vp + ps];
}

}  // namespace lmb
