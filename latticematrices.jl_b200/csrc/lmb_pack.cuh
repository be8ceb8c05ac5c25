// lmb_pack.cuh -- conversion between the reference's halo-padded field layout
// and the internal structure-of-arrays planes, and the clover-block builder.
//
// Reference layout (LatticeMatrices_core.jl:4-9, 361-363): column-major
// (NC1, NC2, X+2nw, Y+2nw, Z+2nw, T+2nw), complex interleaved.  Only the core
// sites are read or written; the halo belongs to the caller, who marks it
// dirty after a write (mark_halo_dirty!, LatticeMatrices_core.jl:196-203).
#pragma once
#include "lmb_common.cuh"

namespace lmb {

struct Padded {
  int P[4];   // padded extents L + 2 nw
  int nw;
};

LMB_D int64_t padded_site(const Padded &pd, const int c[4]) {
  return (c[0] + pd.nw) +
         (int64_t)pd.P[0] * ((c[1] + pd.nw) + (int64_t)pd.P[1] * ((c[2] + pd.nw) + (int64_t)pd.P[2] * (c[3] + pd.nw)));
}

// TIN: double2 (ComplexF64) or float2 (ComplexF32)
template <typename TIN, int PS, int NC>
__global__ void __launch_bounds__(256)
    pack_field_kernel(Field<PS, NC> dst, const TIN *src, const Geom g, const Padded pd) {
  const int s = blockIdx.x * 256 + threadIdx.x;
  if (s >= g.V) return;
  int c[4];
  site_coords(g, s, c);
  const TIN *q = src + padded_site(pd, c) * NC;
  typedef typename Real<PS>::type R;
  Cx<R> v[NC];
#pragma unroll
  for (int k = 0; k < NC; k++) v[k] = Cx<R>((R)q[k].x, (R)q[k].y);
  dst.store(s, v);
}

template <typename TOUT, int PS, int NC>
__global__ void __launch_bounds__(256)
    unpack_field_kernel(TOUT *dst, const Field<PS, NC> src, const Geom g, const Padded pd) {
  const int s = blockIdx.x * 256 + threadIdx.x;
  if (s >= g.V) return;
  int c[4];
  site_coords(g, s, c);
  TOUT *q = dst + padded_site(pd, c) * NC;
  typedef typename Real<PS>::type R;
  Cx<R> v[NC];
  src.load(s, v);
#pragma unroll
  for (int k = 0; k < NC; k++) {
    q[k].x = v[k].re;
    q[k].y = v[k].im;
  }
}

// links: 4 padded (3,3,...) arrays -> 36 double2 planes (mu*9 + r + 3 col)
template <typename TIN>
__global__ void __launch_bounds__(256)
    pack_links_kernel(double2 *dst, const TIN *U0, const TIN *U1, const TIN *U2, const TIN *U3,
                      const Geom g, const Padded pd) {
  const int s = blockIdx.x * 256 + threadIdx.x;
  if (s >= g.V) return;
  int c[4];
  site_coords(g, s, c);
  const int64_t ps = padded_site(pd, c) * 9;
  const TIN *U[4] = {U0, U1, U2, U3};
#pragma unroll
  for (int mu = 0; mu < 4; mu++)
#pragma unroll
    for (int k = 0; k < 9; k++) {
      const TIN t = U[mu][ps + k];
      dst[(mu * 9 + k) * g.V + s] = make_double2((double)t.x, (double)t.y);
    }
}

// 36 double2 link planes -> single / half copies
template <int = 0>
__global__ void __launch_bounds__(256)
    links_to_single_kernel(float4 *dst, const double2 *src, int64_t V) {
  // 36 double2 planes (mu*9 + e) -> Gauge<PREC_SINGLE>: float4 planes
  // (mu*4 + k) holding entries 2k, 2k+1, then float2 planes (mu) holding 8
  const int64_t s = (int64_t)blockIdx.x * 256 + threadIdx.x;
  if (s >= V) return;
  float2 *last = reinterpret_cast<float2 *>(dst + 16 * V);
  for (int mu = 0; mu < 4; mu++) {
    for (int k = 0; k < 4; k++) {
      const double2 a = src[(mu * 9 + 2 * k) * V + s], b = src[(mu * 9 + 2 * k + 1) * V + s];
      dst[(mu * 4 + k) * V + s] = make_float4((float)a.x, (float)a.y, (float)b.x, (float)b.y);
    }
    const double2 c = src[(mu * 9 + 8) * V + s];
    last[mu * V + s] = make_float2((float)c.x, (float)c.y);
  }
}

// k = scale exponent (|values| <= 2^k)
template <int = 0>
__global__ void __launch_bounds__(256)
    links_to_half_kernel(int *dst, const double2 *src, int64_t n, int k) {
  const int64_t i = (int64_t)blockIdx.x * 256 + threadIdx.x;
  if (i >= n) return;
  const double2 t = src[i];
  const float inv = ldexpf(32768.0f, -k);
  dst[i] = enc_pair((float)t.x * inv, (float)t.y * inv);
}

// 36 double2 link planes (mu*9 + r + 3c) -> rows 0, 1 only (SU(3) links)
template <int = 0>
__global__ void __launch_bounds__(256)
    links_to_recon12_kernel(double2 *d12, float4 *f12, int4 *h12, const double2 *src, int64_t V) {
  const int64_t s = (int64_t)blockIdx.x * 256 + threadIdx.x;
  if (s >= V) return;
  double2 e[24];  // q = mu*6 + 3r + c
  for (int mu = 0; mu < 4; mu++)
    for (int r = 0; r < 2; r++)
      for (int c = 0; c < 3; c++) e[mu * 6 + 3 * r + c] = src[(mu * 9 + r + 3 * c) * V + s];
  if (d12)
    for (int q = 0; q < 24; q++) d12[q * V + s] = e[q];
  if (f12)
    for (int k = 0; k < 12; k++)
      f12[k * V + s] = make_float4((float)e[2 * k].x, (float)e[2 * k].y, (float)e[2 * k + 1].x, (float)e[2 * k + 1].y);
  if (h12)
    for (int k = 0; k < 6; k++) {
      int w[4];
      for (int j = 0; j < 4; j++)
        w[j] = enc_pair((float)e[4 * k + j].x * 32768.0f, (float)e[4 * k + j].y * 32768.0f);
      h12[k * V + s] = make_int4(w[0], w[1], w[2], w[3]);
    }
}

// max over links of |U U^+ - 1| and |det U - 1| (float bits, atomicMax)
template <int = 0>
__global__ void __launch_bounds__(256)
    su3_deviation_kernel(const double2 *U, int64_t V, unsigned *out_bits) {
  float m = 0.f;
  for (int64_t t = (int64_t)blockIdx.x * 256 + threadIdx.x; t < 4 * V; t += (int64_t)gridDim.x * 256) {
    const int mu = (int)(t / V);
    const int64_t s = t - mu * V;
    Cx<double> u[9];
    for (int k = 0; k < 9; k++) {
      const double2 x = U[(mu * 9 + k) * V + s];
      u[k] = Cx<double>(x.x, x.y);
    }
    double dev = 0;
    for (int r = 0; r < 3; r++)
      for (int c = 0; c < 3; c++) {
        Cx<double> v(0, 0);
        for (int k = 0; k < 3; k++) v = cfma_conj(u[c + 3 * k], u[r + 3 * k], v);  // (U U^+)_{rc}
        const double re = v.re - (r == c ? 1.0 : 0.0);
        dev = fmax(dev, fmax(fabs(re), fabs(v.im)));
      }
    const Cx<double> det = u[0] * (u[4] * u[8] - u[7] * u[5]) - u[3] * (u[1] * u[8] - u[7] * u[2]) +
                           u[6] * (u[1] * u[5] - u[4] * u[2]);
    dev = fmax(dev, fmax(fabs(det.re - 1.0), fabs(det.im)));
    m = fmaxf(m, (float)dev);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out_bits, __float_as_uint(m));
}

// max |re|, |im| over n complex entries (one atomicMax on the float bits;
// valid because the values are non-negative).  A NaN entry counts as +Inf
// (fmaxf would drop it), so the result is finite exactly when every entry
// is finite and within FP32 range.
template <int = 0>
__global__ void __launch_bounds__(256)
    absmax_kernel(const double2 *src, int64_t n, unsigned *out_bits) {
  float m = 0.f;
  for (int64_t i = (int64_t)blockIdx.x * 256 + threadIdx.x; i < n; i += (int64_t)gridDim.x * 256) {
    const double2 t = src[i];
    const float a = fmaxf(fabsf((float)t.x), fabsf((float)t.y));
    m = fmaxf(m, (isnan(t.x) || isnan(t.y)) ? INFINITY : a);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out_bits, __float_as_uint(m));
}

// ---------------------------------------------------------------------------
// clover field strength F_mu_nu = (Q - Q^+)/8 (WilsonDiracCloverOperator.jl:
// 186-226) and the clover blocks A = 1 + coef * B, coef = -kappa cSW,
// B = sum_{mu<nu} g_mu g_nu F_mu_nu in block form (WilsonDiracCloverOperator.jl:
// 481-525).  F planes: (plane*9 + r + 3 col) double2, planes (12,13,14,23,24,34).
// ---------------------------------------------------------------------------
LMB_D void load_link(const double2 *U, const Geom &g, int mu, int s, Cx<double> *m) {
#pragma unroll
  for (int k = 0; k < 9; k++) {
    const double2 t = U[(mu * 9 + k) * g.V + s];
    m[k] = Cx<double>(t.x, t.y);
  }
}
LMB_D void mat3_mul(const Cx<double> *a, const Cx<double> *b, Cx<double> *c) {
  Cx<double> t[9];
#pragma unroll
  for (int r = 0; r < 3; r++)
#pragma unroll
    for (int col = 0; col < 3; col++) {
      Cx<double> v = a[r] * b[3 * col];
      v = cfma(a[r + 3], b[1 + 3 * col], v);
      v = cfma(a[r + 6], b[2 + 3 * col], v);
      t[r + 3 * col] = v;
    }
#pragma unroll
  for (int k = 0; k < 9; k++) c[k] = t[k];
}
LMB_D void mat3_adj(Cx<double> *m) {
  Cx<double> t[9];
#pragma unroll
  for (int r = 0; r < 3; r++)
#pragma unroll
    for (int col = 0; col < 3; col++) t[r + 3 * col] = conj(m[col + 3 * r]);
#pragma unroll
  for (int k = 0; k < 9; k++) m[k] = t[k];
}

template <int = 0>
__global__ void __launch_bounds__(128)
    clover_field_strength_kernel(double2 *F, const double2 *U, const Geom g) {
  const int64_t tid = (int64_t)blockIdx.x * 128 + threadIdx.x;
  if (tid >= 6 * g.V) return;
  const int plane = (int)(tid / g.V);
  const int s = (int)(tid - (int64_t)plane * g.V);
  const int pmu[6] = {0, 0, 0, 1, 1, 2}, pnu[6] = {1, 2, 3, 2, 3, 3};
  const int mu = pmu[plane], nu = pnu[plane];
  int c[4], w;
  site_coords(g, s, c);
  const int xpmu = fwd_site(g, s, c, mu, 1, &w);
  const int xpnu = fwd_site(g, s, c, nu, 1, &w);
  const int xmmu = bwd_site(g, s, c, mu, 1, &w);
  const int xmnu = bwd_site(g, s, c, nu, 1, &w);
  int cc[4];
  site_coords(g, xpnu, cc);
  const int xpnu_mmu = bwd_site(g, xpnu, cc, mu, 1, &w);
  site_coords(g, xmmu, cc);
  const int xmmu_mnu = bwd_site(g, xmmu, cc, nu, 1, &w);
  site_coords(g, xpmu, cc);
  const int xpmu_mnu = bwd_site(g, xpmu, cc, nu, 1, &w);
  Cx<double> q[9], a[9], b[9];
#pragma unroll
  for (int k = 0; k < 9; k++) q[k] = Cx<double>(0, 0);
  // +mu +nu -mu -nu
  load_link(U, g, mu, s, a);
  load_link(U, g, nu, xpmu, b); mat3_mul(a, b, a);
  load_link(U, g, mu, xpnu, b); mat3_adj(b); mat3_mul(a, b, a);
  load_link(U, g, nu, s, b); mat3_adj(b); mat3_mul(a, b, a);
  for (int k = 0; k < 9; k++) q[k] = q[k] + a[k];
  // +nu -mu -nu +mu
  load_link(U, g, nu, s, a);
  load_link(U, g, mu, xpnu_mmu, b); mat3_adj(b); mat3_mul(a, b, a);
  load_link(U, g, nu, xmmu, b); mat3_adj(b); mat3_mul(a, b, a);
  load_link(U, g, mu, xmmu, b); mat3_mul(a, b, a);
  for (int k = 0; k < 9; k++) q[k] = q[k] + a[k];
  // -mu -nu +mu +nu
  load_link(U, g, mu, xmmu, a); mat3_adj(a);
  load_link(U, g, nu, xmmu_mnu, b); mat3_adj(b); mat3_mul(a, b, a);
  load_link(U, g, mu, xmmu_mnu, b); mat3_mul(a, b, a);
  load_link(U, g, nu, xmnu, b); mat3_mul(a, b, a);
  for (int k = 0; k < 9; k++) q[k] = q[k] + a[k];
  // -nu +mu +nu -mu
  load_link(U, g, nu, xmnu, a); mat3_adj(a);
  load_link(U, g, mu, xmnu, b); mat3_mul(a, b, a);
  load_link(U, g, nu, xpmu_mnu, b); mat3_mul(a, b, a);
  load_link(U, g, mu, s, b); mat3_adj(b); mat3_mul(a, b, a);
  for (int k = 0; k < 9; k++) q[k] = q[k] + a[k];
#pragma unroll
  for (int r = 0; r < 3; r++)
#pragma unroll
    for (int col = 0; col < 3; col++) {
      const Cx<double> v = 0.125 * (q[r + 3 * col] - conj(q[col + 3 * r]));
      F[(plane * 9 + r + 3 * col) * g.V + s] = make_double2(v.re, v.im);
    }
}

// one site: the two packed Hermitian blocks (72 doubles) of A = 1 + coef B
LMB_D void clover_blocks_site(const double2 *F, const Geom &g, int s, double coef, double *out) {
  Cx<double> f[6][9];
#pragma unroll
  for (int p = 0; p < 6; p++)
#pragma unroll
    for (int k = 0; k < 9; k++) {
      const double2 t = F[(p * 9 + k) * g.V + s];
      f[p][k] = Cx<double>(t.x, t.y);
    }
  // planes: 0=12 1=13 2=14 3=23 4=24 5=34
  for (int blk = 0; blk < 2; blk++) {
    Cx<double> B[6][6];
    for (int c = 0; c < 3; c++)
      for (int cp = 0; cp < 3; cp++) {
        const int k = c + 3 * cp;
        const Cx<double> f12 = f[0][k], f13 = f[1][k], f14 = f[2][k], f23 = f[3][k], f24 = f[4][k],
                         f34 = f[5][k];
        Cx<double> d, o01, o10;
        if (blk == 0) {
          d = mul_i(f12 + f34);
          const Cx<double> op = mul_i(f14 + f23);
          o01 = (f24 - f13) + op;
          o10 = (f13 - f24) + op;
        } else {
          d = mul_i(f12 - f34);
          const Cx<double> om = mul_i(f23 - f14);
          o01 = om - f13 - f24;
          o10 = om + f13 + f24;
        }
        B[c][cp] = d;
        B[c][cp + 3] = o01;
        B[c + 3][cp] = o10;
        B[c + 3][cp + 3] = -d;
      }
    double *a = out + 36 * blk;
    for (int i = 0; i < 6; i++) a[i] = 1.0 + coef * B[i][i].re;
    int k = 6;
    for (int i = 1; i < 6; i++)
      for (int j = 0; j < i; j++) {
        a[k] = coef * B[i][j].re;
        a[k + 1] = coef * B[i][j].im;
        k += 2;
      }
  }
}

// FP64: 36 double2 planes (blk*18 + k)
template <int = 0>
__global__ void __launch_bounds__(128)
    clover_blocks_double_kernel(double2 *A, const double2 *F, const Geom g, double coef) {
  const int s = blockIdx.x * 128 + threadIdx.x;
  if (s >= g.V) return;
  double a[72];
  clover_blocks_site(F, g, s, coef, a);
  for (int k = 0; k < 36; k++) A[k * g.V + s] = make_double2(a[2 * k], a[2 * k + 1]);
}

template <int = 0>
__global__ void __launch_bounds__(256)
    clover_to_single_kernel(float4 *dst, const double2 *src, int64_t V) {
  const int64_t s = (int64_t)blockIdx.x * 256 + threadIdx.x;
  if (s >= V) return;
  for (int k = 0; k < 18; k++) {
    const double2 a = src[(2 * k) * V + s], b = src[(2 * k + 1) * V + s];
    dst[k * V + s] = make_float4((float)a.x, (float)a.y, (float)b.x, (float)b.y);
  }
}

template <int = 0>
__global__ void __launch_bounds__(256)
    clover_to_half_kernel(int4 *dst, int2 *tail, const double2 *src, int64_t V, int kexp) {
  const int64_t s = (int64_t)blockIdx.x * 256 + threadIdx.x;
  if (s >= V) return;
  const float inv = ldexpf(32768.0f, -kexp);
  for (int blk = 0; blk < 2; blk++) {
    int w[18];
    for (int k = 0; k < 18; k++) {
      const double2 t = src[(blk * 18 + k) * V + s];
      w[k] = enc_pair((float)t.x * inv, (float)t.y * inv);
    }
    for (int k = 0; k < 4; k++) dst[(blk * 4 + k) * V + s] = make_int4(w[4 * k], w[4 * k + 1], w[4 * k + 2], w[4 * k + 3]);
    tail[blk * V + s] = make_int2(w[16], w[17]);
  }
}

}  // namespace lmb
