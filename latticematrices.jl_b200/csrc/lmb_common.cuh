// lmb_common.cuh -- shared device code for liblmb200: complex arithmetic,
// lattice geometry, the structure-of-arrays field storage used on the GPU,
// and a deterministic grid-wide reduction.
//
// Internal layout.  Every field lives as "planes" of 16-byte (or smaller)
// vectors with the lattice site fastest: plane k of a field holds component
// group k for all V sites, so the 32 lanes of a warp read 32 consecutive
// vectors (fully coalesced 128-bit loads).  Site order is the reference's
// lexicographic order, x fastest (Latticeindices.jl:2-33).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define LMB_HD __host__ __device__ __forceinline__
#define LMB_D __device__ __forceinline__

namespace lmb {

enum Precision { PREC_DOUBLE = 0, PREC_SINGLE = 1, PREC_HALF = 2 };

// ---------------------------------------------------------------------------
// complex numbers
// ---------------------------------------------------------------------------
template <typename R>
struct Cx {
  R re, im;
  LMB_HD Cx() {}
  LMB_HD Cx(R r, R i) : re(r), im(i) {}
};

template <typename R> LMB_HD Cx<R> cx(R r, R i) { return Cx<R>(r, i); }
template <typename R> LMB_HD Cx<R> operator+(Cx<R> a, Cx<R> b) { return Cx<R>(a.re + b.re, a.im + b.im); }
template <typename R> LMB_HD Cx<R> operator-(Cx<R> a, Cx<R> b) { return Cx<R>(a.re - b.re, a.im - b.im); }
template <typename R> LMB_HD Cx<R> operator-(Cx<R> a) { return Cx<R>(-a.re, -a.im); }
template <typename R> LMB_HD Cx<R> operator*(Cx<R> a, Cx<R> b) {
  return Cx<R>(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re);
}
template <typename R> LMB_HD Cx<R> operator*(R s, Cx<R> a) { return Cx<R>(s * a.re, s * a.im); }
template <typename R> LMB_HD Cx<R> conj(Cx<R> a) { return Cx<R>(a.re, -a.im); }
// i * a
template <typename R> LMB_HD Cx<R> mul_i(Cx<R> a) { return Cx<R>(-a.im, a.re); }
// acc + a * b
template <typename R> LMB_HD Cx<R> cfma(Cx<R> a, Cx<R> b, Cx<R> acc) {
  acc.re = acc.re + a.re * b.re;
  acc.re = acc.re - a.im * b.im;
  acc.im = acc.im + a.re * b.im;
  acc.im = acc.im + a.im * b.re;
  return acc;
}
// acc + conj(a) * b
template <typename R> LMB_HD Cx<R> cfma_conj(Cx<R> a, Cx<R> b, Cx<R> acc) {
  acc.re = acc.re + a.re * b.re;
  acc.re = acc.re + a.im * b.im;
  acc.im = acc.im + a.re * b.im;
  acc.im = acc.im - a.im * b.re;
  return acc;
}
template <typename R> LMB_HD R norm2(Cx<R> a) { return a.re * a.re + a.im * a.im; }

// ---------------------------------------------------------------------------
// geometry (single rank: periodic wrap with the fermion boundary phase)
// ---------------------------------------------------------------------------
struct Geom {
  int L[4];
  int stride[4];      // 1, Lx, Lx*Ly, Lx*Ly*Lz
  int64_t V;
  double ph_fwd[4][2];  // factor on a forward wrap (phase)
  double ph_bwd[4][2];  // factor on a backward wrap (1/phase)
  int phase_mask;       // bit mu set when phase[mu] != 1
  int eta_off[4];       // global coordinate of the local origin (staggered eta)
};

LMB_D void site_coords(const Geom &g, int s, int c[4]) {
  int q = s / g.L[0];
  c[0] = s - q * g.L[0];
  int q2 = q / g.L[1];
  c[1] = q - q2 * g.L[1];
  int q3 = q2 / g.L[2];
  c[2] = q2 - q3 * g.L[2];
  c[3] = q3;
}

// neighbour at +d (d in 1..3) along mu; *wrap = 1 when the edge was crossed
LMB_D int fwd_site(const Geom &g, int s, const int c[4], int mu, int d, int *wrap) {
  int cc = c[mu] + d;
  *wrap = cc >= g.L[mu];
  return *wrap ? s + (d - g.L[mu]) * g.stride[mu] : s + d * g.stride[mu];
}
LMB_D int bwd_site(const Geom &g, int s, const int c[4], int mu, int d, int *wrap) {
  int cc = c[mu] - d;
  *wrap = cc < 0;
  return *wrap ? s + (g.L[mu] - d) * g.stride[mu] : s - d * g.stride[mu];
}

// ---------------------------------------------------------------------------
// storage traits
// ---------------------------------------------------------------------------
constexpr float kInt16Scale = 32767.0f;

template <int P> struct Real { typedef float type; };
template <> struct Real<PREC_DOUBLE> { typedef double type; };

// A field of NCOMP complex numbers per site.
//  double: NCOMP planes of double2
//  single: ceil(NCOMP/2) planes of float4
//  half  : ceil(NCOMP/4) planes of int4 (8 x int16) + one float norm per site
template <int P, int NCOMP> struct Field;

template <int NCOMP> struct Field<PREC_DOUBLE, NCOMP> {
  double2 *data;
  float *norm;  // unused
  int64_t V;
  static constexpr int kPlanes = NCOMP;
  static size_t bytes(int64_t V) { return sizeof(double2) * NCOMP * V; }
  static size_t norm_bytes(int64_t) { return 0; }
  template <typename R> LMB_D void load(int64_t s, Cx<R> *v) const {
#pragma unroll
    for (int k = 0; k < NCOMP; k++) {
      double2 t = __ldg(data + k * V + s);
      v[k] = Cx<R>((R)t.x, (R)t.y);
    }
  }
  template <typename R> LMB_D void store(int64_t s, const Cx<R> *v) const {
#pragma unroll
    for (int k = 0; k < NCOMP; k++) data[k * V + s] = make_double2((double)v[k].re, (double)v[k].im);
  }
};

template <int NCOMP> struct Field<PREC_SINGLE, NCOMP> {
  float4 *data;
  float *norm;
  int64_t V;
  static constexpr int kPlanes = (NCOMP + 1) / 2;
  static size_t bytes(int64_t V) { return sizeof(float4) * kPlanes * V; }
  static size_t norm_bytes(int64_t) { return 0; }
  template <typename R> LMB_D void load(int64_t s, Cx<R> *v) const {
#pragma unroll
    for (int k = 0; k < kPlanes; k++) {
      float4 t = __ldg(data + k * V + s);
      v[2 * k] = Cx<R>((R)t.x, (R)t.y);
      if (2 * k + 1 < NCOMP) v[2 * k + 1] = Cx<R>((R)t.z, (R)t.w);
    }
  }
  template <typename R> LMB_D void store(int64_t s, const Cx<R> *v) const {
#pragma unroll
    for (int k = 0; k < kPlanes; k++) {
      float4 t;
      t.x = (float)v[2 * k].re;
      t.y = (float)v[2 * k].im;
      t.z = (2 * k + 1 < NCOMP) ? (float)v[2 * k + 1].re : 0.f;
      t.w = (2 * k + 1 < NCOMP) ? (float)v[2 * k + 1].im : 0.f;
      data[k * V + s] = t;
    }
  }
};

LMB_D short f2s(float x) { return (short)__float2int_rn(x); }

template <int NCOMP> struct Field<PREC_HALF, NCOMP> {
  int4 *data;
  float *norm;
  int64_t V;
  static constexpr int kPlanes = (NCOMP + 3) / 4;
  static size_t bytes(int64_t V) { return sizeof(int4) * kPlanes * V; }
  static size_t norm_bytes(int64_t V) { return sizeof(float) * V; }
  template <typename R> LMB_D void load(int64_t s, Cx<R> *v) const {
    const float scale = __ldg(norm + s) * (1.0f / kInt16Scale);
#pragma unroll
    for (int k = 0; k < kPlanes; k++) {
      int4 t = __ldg(data + k * V + s);
      const int w[4] = {t.x, t.y, t.z, t.w};
#pragma unroll
      for (int j = 0; j < 4; j++) {
        if (4 * k + j < NCOMP) {
          short lo = (short)(w[j] & 0xffff), hi = (short)(w[j] >> 16);
          v[4 * k + j] = Cx<R>((R)((float)lo * scale), (R)((float)hi * scale));
        }
      }
    }
  }
  template <typename R> LMB_D void store(int64_t s, const Cx<R> *v) const {
    float m = 0.f;
#pragma unroll
    for (int k = 0; k < NCOMP; k++) m = fmaxf(m, fmaxf(fabsf((float)v[k].re), fabsf((float)v[k].im)));
    const float inv = m > 0.f ? kInt16Scale / m : 0.f;
#pragma unroll
    for (int k = 0; k < kPlanes; k++) {
      int w[4];
#pragma unroll
      for (int j = 0; j < 4; j++) {
        if (4 * k + j < NCOMP) {
          short lo = f2s((float)v[4 * k + j].re * inv), hi = f2s((float)v[4 * k + j].im * inv);
          w[j] = ((int)(unsigned short)lo) | ((int)hi << 16);
        } else {
          w[j] = 0;
        }
      }
      data[k * V + s] = make_int4(w[0], w[1], w[2], w[3]);
    }
    norm[s] = m;
  }
};

// Gauge links: 4 directions x 9 complex per site, plane (mu*9 + k).
//  double: double2 planes; single: float2 planes; half: int16 pairs scaled
//  by a global `scale` (max |element| over the lattice).
template <int P> struct Gauge;
template <> struct Gauge<PREC_DOUBLE> {
  const double2 *data;
  int64_t V;
  float scale;
  static size_t bytes(int64_t V) { return sizeof(double2) * 36 * V; }
  template <typename R> LMB_D void load(int mu, int64_t s, Cx<R> *u) const {
#pragma unroll
    for (int k = 0; k < 9; k++) {
      double2 t = __ldg(data + (mu * 9 + k) * V + s);
      u[k] = Cx<R>((R)t.x, (R)t.y);
    }
  }
};
template <> struct Gauge<PREC_SINGLE> {
  const float2 *data;
  int64_t V;
  float scale;
  static size_t bytes(int64_t V) { return sizeof(float2) * 36 * V; }
  template <typename R> LMB_D void load(int mu, int64_t s, Cx<R> *u) const {
#pragma unroll
    for (int k = 0; k < 9; k++) {
      float2 t = __ldg(data + (mu * 9 + k) * V + s);
      u[k] = Cx<R>((R)t.x, (R)t.y);
    }
  }
};
template <> struct Gauge<PREC_HALF> {
  const int *data;  // packed (re, im) int16 pairs
  int64_t V;
  float scale;
  static size_t bytes(int64_t V) { return sizeof(int) * 36 * V; }
  template <typename R> LMB_D void load(int mu, int64_t s, Cx<R> *u) const {
    const float f = scale * (1.0f / kInt16Scale);
#pragma unroll
    for (int k = 0; k < 9; k++) {
      int w = __ldg(data + (mu * 9 + k) * V + s);
      u[k] = Cx<R>((R)((float)(short)(w & 0xffff) * f), (R)((float)(short)(w >> 16) * f));
    }
  }
};

// Clover blocks: two Hermitian 6x6 matrices per site (spin pairs (1,2) and
// (3,4)), each packed as 6 real diagonal entries followed by the 15 complex
// entries below the diagonal in row order: 36 reals per block, 72 per site.
//  double: 36 planes of double2 (pairs of reals);  single: 18 float4 planes;
//  half: 9 int4 planes with a global scale.
template <int P> struct Clover;
template <> struct Clover<PREC_DOUBLE> {
  const double2 *data;
  int64_t V;
  float scale;
  static size_t bytes(int64_t V) { return sizeof(double2) * 36 * V; }
  template <typename R> LMB_D void load(int blk, int64_t s, R *a) const {
#pragma unroll
    for (int k = 0; k < 18; k++) {
      double2 t = __ldg(data + (blk * 18 + k) * V + s);
      a[2 * k] = (R)t.x;
      a[2 * k + 1] = (R)t.y;
    }
  }
};
template <> struct Clover<PREC_SINGLE> {
  const float4 *data;
  int64_t V;
  float scale;
  static size_t bytes(int64_t V) { return sizeof(float4) * 18 * V; }
  template <typename R> LMB_D void load(int blk, int64_t s, R *a) const {
#pragma unroll
    for (int k = 0; k < 9; k++) {
      float4 t = __ldg(data + (blk * 9 + k) * V + s);
      a[4 * k] = (R)t.x;
      a[4 * k + 1] = (R)t.y;
      a[4 * k + 2] = (R)t.z;
      a[4 * k + 3] = (R)t.w;
    }
  }
};
template <> struct Clover<PREC_HALF> {
  // per block: 32 int16 in four int4 planes + 4 int16 in one int2 plane
  const int4 *data;  // 8 planes: block*4 + k
  const int2 *tail;  // 2 planes: block
  int64_t V;
  float scale;
  static size_t bytes(int64_t V) { return (sizeof(int4) * 8 + sizeof(int2) * 2) * V; }
  template <typename R> LMB_D void load(int blk, int64_t s, R *a) const {
    const float f = scale * (1.0f / kInt16Scale);
#pragma unroll
    for (int k = 0; k < 4; k++) {
      int4 t = __ldg(data + (blk * 4 + k) * V + s);
      const int w[4] = {t.x, t.y, t.z, t.w};
#pragma unroll
      for (int j = 0; j < 4; j++) {
        a[8 * k + 2 * j] = (R)((float)(short)(w[j] & 0xffff) * f);
        a[8 * k + 2 * j + 1] = (R)((float)(short)(w[j] >> 16) * f);
      }
    }
    int2 t = __ldg(tail + blk * V + s);
    a[32] = (R)((float)(short)(t.x & 0xffff) * f);
    a[33] = (R)((float)(short)(t.x >> 16) * f);
    a[34] = (R)((float)(short)(t.y & 0xffff) * f);
    a[35] = (R)((float)(short)(t.y >> 16) * f);
  }
};

// ---------------------------------------------------------------------------
// deterministic grid reduction of N doubles: each block reduces its values,
// thread 0 stores them in partials[N * block], the last block to arrive sums
// all partials in block order and returns true (others false).
// ---------------------------------------------------------------------------
template <int NT, int N>
LMB_D bool grid_reduce(double (&v)[N], double *partials, unsigned *counter, double (&total)[N]) {
  __shared__ double red[N][NT / 32];
  __shared__ bool last;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int n = 0; n < N; n++) {
    double x = v[n];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    if (lane == 0) red[n][warp] = x;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int n = 0; n < N; n++) {
      double x = 0;
      for (int w = 0; w < NT / 32; w++) x += red[n][w];
      partials[(size_t)N * blockIdx.x + n] = x;
    }
    __threadfence();
    unsigned ticket = atomicAdd(counter, 1u);
    last = (ticket == gridDim.x - 1);
  }
  __syncthreads();
  if (!last) return false;
  __threadfence();
#pragma unroll
  for (int n = 0; n < N; n++) {
    double x = 0;
    for (unsigned b = threadIdx.x; b < gridDim.x; b += NT)
      x += ((volatile double *)partials)[(size_t)N * b + n];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    if (lane == 0) red[n][warp] = x;
  }
  __syncthreads();
#pragma unroll
  for (int n = 0; n < N; n++) {
    double x = 0;
    for (int w = 0; w < NT / 32; w++) x += red[n][w];
    total[n] = x;
  }
  if (threadIdx.x == 0) *counter = 0u;
  return true;
}

}  // namespace lmb
