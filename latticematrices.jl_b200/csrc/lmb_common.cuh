// lmb_common.cuh -- shared device code for liblmb200: complex arithmetic,
// lattice geometry, the structure-of-arrays field storage used on the GPU,
// and a deterministic grid-wide reduction.
//
// Internal layout.  Every field lives as "planes" of 16-byte (or smaller)
// vectors with the lattice site fastest: plane k of a field holds component
// group k for all V sites, so the 32 lanes of a warp read 32 consecutive
// vectors (fully coalesced 128-bit loads).  Site order is the reference's
// lexicographic order, x fastest (Latticeindices.jl:2-33).
//
// Build.  The library is several translation units compiled in parallel, and
// every one of them includes these headers.  A kernel without template
// parameters of its own is declared `template <int = 0>` so that only the
// units that launch it compile it (launch sites need no `<>`).
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

// the sites [lo, hi) of one stencil launch: the whole lattice, or the
// interior slab of a block split along t only (every t-hop stays local)
struct SiteRange {
  int lo, hi;
};
inline SiteRange whole(const Geom &g) { return SiteRange{0, (int)g.V}; }

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

// three-component (staggered) FP32 field, no padding: one float4 plane
// (components 0, 1) followed by one float2 plane (component 2) -- two loads
template <> struct Field<PREC_SINGLE, 3> {
  float4 *data;
  float *norm;
  int64_t V;
  static constexpr int kPlanes = 2;
  static size_t bytes(int64_t V) { return sizeof(float2) * 3 * V; }
  static size_t norm_bytes(int64_t) { return 0; }
  LMB_D float2 *last() const { return reinterpret_cast<float2 *>(data + V); }
  template <typename R> LMB_D void load(int64_t s, Cx<R> *v) const {
    const float4 a = __ldg(data + s);
    const float2 b = __ldg(last() + s);
    v[0] = Cx<R>((R)a.x, (R)a.y);
    v[1] = Cx<R>((R)a.z, (R)a.w);
    v[2] = Cx<R>((R)b.x, (R)b.y);
  }
  template <typename R> LMB_D void store(int64_t s, const Cx<R> *v) const {
    data[s] = make_float4((float)v[0].re, (float)v[0].im, (float)v[1].re, (float)v[1].im);
    last()[s] = make_float2((float)v[2].re, (float)v[2].im);
  }
};

LMB_D short f2s(float x) { return (short)__float2int_rn(x); }

// int16 storage.  Every int16 group (a site's spinor, the links, the clover
// blocks) carries a power-of-two scale 2^k with all |values| <= 2^k; a value
// v is stored as u = q + 32768 with q = rint(v 2^-k 32768) in [-32767, 32767].
// Decoding needs no integer conversion: with base = 2^(8+k), the float whose
// exponent is base's and whose low 16 mantissa bits are u equals
// base (1 + u 2^-23); subtracting base (1 + 2^-8) leaves q 2^(k-15) = v
// exactly.  One byte permute builds each float, one packed FADD2 finishes a
// complex pair.
struct Dec16 {
  unsigned y;  // high 16 bits of base (exponent field)
  float c;     // base (1 + 2^-8)
};
LMB_D Dec16 dec16_of_base(float base) {
  Dec16 d;
  d.y = __float_as_uint(base) >> 16;
  d.c = base * 1.00390625f;
  return d;
}
LMB_D float2 dec_pair(int w, const Dec16 &d) {
  const float lo = __uint_as_float(__byte_perm((unsigned)w, d.y, 0x5410u));
  const float hi = __uint_as_float(__byte_perm((unsigned)w, d.y, 0x5432u));
  return __fadd2_rn(make_float2(lo, hi), make_float2(-d.c, -d.c));
}
// scale exponent k for a maximum magnitude m (|v| <= m <= 2^k), and base
LMB_HD int pow2_exponent(float m) {
  if (!(m > 0.f)) return 0;
  int e;
  frexpf(m, &e);  // m = f 2^e, 0.5 <= f < 1, so m < 2^e
  if (e < -130) e = -130;
  if (e > 110) e = 110;
  return e;
}
LMB_HD float base_of_exponent(int k) { return ldexpf(1.0f, 8 + k); }
// encode a complex pair already scaled to [-32768, 32768]: clamp to
// +-32767 and add 2^23 + 32768, so that the float's low 16 mantissa bits are
// u = rint(q) + 32768; one byte permute packs the two halves (no F2I)
LMB_D int enc_pair(float a, float b) {
  const float fa = fminf(fmaxf(a, -32767.f), 32767.f) + 8421376.0f;
  const float fb = fminf(fmaxf(b, -32767.f), 32767.f) + 8421376.0f;
  return (int)__byte_perm(__float_as_uint(fa), __float_as_uint(fb), 0x5410u);
}

template <int NCOMP> struct Field<PREC_HALF, NCOMP> {
  int4 *data;
  float *norm;  // per-site base 2^(8+k)
  int64_t V;
  static constexpr int kPlanes = (NCOMP + 3) / 4;
  static size_t bytes(int64_t V) { return sizeof(int4) * kPlanes * V; }
  static size_t norm_bytes(int64_t V) { return sizeof(float) * V; }
  template <typename R> LMB_D void load(int64_t s, Cx<R> *v) const {
    const Dec16 d = dec16_of_base(__ldg(norm + s));
#pragma unroll
    for (int k = 0; k < kPlanes; k++) {
      int4 t = __ldg(data + k * V + s);
      const int w[4] = {t.x, t.y, t.z, t.w};
#pragma unroll
      for (int j = 0; j < 4; j++)
        if (4 * k + j < NCOMP) {
          const float2 f = dec_pair(w[j], d);
          v[4 * k + j] = Cx<R>((R)f.x, (R)f.y);
        }
    }
  }
  template <typename R> LMB_D void store(int64_t s, const Cx<R> *v) const {
    float m = 0.f;
#pragma unroll
    for (int k = 0; k < NCOMP; k++) m = fmaxf(m, fmaxf(fabsf((float)v[k].re), fabsf((float)v[k].im)));
    const int e = pow2_exponent(m);
    const float inv = ldexpf(32768.0f, -e);
#pragma unroll
    for (int k = 0; k < kPlanes; k++) {
      int w[4];
#pragma unroll
      for (int j = 0; j < 4; j++)
        w[j] = (4 * k + j < NCOMP) ? enc_pair((float)v[4 * k + j].re * inv, (float)v[4 * k + j].im * inv)
                                   : enc_pair(0.f, 0.f);
      data[k * V + s] = make_int4(w[0], w[1], w[2], w[3]);
    }
    norm[s] = base_of_exponent(e);
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
// FP32, 18 reals: per direction four float4 planes (entries 2k, 2k+1) and one
// float2 plane (entry 8) -- five loads per link; data points at the 16 float4
// planes (mu*4 + k), followed by the 4 float2 planes (mu) at data + 16 V
template <> struct Gauge<PREC_SINGLE> {
  const float4 *data;
  int64_t V;
  float scale;
  static size_t bytes(int64_t V) { return sizeof(float2) * 36 * V; }
  LMB_D const float2 *last() const { return reinterpret_cast<const float2 *>(data + 16 * V); }
  template <typename R> LMB_D void load(int mu, int64_t s, Cx<R> *u) const {
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const float4 t = __ldg(data + (mu * 4 + k) * V + s);
      u[2 * k] = Cx<R>((R)t.x, (R)t.y);
      u[2 * k + 1] = Cx<R>((R)t.z, (R)t.w);
    }
    const float2 t = __ldg(last() + mu * V + s);
    u[8] = Cx<R>((R)t.x, (R)t.y);
  }
};
template <> struct Gauge<PREC_HALF> {
  const int *data;  // packed (re, im) int16 pairs
  int64_t V;
  float scale;      // base 2^(8+k) of the global power-of-two scale
  static size_t bytes(int64_t V) { return sizeof(int) * 36 * V; }
  template <typename R> LMB_D void load(int mu, int64_t s, Cx<R> *u) const {
    const Dec16 d = dec16_of_base(scale);
#pragma unroll
    for (int k = 0; k < 9; k++) {
      const float2 f = dec_pair(__ldg(data + (mu * 9 + k) * V + s), d);
      u[k] = Cx<R>((R)f.x, (R)f.y);
    }
  }
};

// third row of an SU(3) matrix from the first two: row2 = conj(row0 x row1)
// (the reconstruction of kernel_normalize_NC3!, linearalgebra_D.jl:2371-2424);
// u column-major u[r + 3c]
template <typename R>
LMB_D void su3_third_row(Cx<R> *u) {
  u[2] = conj(u[3] * u[7] - u[6] * u[4]);
  u[5] = conj(u[6] * u[1] - u[0] * u[7]);
  u[8] = conj(u[0] * u[4] - u[3] * u[1]);
}

// Links known to be SU(3): only rows 0 and 1 are stored (12 reals), entry
// e = 3 r + c of direction mu.
//  double: 24 double2 planes (mu*6 + e)
//  single: 12 float4 planes (mu*3 + k), float4 k = entries 2k, 2k+1
//  half  : 6 int4 planes; complex q = mu*6 + e sits in plane q/4, lane q%4;
//          int16 values scaled by 1 (|U_ij| <= 1)
template <int P> struct Gauge12;
template <> struct Gauge12<PREC_DOUBLE> {
  const double2 *data;
  int64_t V;
  float scale;
  template <typename R> LMB_D void load(int mu, int64_t s, Cx<R> *u) const {
#pragma unroll
    for (int e = 0; e < 6; e++) {
      const double2 t = __ldg(data + (mu * 6 + e) * V + s);
      u[(e / 3) + 3 * (e % 3)] = Cx<R>((R)t.x, (R)t.y);
    }
    su3_third_row(u);
  }
};
template <> struct Gauge12<PREC_SINGLE> {
  const float4 *data;
  int64_t V;
  float scale;
  template <typename R> LMB_D void load(int mu, int64_t s, Cx<R> *u) const {
#pragma unroll
    for (int k = 0; k < 3; k++) {
      const float4 t = __ldg(data + (mu * 3 + k) * V + s);
      const int e0 = 2 * k, e1 = 2 * k + 1;
      u[(e0 / 3) + 3 * (e0 % 3)] = Cx<R>((R)t.x, (R)t.y);
      u[(e1 / 3) + 3 * (e1 % 3)] = Cx<R>((R)t.z, (R)t.w);
    }
    su3_third_row(u);
  }
};
template <> struct Gauge12<PREC_HALF> {
  const int4 *data;
  int64_t V;
  float scale;  // unused: |U_ij| <= 1, scale exponent 0
  template <typename R> LMB_D void load(int mu, int64_t s, Cx<R> *u) const {
    const int q0 = mu * 6, p0 = q0 >> 2, lane0 = q0 & 3;
    const int4 a = __ldg(data + p0 * V + s), b = __ldg(data + (p0 + 1) * V + s);
    const int w[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
    const Dec16 d{0x4380u, 257.0f};  // base 2^8
#pragma unroll
    for (int e = 0; e < 6; e++) {
      const float2 f = dec_pair(w[lane0 + e], d);
      u[(e / 3) + 3 * (e % 3)] = Cx<R>((R)f.x, (R)f.y);
    }
    su3_third_row(u);
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
  float scale;       // base 2^(8+k) of the global power-of-two scale
  static size_t bytes(int64_t V) { return (sizeof(int4) * 8 + sizeof(int2) * 2) * V; }
  template <typename R> LMB_D void load(int blk, int64_t s, R *a) const {
    const Dec16 d = dec16_of_base(scale);
#pragma unroll
    for (int k = 0; k < 4; k++) {
      int4 t = __ldg(data + (blk * 4 + k) * V + s);
      const int w[4] = {t.x, t.y, t.z, t.w};
#pragma unroll
      for (int j = 0; j < 4; j++) {
        const float2 f = dec_pair(w[j], d);
        a[8 * k + 2 * j] = (R)f.x;
        a[8 * k + 2 * j + 1] = (R)f.y;
      }
    }
    int2 t = __ldg(tail + blk * V + s);
    const float2 f0 = dec_pair(t.x, d), f1 = dec_pair(t.y, d);
    a[32] = (R)f0.x;
    a[33] = (R)f0.y;
    a[34] = (R)f1.x;
    a[35] = (R)f1.y;
  }
};

// ---------------------------------------------------------------------------
// deterministic grid reduction of N doubles: each block reduces its values,
// thread 0 stores them in partials[N * block], the last block to arrive sums
// all partials in block order and returns true (others false).
// ---------------------------------------------------------------------------
template <int NT, int N>
LMB_D bool grid_reduce_slots(double (&v)[N], double *partials, unsigned *counter, double (&total)[N],
                             unsigned slot, unsigned nslots);

template <int NT, int N>
LMB_D bool grid_reduce(double (&v)[N], double *partials, unsigned *counter, double (&total)[N]) {
  return grid_reduce_slots<NT, N>(v, partials, counter, total, blockIdx.x, gridDim.x);
}

// as grid_reduce, for `nslots` cooperating blocks of which this is `slot`
template <int NT, int N>
LMB_D bool grid_reduce_slots(double (&v)[N], double *partials, unsigned *counter, double (&total)[N],
                             unsigned slot, unsigned nslots) {
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
      partials[(size_t)N * slot + n] = x;
    }
    __threadfence();
    unsigned ticket = atomicAdd(counter, 1u);
    last = (ticket == nslots - 1);
  }
  __syncthreads();
  if (!last) return false;
  __threadfence();
#pragma unroll
  for (int n = 0; n < N; n++) {
    double x = 0;
    for (unsigned b = threadIdx.x; b < nslots; b += NT)
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
