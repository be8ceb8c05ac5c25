// lmb_pair.cuh -- two lattice sites per thread in packed FP32.
//
// sm_100 executes FP32 adds, multiplies and fused multiply-adds on register
// pairs (FADD2 / FMUL2 / FFMA2: one instruction, two independent lanes).  The
// FP32 stencils are bound by instruction issue, not by HBM, so a thread works
// on two sites at once, s and s + V/2 (the same x, y, z, t and t + T/2): every
// arithmetic step of the stencil is identical for the two sites, and each
// packed instruction does it for both.  No lane ever needs the other lane's
// value, so nothing is shuffled; the memory accesses of the two lanes are two
// fully coalesced loads from the two halves of every plane.
//
// Here: float2 operators, Cx<float2> products with explicit FFMA2 chains,
// and two-site loads / stores for every FP32 and int16 storage format of
// lmb_common.cuh (lane x = site s0, lane y = site s1).
#pragma once
#include "lmb_common.cuh"

// float2 arithmetic lives in the global namespace, float2's own, so that the
// generic Cx<R> templates find it by argument-dependent lookup
LMB_D float2 operator+(float2 a, float2 b) { return __fadd2_rn(a, b); }
LMB_D float2 operator-(float2 a) { return make_float2(-a.x, -a.y); }
LMB_D float2 operator-(float2 a, float2 b) { return __fadd2_rn(a, -b); }
LMB_D float2 operator*(float2 a, float2 b) { return __fmul2_rn(a, b); }
// double2: two scalar FP64 operations (the FP64 two-site stencils pair the
// sites for their 256-bit loads; FP64 has no packed arithmetic)
LMB_D double2 operator+(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
LMB_D double2 operator-(double2 a) { return make_double2(-a.x, -a.y); }
LMB_D double2 operator-(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
LMB_D double2 operator*(double2 a, double2 b) { return make_double2(a.x * b.x, a.y * b.y); }

namespace lmb {

typedef Cx<float2> Cx2;

LMB_D float2 f2(float a) { return make_float2(a, a); }
LMB_D float2 f2(float a, float b) { return make_float2(a, b); }
LMB_D float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }

LMB_D Cx2 cx2_zero() { return Cx2(f2(0.f), f2(0.f)); }

typedef Cx<double2> Cd2;
LMB_D double2 d2(double a) { return make_double2(a, a); }
LMB_D double2 d2(double a, double b) { return make_double2(a, b); }
LMB_D double2 fmad2(double2 a, double2 b, double2 c) { return make_double2(fma(a.x, b.x, c.x), fma(a.y, b.y, c.y)); }
LMB_D Cd2 cd2_zero() { return Cd2(d2(0.0), d2(0.0)); }

// a * b
LMB_D Cx2 operator*(Cx2 a, Cx2 b) {
  return Cx2(fma2(-a.im, b.im, a.re * b.re), fma2(a.im, b.re, a.re * b.im));
}
// acc + a * b
LMB_D Cx2 cfma(Cx2 a, Cx2 b, Cx2 acc) {
  acc.re = fma2(a.re, b.re, acc.re);
  acc.re = fma2(-a.im, b.im, acc.re);
  acc.im = fma2(a.re, b.im, acc.im);
  acc.im = fma2(a.im, b.re, acc.im);
  return acc;
}
// acc + conj(a) * b
LMB_D Cx2 cfma_conj(Cx2 a, Cx2 b, Cx2 acc) {
  acc.re = fma2(a.re, b.re, acc.re);
  acc.re = fma2(a.im, b.im, acc.re);
  acc.im = fma2(a.re, b.im, acc.im);
  acc.im = fma2(-a.im, b.re, acc.im);
  return acc;
}
// o - k * a  (k real)
LMB_D Cx2 cfms_real(float2 k, Cx2 a, Cx2 o) { return Cx2(fma2(-k, a.re, o.re), fma2(-k, a.im, o.im)); }
// acc + |a|^2 per lane
LMB_D float2 norm2_acc(Cx2 a, float2 acc) { return fma2(a.im, a.im, fma2(a.re, a.re, acc)); }

// U h and U^+ h on both colour vectors of a half spinor (u column-major)
LMB_D void su3_mul_half(const Cx2 *u, const Cx2 *h, Cx2 *o) {
#pragma unroll
  for (int half = 0; half < 2; half++)
#pragma unroll
    for (int r = 0; r < 3; r++) {
      Cx2 v = u[r] * h[3 * half];
      v = cfma(u[r + 3], h[3 * half + 1], v);
      o[r + 3 * half] = cfma(u[r + 6], h[3 * half + 2], v);
    }
}
LMB_D void su3_adj_mul_half(const Cx2 *u, const Cx2 *h, Cx2 *o) {
#pragma unroll
  for (int half = 0; half < 2; half++)
#pragma unroll
    for (int r = 0; r < 3; r++) {
      const Cx2 a = u[3 * r], b = h[3 * half];
      Cx2 v(fma2(a.im, b.im, a.re * b.re), fma2(-a.im, b.re, a.re * b.im));
      v = cfma_conj(u[3 * r + 1], h[3 * half + 1], v);
      o[r + 3 * half] = cfma_conj(u[3 * r + 2], h[3 * half + 2], v);
    }
}

// row 2 = conj(row0 x row1) as FFMA2 chains: conj(a d - b c) per entry
LMB_D Cx2 conj_cross(Cx2 a, Cx2 d, Cx2 b, Cx2 c) {
  // re(a d - b c) and -im(a d - b c)
  const float2 re = fma2(a.re, d.re, fma2(-a.im, d.im, fma2(-b.re, c.re, b.im * c.im)));
  const float2 nim = fma2(-a.re, d.im, fma2(-a.im, d.re, fma2(b.re, c.im, b.im * c.re)));
  return Cx2(re, nim);
}
LMB_D void su3_third_row(Cx2 *u) {
  u[2] = conj_cross(u[3], u[7], u[6], u[4]);
  u[5] = conj_cross(u[6], u[1], u[0], u[7]);
  u[8] = conj_cross(u[0], u[4], u[3], u[1]);
}

// ---------------------------------------------------------------------------
// int16 codec on pairs (format of Field<PREC_HALF>: value = q 2^(e-15) with
// u = q + 32768 in the low 16 bits of a word half, base 2^(8+e) per site)
// ---------------------------------------------------------------------------
// the two int16 halves of words w0 (site s0) and w1 (site s1) with bases
// whose high 16 bits are y0, y1 and negc = -base (1 + 2^-8) per lane
LMB_D Cx2 dec_pair2(int w0, int w1, unsigned y0, unsigned y1, float2 negc) {
  const float2 lo = make_float2(__uint_as_float(__byte_perm((unsigned)w0, y0, 0x5410u)),
                                __uint_as_float(__byte_perm((unsigned)w1, y1, 0x5410u)));
  const float2 hi = make_float2(__uint_as_float(__byte_perm((unsigned)w0, y0, 0x5432u)),
                                __uint_as_float(__byte_perm((unsigned)w1, y1, 0x5432u)));
  return Cx2(lo + negc, hi + negc);
}

// The same two words without the offset subtraction: the floats hold
// value + c, c = base (1 + 2^-8) of the word's site (see project_raw)
LMB_D Cx2 raw_pair2(int w0, int w1, unsigned y0, unsigned y1) {
  return Cx2(make_float2(__uint_as_float(__byte_perm((unsigned)w0, y0, 0x5410u)),
                         __uint_as_float(__byte_perm((unsigned)w1, y1, 0x5410u))),
             make_float2(__uint_as_float(__byte_perm((unsigned)w0, y0, 0x5432u)),
                         __uint_as_float(__byte_perm((unsigned)w1, y1, 0x5432u))));
}

// Encoding exponent of a site: the smallest e with m (1 + 2^-15) < 2^e, so
// that |v| 2^(15-e) < 32768 / (1 + 2^-15) and rint() of it never exceeds
// 32767: no clamp is needed.  e is clamped to [-100, 110]: a site whose
// largest component is below about 2^-115 is stored as zeros.
LMB_D int enc_exponent(float m) {
  const float mm = m * 1.000030517578125f;
  int e = (int)((__float_as_uint(mm) >> 23) & 0xffu) - 126;
  e = e < -100 ? -100 : e;
  return e > 110 ? 110 : e;
}
LMB_D float enc_inv(int e) { return __uint_as_float((unsigned)(142 - e) << 23); }   // 2^(15-e)
LMB_D float enc_base(int e) { return __uint_as_float((unsigned)(135 + e) << 23); }  // 2^(8+e)

// q + 2^23 + 2^15 rounded to an integer: its low 16 mantissa bits are u
LMB_D int enc_word(float re_q, float im_q) {
  return (int)__byte_perm(__float_as_uint(re_q), __float_as_uint(im_q), 0x5410u);
}

// ---------------------------------------------------------------------------
// two-site loads and stores
// ---------------------------------------------------------------------------
template <int NC>
LMB_D void load2(const Field<PREC_HALF, NC> &f, int64_t s0, int64_t s1, Cx2 *v) {
  const float b0 = __ldg(f.norm + s0), b1 = __ldg(f.norm + s1);
  const unsigned y0 = __float_as_uint(b0) >> 16, y1 = __float_as_uint(b1) >> 16;
  const float2 negc = make_float2(-b0 * 1.00390625f, -b1 * 1.00390625f);
  constexpr int P = Field<PREC_HALF, NC>::kPlanes;
#pragma unroll
  for (int k = 0; k < P; k++) {
    const int4 t0 = __ldg(f.data + k * f.V + s0), t1 = __ldg(f.data + k * f.V + s1);
    const int w0[4] = {t0.x, t0.y, t0.z, t0.w}, w1[4] = {t1.x, t1.y, t1.z, t1.w};
#pragma unroll
    for (int j = 0; j < 4; j++)
      if (4 * k + j < NC) v[4 * k + j] = dec_pair2(w0[j], w1[j], y0, y1, negc);
  }
}

template <int NC>
LMB_D void store2(const Field<PREC_HALF, NC> &f, int64_t s0, int64_t s1, const Cx2 *v) {
  float m0 = 0.f, m1 = 0.f;
#pragma unroll
  for (int k = 0; k < NC; k++) {
    m0 = fmaxf(m0, fmaxf(fabsf(v[k].re.x), fabsf(v[k].im.x)));
    m1 = fmaxf(m1, fmaxf(fabsf(v[k].re.y), fabsf(v[k].im.y)));
  }
  const int e0 = enc_exponent(m0), e1 = enc_exponent(m1);
  const float2 inv = make_float2(enc_inv(e0), enc_inv(e1));
  const float2 mag = f2(8421376.0f);  // 2^23 + 2^15
  constexpr int P = Field<PREC_HALF, NC>::kPlanes;
#pragma unroll
  for (int k = 0; k < P; k++) {
    int w0[4], w1[4];
#pragma unroll
    for (int j = 0; j < 4; j++) {
      if (4 * k + j < NC) {
        const float2 qr = fma2(v[4 * k + j].re, inv, mag), qi = fma2(v[4 * k + j].im, inv, mag);
        w0[j] = enc_word(qr.x, qi.x);
        w1[j] = enc_word(qr.y, qi.y);
      } else {
        w0[j] = w1[j] = (int)0x80008000u;  // q = 0
      }
    }
    f.data[k * f.V + s0] = make_int4(w0[0], w0[1], w0[2], w0[3]);
    f.data[k * f.V + s1] = make_int4(w1[0], w1[1], w1[2], w1[3]);
  }
  f.norm[s0] = enc_base(e0);
  f.norm[s1] = enc_base(e1);
}

template <int NC>
LMB_D void load2(const Field<PREC_SINGLE, NC> &f, int64_t s0, int64_t s1, Cx2 *v) {
  constexpr int P = Field<PREC_SINGLE, NC>::kPlanes;
#pragma unroll
  for (int k = 0; k < P; k++) {
    const float4 a = __ldg(f.data + k * f.V + s0), b = __ldg(f.data + k * f.V + s1);
    v[2 * k] = Cx2(f2(a.x, b.x), f2(a.y, b.y));
    if (2 * k + 1 < NC) v[2 * k + 1] = Cx2(f2(a.z, b.z), f2(a.w, b.w));
  }
}

template <int NC>
LMB_D void store2(const Field<PREC_SINGLE, NC> &f, int64_t s0, int64_t s1, const Cx2 *v) {
  constexpr int P = Field<PREC_SINGLE, NC>::kPlanes;
#pragma unroll
  for (int k = 0; k < P; k++) {
    const bool two = 2 * k + 1 < NC;
    f.data[k * f.V + s0] = make_float4(v[2 * k].re.x, v[2 * k].im.x, two ? v[2 * k + 1].re.x : 0.f,
                                       two ? v[2 * k + 1].im.x : 0.f);
    f.data[k * f.V + s1] = make_float4(v[2 * k].re.y, v[2 * k].im.y, two ? v[2 * k + 1].re.y : 0.f,
                                       two ? v[2 * k + 1].im.y : 0.f);
  }
}

// links: 18 reals
LMB_D void load2(const Gauge<PREC_SINGLE> &U, int mu, int64_t s0, int64_t s1, Cx2 *u) {
#pragma unroll
  for (int k = 0; k < 4; k++) {
    const float4 a = __ldg(U.data + (mu * 4 + k) * U.V + s0), b = __ldg(U.data + (mu * 4 + k) * U.V + s1);
    u[2 * k] = Cx2(f2(a.x, b.x), f2(a.y, b.y));
    u[2 * k + 1] = Cx2(f2(a.z, b.z), f2(a.w, b.w));
  }
  const float2 a = __ldg(U.last() + mu * U.V + s0), b = __ldg(U.last() + mu * U.V + s1);
  u[8] = Cx2(f2(a.x, b.x), f2(a.y, b.y));
}
LMB_D void load2(const Gauge<PREC_HALF> &U, int mu, int64_t s0, int64_t s1, Cx2 *u) {
  const unsigned y = __float_as_uint(U.scale) >> 16;
  const float2 negc = f2(-U.scale * 1.00390625f);
#pragma unroll
  for (int k = 0; k < 9; k++)
    u[k] = dec_pair2(__ldg(U.data + (mu * 9 + k) * U.V + s0), __ldg(U.data + (mu * 9 + k) * U.V + s1), y, y,
                     negc);
}
// links: 12 reals, third row rebuilt
LMB_D void load2(const Gauge12<PREC_SINGLE> &U, int mu, int64_t s0, int64_t s1, Cx2 *u) {
#pragma unroll
  for (int k = 0; k < 3; k++) {
    const float4 a = __ldg(U.data + (mu * 3 + k) * U.V + s0), b = __ldg(U.data + (mu * 3 + k) * U.V + s1);
    const int e0 = 2 * k, e1 = 2 * k + 1;
    u[(e0 / 3) + 3 * (e0 % 3)] = Cx2(f2(a.x, b.x), f2(a.y, b.y));
    u[(e1 / 3) + 3 * (e1 % 3)] = Cx2(f2(a.z, b.z), f2(a.w, b.w));
  }
  su3_third_row(u);
}
LMB_D void load2(const Gauge12<PREC_HALF> &U, int mu, int64_t s0, int64_t s1, Cx2 *u) {
  const int q0 = mu * 6, p0 = q0 >> 2, lane0 = q0 & 3;
  const int4 a0 = __ldg(U.data + p0 * U.V + s0), b0 = __ldg(U.data + (p0 + 1) * U.V + s0);
  const int4 a1 = __ldg(U.data + p0 * U.V + s1), b1 = __ldg(U.data + (p0 + 1) * U.V + s1);
  const int w0[8] = {a0.x, a0.y, a0.z, a0.w, b0.x, b0.y, b0.z, b0.w};
  const int w1[8] = {a1.x, a1.y, a1.z, a1.w, b1.x, b1.y, b1.z, b1.w};
  const float2 negc = f2(-257.0f);  // base 2^8
#pragma unroll
  for (int e = 0; e < 6; e++)
    u[(e / 3) + 3 * (e % 3)] = dec_pair2(w0[lane0 + e], w1[lane0 + e], 0x4380u, 0x4380u, negc);
  su3_third_row(u);
}

// clover blocks (36 reals per block)
LMB_D void load2(const Clover<PREC_SINGLE> &A, int blk, int64_t s0, int64_t s1, float2 *a) {
#pragma unroll
  for (int k = 0; k < 9; k++) {
    const float4 x = __ldg(A.data + (blk * 9 + k) * A.V + s0), y = __ldg(A.data + (blk * 9 + k) * A.V + s1);
    a[4 * k] = f2(x.x, y.x);
    a[4 * k + 1] = f2(x.y, y.y);
    a[4 * k + 2] = f2(x.z, y.z);
    a[4 * k + 3] = f2(x.w, y.w);
  }
}
LMB_D void load2(const Clover<PREC_HALF> &A, int blk, int64_t s0, int64_t s1, float2 *a) {
  const unsigned y = __float_as_uint(A.scale) >> 16;
  const float2 negc = f2(-A.scale * 1.00390625f);
#pragma unroll
  for (int k = 0; k < 4; k++) {
    const int4 t0 = __ldg(A.data + (blk * 4 + k) * A.V + s0), t1 = __ldg(A.data + (blk * 4 + k) * A.V + s1);
    const int w0[4] = {t0.x, t0.y, t0.z, t0.w}, w1[4] = {t1.x, t1.y, t1.z, t1.w};
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const Cx2 v = dec_pair2(w0[j], w1[j], y, y, negc);
      a[8 * k + 2 * j] = v.re;
      a[8 * k + 2 * j + 1] = v.im;
    }
  }
  const int2 t0 = __ldg(A.tail + blk * A.V + s0), t1 = __ldg(A.tail + blk * A.V + s1);
  const Cx2 v0 = dec_pair2(t0.x, t1.x, y, y, negc), v1 = dec_pair2(t0.y, t1.y, y, y, negc);
  a[32] = v0.re;
  a[33] = v0.im;
  a[34] = v1.re;
  a[35] = v1.im;
}

// ---------------------------------------------------------------------------
// adjacent pairs: lanes are sites s and s + 1 (s even).  One 256-bit load
// (sm_100 ld.global.v8) fetches a plane's 16-byte words of both sites; the
// address must be 32-byte aligned, which holds for even s on planes of an
// even number of sites.
// ---------------------------------------------------------------------------
LMB_D void ld256(const int4 *p, int4 &a, int4 &b) {
  asm("ld.global.nc.v8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
      : "=r"(a.x), "=r"(a.y), "=r"(a.z), "=r"(a.w), "=r"(b.x), "=r"(b.y), "=r"(b.z), "=r"(b.w)
      : "l"(p));
}

LMB_D void st256(int4 *p, const int4 &a, const int4 &b) {
  asm volatile("st.global.v8.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};" ::"l"(p), "r"(a.x), "r"(a.y), "r"(a.z),
               "r"(a.w), "r"(b.x), "r"(b.y), "r"(b.z), "r"(b.w)
               : "memory");
}
// 256-bit load of data this kernel also writes (no read-only cache path)
LMB_D void ld256_rw(const int4 *p, int4 &a, int4 &b) {
  asm volatile("ld.global.v8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
               : "=r"(a.x), "=r"(a.y), "=r"(a.z), "=r"(a.w), "=r"(b.x), "=r"(b.y), "=r"(b.z), "=r"(b.w)
               : "l"(p)
               : "memory");
}

// FP64 fields and 18-real links on two sites: x-adjacent (s even, one
// 256-bit load per plane) or arbitrary (two 128-bit loads)
LMB_D void ld256d(const double2 *p, double2 &a, double2 &b) {
  asm("ld.global.nc.v4.f64 {%0,%1,%2,%3}, [%4];" : "=d"(a.x), "=d"(a.y), "=d"(b.x), "=d"(b.y) : "l"(p));
}
template <int NC>
LMB_D void load_adj(const Field<PREC_DOUBLE, NC> &f, int64_t s, Cd2 *v) {
#pragma unroll
  for (int k = 0; k < NC; k++) {
    double2 a, b;
    ld256d(f.data + k * f.V + s, a, b);
    v[k] = Cd2(d2(a.x, b.x), d2(a.y, b.y));
  }
}
template <int NC>
LMB_D void load2(const Field<PREC_DOUBLE, NC> &f, int64_t s0, int64_t s1, Cd2 *v) {
#pragma unroll
  for (int k = 0; k < NC; k++) {
    const double2 a = __ldg(f.data + k * f.V + s0), b = __ldg(f.data + k * f.V + s1);
    v[k] = Cd2(d2(a.x, b.x), d2(a.y, b.y));
  }
}
LMB_D void load_adj(const Gauge<PREC_DOUBLE> &U, int mu, int64_t s, Cd2 *u) {
#pragma unroll
  for (int k = 0; k < 9; k++) {
    double2 a, b;
    ld256d(U.data + (mu * 9 + k) * U.V + s, a, b);
    u[k] = Cd2(d2(a.x, b.x), d2(a.y, b.y));
  }
}
LMB_D void load2(const Gauge<PREC_DOUBLE> &U, int mu, int64_t s0, int64_t s1, Cd2 *u) {
#pragma unroll
  for (int k = 0; k < 9; k++) {
    const double2 a = __ldg(U.data + (mu * 9 + k) * U.V + s0), b = __ldg(U.data + (mu * 9 + k) * U.V + s1);
    u[k] = Cd2(d2(a.x, b.x), d2(a.y, b.y));
  }
}

// own-site fields of the epilogues (read and written by the same kernel)
template <int NC>
LMB_D void load_adj_rw(const Field<PREC_HALF, NC> &f, int64_t s, Cx2 *v) {
  const float2 nb = *reinterpret_cast<const float2 *>(f.norm + s);
  const unsigned y0 = __float_as_uint(nb.x) >> 16, y1 = __float_as_uint(nb.y) >> 16;
  const float2 negc = make_float2(-nb.x * 1.00390625f, -nb.y * 1.00390625f);
  constexpr int P = Field<PREC_HALF, NC>::kPlanes;
#pragma unroll
  for (int k = 0; k < P; k++) {
    int4 t0, t1;
    ld256_rw(f.data + k * f.V + s, t0, t1);
    const int w0[4] = {t0.x, t0.y, t0.z, t0.w}, w1[4] = {t1.x, t1.y, t1.z, t1.w};
#pragma unroll
    for (int j = 0; j < 4; j++)
      if (4 * k + j < NC) v[4 * k + j] = dec_pair2(w0[j], w1[j], y0, y1, negc);
  }
}
template <int NC>
LMB_D void load_adj_rw(const Field<PREC_SINGLE, NC> &f, int64_t s, Cx2 *v) {
  constexpr int P = Field<PREC_SINGLE, NC>::kPlanes;
#pragma unroll
  for (int k = 0; k < P; k++) {
    int4 ia, ib;
    ld256_rw(reinterpret_cast<const int4 *>(f.data + k * f.V + s), ia, ib);
    const float4 a = *reinterpret_cast<const float4 *>(&ia), b = *reinterpret_cast<const float4 *>(&ib);
    v[2 * k] = Cx2(f2(a.x, b.x), f2(a.y, b.y));
    if (2 * k + 1 < NC) v[2 * k + 1] = Cx2(f2(a.z, b.z), f2(a.w, b.w));
  }
}
template <int NC>
LMB_D void store_adj(const Field<PREC_HALF, NC> &f, int64_t s, const Cx2 *v) {
  float m0 = 0.f, m1 = 0.f;
#pragma unroll
  for (int k = 0; k < NC; k++) {
    m0 = fmaxf(m0, fmaxf(fabsf(v[k].re.x), fabsf(v[k].im.x)));
    m1 = fmaxf(m1, fmaxf(fabsf(v[k].re.y), fabsf(v[k].im.y)));
  }
  const int e0 = enc_exponent(m0), e1 = enc_exponent(m1);
  const float2 inv = make_float2(enc_inv(e0), enc_inv(e1));
  const float2 mag = f2(8421376.0f);  // 2^23 + 2^15
  constexpr int P = Field<PREC_HALF, NC>::kPlanes;
#pragma unroll
  for (int k = 0; k < P; k++) {
    int w0[4], w1[4];
#pragma unroll
    for (int j = 0; j < 4; j++) {
      if (4 * k + j < NC) {
        const float2 qr = fma2(v[4 * k + j].re, inv, mag), qi = fma2(v[4 * k + j].im, inv, mag);
        w0[j] = enc_word(qr.x, qi.x);
        w1[j] = enc_word(qr.y, qi.y);
      } else {
        w0[j] = w1[j] = (int)0x80008000u;  // q = 0
      }
    }
    st256(f.data + k * f.V + s, make_int4(w0[0], w0[1], w0[2], w0[3]), make_int4(w1[0], w1[1], w1[2], w1[3]));
  }
  *reinterpret_cast<float2 *>(f.norm + s) = make_float2(enc_base(e0), enc_base(e1));
}
template <int NC>
LMB_D void store_adj(const Field<PREC_SINGLE, NC> &f, int64_t s, const Cx2 *v) {
  constexpr int P = Field<PREC_SINGLE, NC>::kPlanes;
#pragma unroll
  for (int k = 0; k < P; k++) {
    const bool two = 2 * k + 1 < NC;
    const float4 a = make_float4(v[2 * k].re.x, v[2 * k].im.x, two ? v[2 * k + 1].re.x : 0.f,
                                 two ? v[2 * k + 1].im.x : 0.f);
    const float4 b = make_float4(v[2 * k].re.y, v[2 * k].im.y, two ? v[2 * k + 1].re.y : 0.f,
                                 two ? v[2 * k + 1].im.y : 0.f);
    st256(reinterpret_cast<int4 *>(f.data + k * f.V + s), *reinterpret_cast<const int4 *>(&a),
          *reinterpret_cast<const int4 *>(&b));
  }
}

// raw words (value + c per lane) of the two sites s, s + 1 (s even) and of
// two arbitrary sites; nc2 = -2c per lane
template <int NC>
LMB_D void load_adj_raw(const Field<PREC_HALF, NC> &f, int64_t s, Cx2 *v, float2 &nc2) {
  const float2 nb = __ldg(reinterpret_cast<const float2 *>(f.norm + s));
  const unsigned y0 = __float_as_uint(nb.x) >> 16, y1 = __float_as_uint(nb.y) >> 16;
  nc2 = make_float2(-nb.x * 2.0078125f, -nb.y * 2.0078125f);
  constexpr int P = Field<PREC_HALF, NC>::kPlanes;
#pragma unroll
  for (int k = 0; k < P; k++) {
    int4 t0, t1;
    ld256(f.data + k * f.V + s, t0, t1);
    const int w0[4] = {t0.x, t0.y, t0.z, t0.w}, w1[4] = {t1.x, t1.y, t1.z, t1.w};
#pragma unroll
    for (int j = 0; j < 4; j++)
      if (4 * k + j < NC) v[4 * k + j] = raw_pair2(w0[j], w1[j], y0, y1);
  }
}
template <int NC>
LMB_D void load2_raw(const Field<PREC_HALF, NC> &f, int64_t s0, int64_t s1, Cx2 *v, float2 &nc2) {
  const float b0 = __ldg(f.norm + s0), b1 = __ldg(f.norm + s1);
  const unsigned y0 = __float_as_uint(b0) >> 16, y1 = __float_as_uint(b1) >> 16;
  nc2 = make_float2(-b0 * 2.0078125f, -b1 * 2.0078125f);
  constexpr int P = Field<PREC_HALF, NC>::kPlanes;
#pragma unroll
  for (int k = 0; k < P; k++) {
    const int4 t0 = __ldg(f.data + k * f.V + s0), t1 = __ldg(f.data + k * f.V + s1);
    const int w0[4] = {t0.x, t0.y, t0.z, t0.w}, w1[4] = {t1.x, t1.y, t1.z, t1.w};
#pragma unroll
    for (int j = 0; j < 4; j++)
      if (4 * k + j < NC) v[4 * k + j] = raw_pair2(w0[j], w1[j], y0, y1);
  }
}

template <int NC>
LMB_D void load_adj(const Field<PREC_HALF, NC> &f, int64_t s, Cx2 *v) {
  const float2 nb = __ldg(reinterpret_cast<const float2 *>(f.norm + s));
  const unsigned y0 = __float_as_uint(nb.x) >> 16, y1 = __float_as_uint(nb.y) >> 16;
  const float2 negc = make_float2(-nb.x * 1.00390625f, -nb.y * 1.00390625f);
  constexpr int P = Field<PREC_HALF, NC>::kPlanes;
#pragma unroll
  for (int k = 0; k < P; k++) {
    int4 t0, t1;
    ld256(f.data + k * f.V + s, t0, t1);
    const int w0[4] = {t0.x, t0.y, t0.z, t0.w}, w1[4] = {t1.x, t1.y, t1.z, t1.w};
#pragma unroll
    for (int j = 0; j < 4; j++)
      if (4 * k + j < NC) v[4 * k + j] = dec_pair2(w0[j], w1[j], y0, y1, negc);
  }
}
LMB_D void load_adj(const Gauge12<PREC_HALF> &U, int mu, int64_t s, Cx2 *u) {
  const int q0 = mu * 6, p0 = q0 >> 2, lane0 = q0 & 3;
  int4 a0, a1, b0, b1;
  ld256(U.data + p0 * U.V + s, a0, a1);
  ld256(U.data + (p0 + 1) * U.V + s, b0, b1);
  const int w0[8] = {a0.x, a0.y, a0.z, a0.w, b0.x, b0.y, b0.z, b0.w};
  const int w1[8] = {a1.x, a1.y, a1.z, a1.w, b1.x, b1.y, b1.z, b1.w};
  const float2 negc = f2(-257.0f);  // base 2^8
#pragma unroll
  for (int e = 0; e < 6; e++)
    u[(e / 3) + 3 * (e % 3)] = dec_pair2(w0[lane0 + e], w1[lane0 + e], 0x4380u, 0x4380u, negc);
  su3_third_row(u);
}
LMB_D void load_adj(const Clover<PREC_HALF> &A, int blk, int64_t s, float2 *a) {
  const unsigned y = __float_as_uint(A.scale) >> 16;
  const float2 negc = f2(-A.scale * 1.00390625f);
#pragma unroll
  for (int k = 0; k < 4; k++) {
    int4 t0, t1;
    ld256(A.data + (blk * 4 + k) * A.V + s, t0, t1);
    const int w0[4] = {t0.x, t0.y, t0.z, t0.w}, w1[4] = {t1.x, t1.y, t1.z, t1.w};
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const Cx2 v = dec_pair2(w0[j], w1[j], y, y, negc);
      a[8 * k + 2 * j] = v.re;
      a[8 * k + 2 * j + 1] = v.im;
    }
  }
  // the two sites' int2 tails are one 16-byte word
  const int4 t = __ldg(reinterpret_cast<const int4 *>(A.tail + blk * A.V + s));
  const Cx2 v0 = dec_pair2(t.x, t.z, y, y, negc), v1 = dec_pair2(t.y, t.w, y, y, negc);
  a[32] = v0.re;
  a[33] = v0.im;
  a[34] = v1.re;
  a[35] = v1.im;
}

// 18-real int16 links (one (re, im) int32 word per entry, global scale),
// adjacent pairs: one 64-bit load per entry
LMB_D void load_adj(const Gauge<PREC_HALF> &U, int mu, int64_t s, Cx2 *u) {
  const unsigned y = __float_as_uint(U.scale) >> 16;
  const float2 negc = f2(-U.scale * 1.00390625f);
#pragma unroll
  for (int k = 0; k < 9; k++) {
    const int2 t = __ldg(reinterpret_cast<const int2 *>(U.data + (mu * 9 + k) * U.V + s));
    u[k] = dec_pair2(t.x, t.y, y, y, negc);
  }
}

// 3-component FP32 fields (float4 plane + float2 plane) and 18-real FP32
// links (four float4 planes + one float2 plane per direction), adjacent pairs
LMB_D float4 as_f4(const int4 &v) { return make_float4(__int_as_float(v.x), __int_as_float(v.y), __int_as_float(v.z), __int_as_float(v.w)); }
LMB_D int4 as_i4(const float4 &v) { return make_int4(__float_as_int(v.x), __float_as_int(v.y), __float_as_int(v.z), __float_as_int(v.w)); }

LMB_D void load_adj(const Field<PREC_SINGLE, 3> &f, int64_t s, Cx2 *v) {
  int4 ia, ib;
  ld256(reinterpret_cast<const int4 *>(f.data + s), ia, ib);
  const float4 a = as_f4(ia), b = as_f4(ib);
  const float4 c = __ldg(reinterpret_cast<const float4 *>(f.last() + s));  // (s).xy, (s + 1).xy
  v[0] = Cx2(f2(a.x, b.x), f2(a.y, b.y));
  v[1] = Cx2(f2(a.z, b.z), f2(a.w, b.w));
  v[2] = Cx2(f2(c.x, c.z), f2(c.y, c.w));
}
LMB_D void load_adj_rw(const Field<PREC_SINGLE, 3> &f, int64_t s, Cx2 *v) {
  int4 ia, ib;
  ld256_rw(reinterpret_cast<const int4 *>(f.data + s), ia, ib);
  const float4 a = as_f4(ia), b = as_f4(ib);
  const float4 c = *reinterpret_cast<const float4 *>(f.last() + s);
  v[0] = Cx2(f2(a.x, b.x), f2(a.y, b.y));
  v[1] = Cx2(f2(a.z, b.z), f2(a.w, b.w));
  v[2] = Cx2(f2(c.x, c.z), f2(c.y, c.w));
}
LMB_D void store_adj(const Field<PREC_SINGLE, 3> &f, int64_t s, const Cx2 *v) {
  st256(reinterpret_cast<int4 *>(f.data + s), as_i4(make_float4(v[0].re.x, v[0].im.x, v[1].re.x, v[1].im.x)),
        as_i4(make_float4(v[0].re.y, v[0].im.y, v[1].re.y, v[1].im.y)));
  *reinterpret_cast<float4 *>(f.last() + s) = make_float4(v[2].re.x, v[2].im.x, v[2].re.y, v[2].im.y);
}
// two arbitrary sites
LMB_D void load2(const Field<PREC_SINGLE, 3> &f, int64_t s0, int64_t s1, Cx2 *v) {
  const float4 a = __ldg(f.data + s0), b = __ldg(f.data + s1);
  const float2 c = __ldg(f.last() + s0), d = __ldg(f.last() + s1);
  v[0] = Cx2(f2(a.x, b.x), f2(a.y, b.y));
  v[1] = Cx2(f2(a.z, b.z), f2(a.w, b.w));
  v[2] = Cx2(f2(c.x, d.x), f2(c.y, d.y));
}
LMB_D void load_adj(const Gauge<PREC_SINGLE> &U, int mu, int64_t s, Cx2 *u) {
#pragma unroll
  for (int k = 0; k < 4; k++) {
    int4 ia, ib;
    ld256(reinterpret_cast<const int4 *>(U.data + (mu * 4 + k) * U.V + s), ia, ib);
    const float4 a = as_f4(ia), b = as_f4(ib);
    u[2 * k] = Cx2(f2(a.x, b.x), f2(a.y, b.y));
    u[2 * k + 1] = Cx2(f2(a.z, b.z), f2(a.w, b.w));
  }
  const float4 c = __ldg(reinterpret_cast<const float4 *>(U.last() + mu * U.V + s));
  u[8] = Cx2(f2(c.x, c.z), f2(c.y, c.w));
}

// o += A v, A Hermitian 6x6 (6 real diagonal, 15 complex lower entries)
LMB_D void herm6_mul_acc(const float2 *a, const Cx2 *v, Cx2 *o) {
#pragma unroll
  for (int i = 0; i < 6; i++) o[i] = Cx2(fma2(a[i], v[i].re, o[i].re), fma2(a[i], v[i].im, o[i].im));
  int k = 6;
#pragma unroll
  for (int i = 1; i < 6; i++)
#pragma unroll
    for (int j = 0; j < i; j++) {
      const Cx2 aij(a[k], a[k + 1]);
      o[i] = cfma(aij, v[j], o[i]);
      o[j] = cfma_conj(aij, v[i], o[j]);
      k += 2;
    }
}

// Hermitian 6x6 (6 real diagonal, 15 complex lower entries) times a 6-vector
LMB_D void herm6_mul(const float2 *a, const Cx2 *v, Cx2 *o) {
#pragma unroll
  for (int i = 0; i < 6; i++) o[i] = Cx2(a[i] * v[i].re, a[i] * v[i].im);
  int k = 6;
#pragma unroll
  for (int i = 1; i < 6; i++)
#pragma unroll
    for (int j = 0; j < i; j++) {
      const Cx2 aij(a[k], a[k + 1]);
      o[i] = cfma(aij, v[j], o[i]);
      o[j] = cfma_conj(aij, v[i], o[j]);
      k += 2;
    }
}

}  // namespace lmb
