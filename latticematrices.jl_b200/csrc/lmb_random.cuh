// lmb_random.cuh -- seeded synthetic inputs on the GPU.
//
// Philox4x32-10 counter-based generator (Salmon, Moraes, Dror and Shaw,
// "Parallel random numbers: as easy as 1, 2, 3", SC 2011), the generator
// family of the reference's decomposition-independent site streams
// (utilities/randomgenerator.jl:247-340).  The counter is (global site, lane,
// draw, tag), so every field depends only on the seed and the global site
// index, not on the launch shape.
//  * links: U_mu(x) = reunitarize(exp(i a H)), H traceless Hermitian with
//    N(0,1) diagonal (minus its mean) and (N + iN)/sqrt(2) off-diagonal;
//    exp by scaling and squaring of a degree-16 Taylor polynomial;
//    reunitarize = Gram-Schmidt of rows 1, 2 and row 3 = conj(row1 x row2)
//    (linearalgebra_D.jl:2371-2424).
//  * sources: complex Gaussian with re, im ~ N(0, 1/2)
//    (benchmark/ddagd_cg/README.md:161-162).
#pragma once
#include "lmb_pack.cuh"

namespace lmb {

LMB_D void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
#pragma unroll
  for (int r = 0; r < 10; r++) {
    const uint32_t lo0 = 0xD2511F53u * c[0], hi0 = __umulhi(0xD2511F53u, c[0]);
    const uint32_t lo1 = 0xCD9E8D57u * c[2], hi1 = __umulhi(0xCD9E8D57u, c[2]);
    const uint32_t n0 = hi1 ^ c[1] ^ k0, n2 = hi0 ^ c[3] ^ k1;
    c[0] = n0;
    c[1] = lo1;
    c[2] = n2;
    c[3] = lo0;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
}

LMB_D void philox_normals(uint32_t site, uint32_t lane, uint32_t draw, uint32_t tag, uint64_t seed,
                          double *g) {
  uint32_t c[4] = {site, lane, draw, tag};
  philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32) ^ 0x4C4D4232u);
  const double u1 = ((double)(c[0] >> 5) * 67108864.0 + (double)(c[1] >> 6) + 0.5) / 9007199254740992.0;
  const double u2 = ((double)(c[2] >> 5) * 67108864.0 + (double)(c[3] >> 6) + 0.5) / 9007199254740992.0;
  const double rad = sqrt(-2.0 * log(u1));
  double sn, cs;
  sincospi(2.0 * u2, &sn, &cs);
  g[0] = rad * cs;
  g[1] = rad * sn;
}

LMB_D void expm3_taylor(const Cx<double> *M, Cx<double> *E) {
  double nrm = 0;
#pragma unroll
  for (int k = 0; k < 9; k++) nrm += norm2(M[k]);
  nrm = sqrt(nrm);
  int sq = 0;
  while (nrm > 0.125) {
    nrm *= 0.5;
    sq++;
  }
  const double scale = ldexp(1.0, -sq);
  Cx<double> A[9], term[9];
#pragma unroll
  for (int k = 0; k < 9; k++) {
    A[k] = scale * M[k];
    E[k] = Cx<double>(0, 0);
    term[k] = Cx<double>(0, 0);
  }
#pragma unroll
  for (int k = 0; k < 3; k++) {
    E[k + 3 * k] = Cx<double>(1, 0);
    term[k + 3 * k] = Cx<double>(1, 0);
  }
  for (int n = 1; n <= 16; n++) {
    mat3_mul(term, A, term);
#pragma unroll
    for (int k = 0; k < 9; k++) {
      term[k] = (1.0 / n) * term[k];
      E[k] = E[k] + term[k];
    }
  }
  for (int s = 0; s < sq; s++) mat3_mul(E, E, E);
}

LMB_D void reunitarize3(Cx<double> *u) {
#define UE(r, c) u[(r) + 3 * (c)]
  Cx<double> w1(0, 0);
  double w2 = 0;
  for (int ic = 0; ic < 3; ic++) {
    w1 = w1 + UE(1, ic) * conj(UE(0, ic));
    w2 += norm2(UE(0, ic));
  }
  w1 = (-1.0 / w2) * w1;
  const Cx<double> x4 = UE(1, 0) + w1 * UE(0, 0);
  const Cx<double> x5 = UE(1, 1) + w1 * UE(0, 1);
  const Cx<double> x6 = UE(1, 2) + w1 * UE(0, 2);
  const double w3 = 1.0 / sqrt(norm2(x4) + norm2(x5) + norm2(x6));
  w2 = 1.0 / sqrt(w2);
  UE(1, 0) = w3 * x4;
  UE(1, 1) = w3 * x5;
  UE(1, 2) = w3 * x6;
  for (int ic = 0; ic < 3; ic++) UE(0, ic) = w2 * UE(0, ic);
  UE(2, 0) = conj(UE(0, 1) * UE(1, 2) - UE(0, 2) * UE(1, 1));
  UE(2, 1) = conj(UE(0, 2) * UE(1, 0) - UE(0, 0) * UE(1, 2));
  UE(2, 2) = conj(UE(0, 0) * UE(1, 1) - UE(0, 1) * UE(1, 0));
#undef UE
}

// one thread per (site, mu); writes the padded (3,3,...) link fields
template <typename TOUT>
__global__ void __launch_bounds__(128)
    random_su3_kernel(TOUT *U0, TOUT *U1, TOUT *U2, TOUT *U3, const Geom g, const Padded pd, double amplitude,
                      uint64_t seed) {
  const int64_t tid = (int64_t)blockIdx.x * 128 + threadIdx.x;
  if (tid >= 4 * g.V) return;
  const int mu = (int)(tid % 4);
  const int s = (int)(tid / 4);
  int c[4];
  site_coords(g, s, c);
  // stream counter: the lexicographic site index (single rank: local = global)
  double gn[10];
  for (int d = 0; d < 5; d++) philox_normals((uint32_t)s, (uint32_t)mu, (uint32_t)d, 0x4C4Bu, seed, gn + 2 * d);
  Cx<double> H[9];
  const double mean = (gn[0] + gn[1] + gn[2]) / 3.0;
  H[0] = Cx<double>(gn[0] - mean, 0);
  H[4] = Cx<double>(gn[1] - mean, 0);
  H[8] = Cx<double>(gn[2] - mean, 0);
  const double r2 = 0.70710678118654752440;
  const Cx<double> h01(gn[3] * r2, gn[4] * r2), h02(gn[5] * r2, gn[6] * r2), h12(gn[7] * r2, gn[8] * r2);
  H[3] = h01;
  H[1] = conj(h01);
  H[6] = h02;
  H[2] = conj(h02);
  H[7] = h12;
  H[5] = conj(h12);
  Cx<double> M[9], E[9];
#pragma unroll
  for (int k = 0; k < 9; k++) M[k] = amplitude * mul_i(H[k]);
  expm3_taylor(M, E);
  reunitarize3(E);
  TOUT *U = mu == 0 ? U0 : (mu == 1 ? U1 : (mu == 2 ? U2 : U3));
  TOUT *q = U + padded_site(pd, c) * 9;
#pragma unroll
  for (int k = 0; k < 9; k++) {
    q[k].x = E[k].re;
    q[k].y = E[k].im;
  }
}

template <typename TOUT>
__global__ void __launch_bounds__(256)
    gaussian_field_kernel(TOUT *out, int ncomp, const Geom g, const Padded pd, uint64_t seed) {
  const int s = blockIdx.x * 256 + threadIdx.x;
  if (s >= g.V) return;
  int c[4];
  site_coords(g, s, c);
  TOUT *q = out + padded_site(pd, c) * ncomp;
  const double r2 = 0.70710678118654752440;
  for (int k = 0; k < ncomp; k++) {
    double gn[2];
    philox_normals((uint32_t)s, (uint32_t)k, 0u, 0x5350u, seed, gn);
    q[k].x = gn[0] * r2;
    q[k].y = gn[1] * r2;
  }
}

}  // namespace lmb
