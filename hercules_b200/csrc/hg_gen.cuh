// hg_gen.cuh -- seeded synthetic data series, identical bits on host and GPU.
//
// The reference generator (tools/Cgenerator/generator/main.c:27-65) draws
// N(0,1) steps from GSL, accumulates a float random walk and z-normalises it
// in float with the population standard deviation.  GSL is not available
// and its stream cannot be reproduced, so this generator keeps the walk and
// the normalisation and draws the steps from a counter-based Philox4x32-10
// stream (Salmon et al., SC'11) through Box-Muller.  The logarithm and the
// sine/cosine are evaluated with series built only from correctly rounded
// double +, -, *, / so that the host C++ and the device code give the same
// bits; no libm transcendental is called.
#pragma once

#include "hg_arith.cuh"

namespace hg {

enum : uint32_t { kTagWalk = 0x57414C4Bu, kTagPick = 0x5049434Bu, kTagNoise = 0x4E4F4953u };

HG_HD void philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0, uint32_t k1,
                         uint32_t out[4]) {
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u, W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    uint64_t p0 = (uint64_t)M0 * c0;
    uint64_t p1 = (uint64_t)M1 * c2;
    uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
    c0 = n0;
    c1 = lo1;
    c2 = n2;
    c3 = lo0;
    k0 += W0;
    k1 += W1;
  }
  out[0] = c0;
  out[1] = c1;
  out[2] = c2;
  out[3] = c3;
}

// uniform in (0, 1): (x + 0.5) / 2^32, exact in double
HG_HD double u01(uint32_t x) { return HG_DMUL((double)x + 0.5, 2.3283064365386963e-10); }

// natural log on (0, 1]: x = m 2^e with m in [sqrt(2)/2, sqrt(2)), then
// log m = 2 atanh(s), s = (m-1)/(m+1), as an odd series in s.
HG_HD double det_log(double x) {
  union {
    double d;
    uint64_t u;
  } c;
  c.d = x;
  int e = (int)((c.u >> 52) & 0x7FF) - 1023;
  c.u = (c.u & 0x000FFFFFFFFFFFFFull) | 0x3FF0000000000000ull;  // m in [1, 2)
  double m = c.d;
  if (m > 1.4142135623730951) {
    m = HG_DMUL(m, 0.5);
    e += 1;
  }
  double s = HG_DDIV(HG_DSUB(m, 1.0), HG_DADD(m, 1.0));
  double s2 = HG_DMUL(s, s);
  double p = 1.0 / 23.0;
  p = HG_DADD(HG_DMUL(p, s2), 1.0 / 21.0);
  p = HG_DADD(HG_DMUL(p, s2), 1.0 / 19.0);
  p = HG_DADD(HG_DMUL(p, s2), 1.0 / 17.0);
  p = HG_DADD(HG_DMUL(p, s2), 1.0 / 15.0);
  p = HG_DADD(HG_DMUL(p, s2), 1.0 / 13.0);
  p = HG_DADD(HG_DMUL(p, s2), 1.0 / 11.0);
  p = HG_DADD(HG_DMUL(p, s2), 1.0 / 9.0);
  p = HG_DADD(HG_DMUL(p, s2), 1.0 / 7.0);
  p = HG_DADD(HG_DMUL(p, s2), 1.0 / 5.0);
  p = HG_DADD(HG_DMUL(p, s2), 1.0 / 3.0);
  p = HG_DADD(HG_DMUL(p, s2), 1.0);
  double lm = HG_DMUL(HG_DMUL(2.0, s), p);
  return HG_DADD(HG_DMUL((double)e, 0.6931471805599453), lm);
}

// sin and cos of a in [0, pi/2) by Taylor series (Horner in a^2).
HG_HD void det_sincos_q(double a, double* sn, double* cs) {
  double a2 = HG_DMUL(a, a);
  double s = -1.0 / 1307674368000.0;            // -1/15!
  s = HG_DADD(HG_DMUL(s, a2), 1.0 / 6227020800.0);   // 1/13!
  s = HG_DADD(HG_DMUL(s, a2), -1.0 / 39916800.0);    // -1/11!
  s = HG_DADD(HG_DMUL(s, a2), 1.0 / 362880.0);       // 1/9!
  s = HG_DADD(HG_DMUL(s, a2), -1.0 / 5040.0);        // -1/7!
  s = HG_DADD(HG_DMUL(s, a2), 1.0 / 120.0);          // 1/5!
  s = HG_DADD(HG_DMUL(s, a2), -1.0 / 6.0);           // -1/3!
  s = HG_DADD(HG_DMUL(s, a2), 1.0);
  *sn = HG_DMUL(s, a);
  double c = 1.0 / 20922789888000.0;            // 1/16!
  c = HG_DADD(HG_DMUL(c, a2), -1.0 / 87178291200.0);  // -1/14!
  c = HG_DADD(HG_DMUL(c, a2), 1.0 / 479001600.0);     // 1/12!
  c = HG_DADD(HG_DMUL(c, a2), -1.0 / 3628800.0);      // -1/10!
  c = HG_DADD(HG_DMUL(c, a2), 1.0 / 40320.0);         // 1/8!
  c = HG_DADD(HG_DMUL(c, a2), -1.0 / 720.0);          // -1/6!
  c = HG_DADD(HG_DMUL(c, a2), 1.0 / 24.0);            // 1/4!
  c = HG_DADD(HG_DMUL(c, a2), -0.5);
  *cs = HG_DADD(HG_DMUL(c, a2), 1.0);
}

// Box-Muller pair from two uniforms.
HG_HD void box_muller(uint32_t x1, uint32_t x2, double* z0, double* z1) {
  double r = HG_DSQRT(HG_DMUL(-2.0, det_log(u01(x1))));
  double v = HG_DMUL(u01(x2), 4.0);  // quadrant reduction of 2*pi*u
  int q = (int)v;
  if (q > 3) q = 3;
  double a = HG_DMUL(HG_DSUB(v, (double)q), 1.5707963267948966);
  double sn, cs;
  det_sincos_q(a, &sn, &cs);
  double c, s;
  if (q == 0) { c = cs; s = sn; }
  else if (q == 1) { c = -sn; s = cs; }
  else if (q == 2) { c = -cs; s = -sn; }
  else { c = sn; s = -cs; }
  *z0 = HG_DMUL(r, c);
  *z1 = HG_DMUL(r, s);
}

// Four N(0,1) draws for (stream id, block b) of a stream tagged `tag`.
HG_HD void normal4(uint64_t seed, uint64_t id, uint32_t b, uint32_t tag, double z[4]) {
  uint32_t o[4];
  philox4x32_10((uint32_t)id, (uint32_t)(id >> 32), b, tag, (uint32_t)seed, (uint32_t)(seed >> 32), o);
  box_muller(o[0], o[1], &z[0], &z[1]);
  box_muller(o[2], o[3], &z[2], &z[3]);
}

// z_normalize of tools/Cgenerator/generator/main.c:27-46: float mean, float
// population variance, sqrt, then (x - mean) / std.
HG_HD void znorm(float* ts, int L) {
  float mean = 0.0f;
  for (int i = 0; i < L; ++i) mean = HG_FADD(mean, ts[i]);
  mean = HG_FDIV(mean, (float)L);
  float sd = 0.0f;
  for (int i = 0; i < L; ++i) {
    float d = HG_FSUB(ts[i], mean);
    sd = HG_FADD(sd, HG_FMUL(d, d));
  }
  sd = HG_FDIV(sd, (float)L);
  sd = HG_FSQRT(sd);
  for (int i = 0; i < L; ++i) ts[i] = HG_FDIV(HG_FSUB(ts[i], mean), sd);
}

// Series `id` of the random-walk stream `seed` (L a multiple of 4).
HG_HD void random_walk(uint64_t seed, uint64_t id, int L, float* out) {
  float x = 0.0f;
  for (int b = 0; b < L / 4; ++b) {
    double z[4];
    normal4(seed, id, (uint32_t)b, kTagWalk, z);
    for (int j = 0; j < 4; ++j) {
      x = HG_FADD(x, (float)z[j]);
      out[4 * b + j] = x;
    }
  }
  znorm(out, L);
}

// L2 normalisation in float: sequential sum of squares, sqrt, divide.
HG_HD void l2norm(float* v, int L) {
  float ss = 0.0f;
  for (int i = 0; i < L; ++i) ss = HG_FADD(ss, HG_FMUL(v[i], v[i]));
  const float nrm = HG_FSQRT(ss);
  if (nrm > 0.0f)
    for (int i = 0; i < L; ++i) v[i] = HG_FDIV(v[i], nrm);
}

// Row `id` of the unit-normalised Gaussian stream `seed`: N(0, I) then L2
// normalisation (the short-series vector shape; L a multiple of 4).
HG_HD void gaussian_unit(uint64_t seed, uint64_t id, int L, float* out) {
  for (int b = 0; b < L / 4; ++b) {
    double z[4];
    normal4(seed, id, (uint32_t)b, kTagWalk, z);
    for (int j = 0; j < 4; ++j) out[4 * b + j] = (float)z[j];
  }
  l2norm(out, L);
}

// The dataset row a noisy query starts from.
HG_HD uint64_t pick_row(uint64_t seed, uint64_t qid, uint64_t n) {
  uint32_t o[4];
  philox4x32_10((uint32_t)qid, (uint32_t)(qid >> 32), 0u, kTagPick, (uint32_t)seed, (uint32_t)(seed >> 32), o);
  uint64_t r = ((uint64_t)o[0] << 32) | o[1];
  return r % n;
}

// Query `qid`: dataset row `base` plus N(0, sigma2) noise per point, then
// z-normalised (the workload of the noisy-query configurations).
// unit = 1: L2-normalised instead (queries of the unit-vector shape).
HG_HD void noisy_query(uint64_t seed, uint64_t qid, const float* base, int L, double sigma2, float* out,
                       int unit = 0) {
  double sigma = HG_DSQRT(sigma2);
  for (int b = 0; b < L / 4; ++b) {
    double z[4];
    normal4(seed, qid, (uint32_t)b, kTagNoise, z);
    for (int j = 0; j < 4; ++j) out[4 * b + j] = HG_FADD(base[4 * b + j], (float)HG_DMUL(sigma, z[j]));
  }
  if (unit) l2norm(out, L);
  else znorm(out, L);
}

}  // namespace hg
