/*
 * oracle_gen.c -- TEST INFRASTRUCTURE ONLY (part of the parity checker).
 *
 * A plain-C restatement of the seeded synthetic-data generator of
 * hercules_b200 (z-normalised random walks, unit-normalised Gaussian rows
 * and noisy queries, with steps drawn from a counter-based Philox4x32-10
 * stream through Box-Muller, transcendentals evaluated by series of
 * correctly rounded double operations).  It exists so that the CPU legs of
 * the benchmark (the reference's own query path, timed on the host cores)
 * can make the same inputs without loading the GPU library; tests check its
 * output bit for bit against hg_generate_walks / hg_generate_queries.
 *
 * The random walk and its z-normalisation follow the reference generator
 * (tools/Cgenerator/generator/main.c:27-65: float accumulation of N(0,1)
 * steps, float mean, float population variance, sqrt, (x - mean) / sd);
 * the reference draws its steps from GSL, which is absent, so the step
 * stream here is the project's own.
 *
 * Compiled with -ffp-contract=off: every float/double operation below is
 * one correctly rounded IEEE-754 operation, in the order written.
 */
#include <math.h>
#include <stdint.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

enum { TAG_WALK = 0x57414C4Bu, TAG_PICK = 0x5049434Bu, TAG_NOISE = 0x4E4F4953u };

/* Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11): ten rounds of the
 * multiply-xor bijection with the Weyl key schedule. */
static void philox(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0, uint32_t k1, uint32_t out[4]) {
  for (int r = 0; r < 10; ++r) {
    const uint64_t p0 = (uint64_t)0xD2511F53u * c0;
    const uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
    const uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0;
    const uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
    c1 = (uint32_t)p1;
    c3 = (uint32_t)p0;
    c0 = n0;
    c2 = n2;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  out[0] = c0;
  out[1] = c1;
  out[2] = c2;
  out[3] = c3;
}

/* (x + 1/2) / 2^32, exact in double */
static double unit_open(uint32_t x) { return ((double)x + 0.5) * 2.3283064365386963e-10; }

/* ln x for x in (0, 1]: x = m 2^e with m in [sqrt(1/2), sqrt(2)), then
 * ln m = 2 atanh(s) = 2 s (1 + s^2/3 + s^4/5 + ...), s = (m - 1) / (m + 1),
 * truncated after the s^22 term (|s| < 0.172). */
static double series_log(double x) {
  uint64_t u;
  memcpy(&u, &x, sizeof u);
  int e = (int)((u >> 52) & 0x7FF) - 1023;
  u = (u & 0x000FFFFFFFFFFFFFull) | 0x3FF0000000000000ull;
  double m;
  memcpy(&m, &u, sizeof m);
  if (m > 1.4142135623730951) {
    m = m * 0.5;
    e += 1;
  }
  const double s = (m - 1.0) / (m + 1.0);
  const double s2 = s * s;
  double p = 1.0 / 23.0;
  static const double inv_odd[11] = {1.0 / 21.0, 1.0 / 19.0, 1.0 / 17.0, 1.0 / 15.0, 1.0 / 13.0, 1.0 / 11.0,
                                     1.0 / 9.0,  1.0 / 7.0,  1.0 / 5.0,  1.0 / 3.0,  1.0};
  for (int i = 0; i < 11; ++i) p = p * s2 + inv_odd[i];
  const double lm = (2.0 * s) * p;
  return (double)e * 0.6931471805599453 + lm;
}

/* sin and cos of a in [0, pi/2) by their Taylor series to the a^15 and a^16
 * terms, Horner in a^2. */
static void series_sincos(double a, double *sn, double *cs) {
  const double a2 = a * a;
  static const double sin_c[7] = {1.0 / 6227020800.0, -1.0 / 39916800.0, 1.0 / 362880.0, -1.0 / 5040.0,
                                  1.0 / 120.0,        -1.0 / 6.0,        1.0};
  double s = -1.0 / 1307674368000.0;
  for (int i = 0; i < 7; ++i) s = s * a2 + sin_c[i];
  *sn = s * a;
  static const double cos_c[7] = {-1.0 / 87178291200.0, 1.0 / 479001600.0, -1.0 / 3628800.0, 1.0 / 40320.0,
                                  -1.0 / 720.0,         1.0 / 24.0,        -0.5};
  double c = 1.0 / 20922789888000.0;
  for (int i = 0; i < 7; ++i) c = c * a2 + cos_c[i];
  *cs = c * a2 + 1.0;
}

/* Box-Muller: r = sqrt(-2 ln u1), angle 2 pi u2 reduced to a quadrant. */
static void box_muller(uint32_t x1, uint32_t x2, double *z0, double *z1) {
  const double r = sqrt(-2.0 * series_log(unit_open(x1)));
  const double v = unit_open(x2) * 4.0;
  int q = (int)v;
  if (q > 3) q = 3;
  const double a = (v - (double)q) * 1.5707963267948966;
  double sn, cs, c, s;
  series_sincos(a, &sn, &cs);
  switch (q) {
    case 0: c = cs; s = sn; break;
    case 1: c = -sn; s = cs; break;
    case 2: c = -cs; s = -sn; break;
    default: c = sn; s = -cs; break;
  }
  *z0 = r * c;
  *z1 = r * s;
}

/* Four N(0,1) draws: block b of stream element `id` of stream (seed, tag). */
static void normal4(uint64_t seed, uint64_t id, uint32_t b, uint32_t tag, double z[4]) {
  uint32_t o[4];
  philox((uint32_t)id, (uint32_t)(id >> 32), b, tag, (uint32_t)seed, (uint32_t)(seed >> 32), o);
  box_muller(o[0], o[1], &z[0], &z[1]);
  box_muller(o[2], o[3], &z[2], &z[3]);
}

static void znorm(float *ts, int L) {
  float mean = 0.0f;
  for (int i = 0; i < L; ++i) mean = mean + ts[i];
  mean = mean / (float)L;
  float sd = 0.0f;
  for (int i = 0; i < L; ++i) {
    const float d = ts[i] - mean;
    sd = sd + d * d;
  }
  sd = sd / (float)L;
  sd = sqrtf(sd);
  for (int i = 0; i < L; ++i) ts[i] = (ts[i] - mean) / sd;
}

static void l2norm(float *v, int L) {
  float ss = 0.0f;
  for (int i = 0; i < L; ++i) ss = ss + v[i] * v[i];
  const float nrm = sqrtf(ss);
  if (nrm > 0.0f)
    for (int i = 0; i < L; ++i) v[i] = v[i] / nrm;
}

static void walk_row(uint64_t seed, uint64_t id, int L, float *out) {
  float x = 0.0f;
  for (int b = 0; b < L / 4; ++b) {
    double z[4];
    normal4(seed, id, (uint32_t)b, TAG_WALK, z);
    for (int j = 0; j < 4; ++j) {
      x = x + (float)z[j];
      out[4 * b + j] = x;
    }
  }
  znorm(out, L);
}

static void unit_row(uint64_t seed, uint64_t id, int L, float *out) {
  for (int b = 0; b < L / 4; ++b) {
    double z[4];
    normal4(seed, id, (uint32_t)b, TAG_WALK, z);
    for (int j = 0; j < 4; ++j) out[4 * b + j] = (float)z[j];
  }
  l2norm(out, L);
}

static uint64_t pick_row(uint64_t seed, uint64_t qid, uint64_t n) {
  uint32_t o[4];
  philox((uint32_t)qid, (uint32_t)(qid >> 32), 0u, TAG_PICK, (uint32_t)seed, (uint32_t)(seed >> 32), o);
  return ((((uint64_t)o[0]) << 32) | o[1]) % n;
}

static void noisy_row(uint64_t seed, uint64_t qid, const float *base, int L, double sigma2, float *out, int unit) {
  const double sigma = sqrt(sigma2);
  for (int b = 0; b < L / 4; ++b) {
    double z[4];
    normal4(seed, qid, (uint32_t)b, TAG_NOISE, z);
    for (int j = 0; j < 4; ++j) out[4 * b + j] = base[4 * b + j] + (float)(sigma * z[j]);
  }
  if (unit) l2norm(out, L);
  else znorm(out, L);
}

/* Rows [first, first + n) of stream `seed`: random walks (unit = 0) or unit
 * vectors (unit = 1); L a multiple of 4.  threads <= 0: every core. */
void or_gen_rows(uint64_t seed, uint64_t first, uint64_t n, int L, float *out, int unit, int threads) {
#ifdef _OPENMP
  if (threads <= 0) threads = omp_get_max_threads();
#pragma omp parallel for schedule(static, 1024) num_threads(threads)
#endif
  for (int64_t i = 0; i < (int64_t)n; ++i) {
    if (unit) unit_row(seed, first + (uint64_t)i, L, out + (uint64_t)i * L);
    else walk_row(seed, first + (uint64_t)i, L, out + (uint64_t)i * L);
  }
  (void)threads;
}

/* Noisy queries j = 0..nq-1 of stream `seed` over a collection of n rows:
 * row pick(j) plus N(0, sigma2[j]) noise, then z-normalised (unit = 0) or
 * L2-normalised (unit = 1).  The base row is regenerated from data_seed, so
 * the collection itself is not needed.  base_ids (may be NULL) gets pick(j). */
void or_gen_queries(uint64_t data_seed, uint64_t seed, uint64_t n, int L, int nq, const double *sigma2, float *out,
                    uint64_t *base_ids, int unit) {
  float base[16384];
  if (L > 16384) return;
  for (int j = 0; j < nq; ++j) {
    const uint64_t b = pick_row(seed, (uint64_t)j, n);
    if (base_ids) base_ids[j] = b;
    if (unit) unit_row(data_seed, b, L, base);
    else walk_row(data_seed, b, L, base);
    noisy_row(seed, (uint64_t)j, base, L, sigma2[j], out + (uint64_t)j * L, unit);
  }
}
