// hg_arith.cuh -- the Hercules float arithmetic, shared by host and device.
//
// Every function reproduces one reference function's IEEE-754 binary32
// operation order exactly, so the B200 kernels and the host tree code give
// bit-identical results to the reference's AVX2 code.  Device code is built
// with -fmad=false and host code with -ffp-contract=off; the explicit
// round-to-nearest intrinsics below make the order independent of those
// flags on the device side as well.
#pragma once

#include <stdint.h>

#ifdef __CUDACC__
#define HG_HD __host__ __device__ __forceinline__
#else
#define HG_HD inline
#endif

#if defined(__CUDA_ARCH__)
#define HG_FADD(a, b) __fadd_rn((a), (b))
#define HG_FSUB(a, b) __fsub_rn((a), (b))
#define HG_FMUL(a, b) __fmul_rn((a), (b))
#define HG_FDIV(a, b) __fdiv_rn((a), (b))
#define HG_FSQRT(a) __fsqrt_rn((a))
#define HG_DADD(a, b) __dadd_rn((a), (b))
#define HG_DSUB(a, b) __dsub_rn((a), (b))
#define HG_DMUL(a, b) __dmul_rn((a), (b))
#define HG_DDIV(a, b) __ddiv_rn((a), (b))
#define HG_DSQRT(a) __dsqrt_rn((a))
#else
#include <math.h>
#define HG_FADD(a, b) ((a) + (b))
#define HG_FSUB(a, b) ((a) - (b))
#define HG_FMUL(a, b) ((a) * (b))
#define HG_FDIV(a, b) ((a) / (b))
#define HG_FSQRT(a) sqrtf((a))
#define HG_DADD(a, b) ((a) + (b))
#define HG_DSUB(a, b) ((a) - (b))
#define HG_DMUL(a, b) ((a) * (b))
#define HG_DDIV(a, b) ((a) / (b))
#define HG_DSQRT(a) sqrt((a))
#endif

#define HG_PAA_SEGMENTS 16
#define HG_SAX_CARD 256
#define HG_MINVAL (-2000000.0f)  // globals.h:66
#define HG_MAXVAL (2000000.0f)   // globals.h:67

// Horizontal sum of one 8-float chunk in the order two _mm256_hadd_ps plus
// lane0 + lane4 produce (ts.c:99-102): ((v0+v1)+(v2+v3)) + ((v4+v5)+(v6+v7)).
HG_HD float hg_hsum8(float v0, float v1, float v2, float v3, float v4, float v5, float v6,
                     float v7) {
  float a = HG_FADD(v0, v1), b = HG_FADD(v2, v3), c = HG_FADD(v4, v5), d = HG_FADD(v6, v7);
  return HG_FADD(HG_FADD(a, b), HG_FADD(c, d));
}

// Squared distance of one 8-float chunk: (q_i - x_i)^2 per lane, then hsum8.
HG_HD float hg_chunk_d2(const float* q, const float* x) {
  float d[8];
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    float v = HG_FSUB(q[j], x[j]);
    d[j] = HG_FMUL(v, v);
  }
  return hg_hsum8(d[0], d[1], d[2], d[3], d[4], d[5], d[6], d[7]);
}

// ts_euclidean_distance_SIMD (ts.c:83-109): early-abandoning squared
// distance; the test `dist < bound` precedes every chunk, so an abandoned
// call returns the partial sum.  L must be a multiple of 8.
HG_HD float hg_ed(const float* q, const float* x, int L, float bound) {
  float dist = 0.0f;
  for (int i = 0; i < L && dist < bound; i += 8) dist = HG_FADD(dist, hg_chunk_d2(q + i, x + i));
  return dist;
}

// calc_mean_stdev_SIMD (calc_utils.c:48-112): per 8-chunk hsum8 of x and of
// x*x accumulated sequentially, tail zero-padded (masked_read_8,
// calc_utils.c:129-150); stdev = sqrt((double)(sumsq/n)) rounded to float,
// which equals the correctly rounded float square root.
HG_HD void hg_mean_stdev(const float* series, int start, int end, float* mean, float* stdev) {
  *mean = 0.0f;
  *stdev = 0.0f;
  if (start >= end) return;  // the reference prints an error and keeps 0, 0
  int count = end - start;
  const float* x = series + start;
  float sum = 0.0f, sumsq = 0.0f;
  for (int off = 0; off < count; off += 8) {
    float v[8], v2[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      v[j] = (off + j < count) ? x[off + j] : 0.0f;
      v2[j] = HG_FMUL(v[j], v[j]);
    }
    sum = HG_FADD(sum, hg_hsum8(v[0], v[1], v[2], v[3], v[4], v[5], v[6], v[7]));
    sumsq = HG_FADD(sumsq, hg_hsum8(v2[0], v2[1], v2[2], v2[3], v2[4], v2[5], v2[6], v2[7]));
  }
  float fc = (float)count;
  *mean = HG_FDIV(sum, fc);
  sumsq = HG_FSUB(sumsq, HG_FDIV(HG_FMUL(sum, sum), fc));
  *stdev = HG_FSQRT(HG_FDIV(sumsq, fc));
}

// paa_from_ts (sax.c:46-56): a sequential float sum of L/16 values per
// segment, then one division.
HG_HD void hg_paa(const float* ts, float* paa, int L) {
  int per = L / HG_PAA_SEGMENTS;
  for (int s = 0; s < HG_PAA_SEGMENTS; ++s) {
    float acc = 0.0f;
    for (int i = 0; i < per; ++i) acc = HG_FADD(acc, ts[s * per + i]);
    paa[s] = HG_FDIV(acc, (float)per);
  }
}

// The iSAX symbol of sax_from_ts (sax.c:86-135, bsearch with the comparator
// of sax.c:28-41): the number of the 255 breakpoints strictly below paa
// (0 for NaN, 255 above the last breakpoint).
HG_HD int hg_sax_symbol(float paa, const float* bp255) {
  int lo = 0, hi = HG_SAX_CARD - 1;
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (bp255[mid] < paa) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

// One lane of minidist_paa_to_isax_raw_SIMD (sax.c:310-479) at the full
// 8-bit cardinality: the squared gap between paa and the symbol's region.
HG_HD float hg_lb_sax_lane(float paa, int sym, const float* bp255) {
  float lo = (sym == 0) ? HG_MINVAL : bp255[sym - 1];
  float hi = (sym == HG_SAX_CARD - 1) ? HG_MAXVAL : bp255[sym];
  if (lo > paa) {
    float t = HG_FSUB(lo, paa);
    return HG_FMUL(t, t);
  }
  if (hi < paa) {
    float t = HG_FSUB(hi, paa);
    return HG_FMUL(t, t);
  }
  return 0.0f;
}

// minidist_paa_to_isax_raw_SIMD reduction: s_j = d_j + d_{j+8}, hsum8, then
// times mindist_sqrt = L/16 (hercules_index.c:106-107).
HG_HD float hg_lb_sax(const float* paa, const uint8_t* sax, int L, const float* bp255) {
  float d[16];
#pragma unroll
  for (int j = 0; j < 16; ++j) d[j] = hg_lb_sax_lane(paa[j], sax[j], bp255);
  float s[8];
#pragma unroll
  for (int j = 0; j < 8; ++j) s[j] = HG_FADD(d[j], d[j + 8]);
  return HG_FMUL(hg_hsum8(s[0], s[1], s[2], s[3], s[4], s[5], s[6], s[7]),
                 (float)(L / HG_PAA_SEGMENTS));
}

// One segment term of calculate_node_min_distance (hercules_node.c:898-918):
// ind = {mean max, mean min, stdev max, stdev min}.  fmin/fabs run in double
// on float arguments there, which is exact, so float min/abs restate them.
HG_HD float hg_eapca_term(float mq, float sq, const float* ind, int len) {
  float temp_dist = 0.0f;
  float a = HG_FSUB(sq, ind[2]), b = HG_FSUB(sq, ind[3]);
  if (HG_FMUL(a, b) > 0.0f) {
    float fa = a < 0.0f ? -a : a, fb = b < 0.0f ? -b : b;
    float t = fa < fb ? fa : fb;
    temp_dist = HG_FADD(temp_dist, HG_FMUL(t, t));
  }
  a = HG_FSUB(mq, ind[0]);
  b = HG_FSUB(mq, ind[1]);
  if (HG_FMUL(a, b) > 0.0f) {
    float fa = a < 0.0f ? -a : a, fb = b < 0.0f ? -b : b;
    float t = fa < fb ? fa : fb;
    temp_dist = HG_FADD(temp_dist, HG_FMUL(t, t));
  }
  return HG_FMUL(temp_dist, (float)len);
}

// calculate_node_min_distance (hercules_node.c:879-924), LB_EAPCA.
HG_HD float hg_lb_eapca(const float* q, int nseg, const short* points, const float* sk) {
  float sum = 0.0f;
  int start = 0;
  for (int i = 0; i < nseg; ++i) {
    float mq, sq;
    hg_mean_stdev(q, start, points[i], &mq, &sq);
    sum = HG_FADD(sum, hg_eapca_term(mq, sq, sk + 4 * i, points[i] - start));
    start = points[i];
  }
  return sum;
}

// Order-preserving map of a non-negative float (or +inf/NaN) to uint32 for
// atomicMin; squared distances are never negative.
HG_HD uint32_t hg_f2key(float f) {
  union {
    float f;
    uint32_t u;
  } c;
  c.f = f;
  return c.u;
}
HG_HD float hg_key2f(uint32_t u) {
  union {
    float f;
    uint32_t u;
  } c;
  c.u = u;
  return c.f;
}
