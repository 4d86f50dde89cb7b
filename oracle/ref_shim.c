/*
 * ref_shim.c -- thin C entry points into the reference's own primitives.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is compiled together with the
 * reference sources (code/hercules/src/*.c, read in place) into
 * oracle/_ref/libref_hercules.so by oracle/Makefile.  The tests call these
 * entry points to pin the CPU restatement (hercules_oracle.c) bit for bit
 * against the reference functions themselves.  Nothing here is shipped.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "globals.h"
#include "include/calc_utils.h"
#include "include/hercules_node.h"
#include "include/hercules_query_engine.h"
#include "include/sax.h"
#include "include/ts.h"
#include "include/sax_breakpoints.h"

/* ts.c:83 */
float shim_ed(const float *t, const float *s, int L, float bound) {
  return ts_euclidean_distance_SIMD((ts_type *)t, (ts_type *)s, L, bound);
}

/* calc_utils.c:48 */
void shim_mean_stdev(const float *x, int start, int end, float *mean, float *stdev) {
  calc_mean_stdev_SIMD((ts_type *)x, start, end, mean, stdev);
}

/* sax.c:46 */
void shim_paa(const float *ts, float *paa, int L) { paa_from_ts((ts_type *)ts, paa, 16, L / 16); }

/* sax.c:86 */
void shim_sax(const float *ts, unsigned char *sax, int L) {
  sax_from_ts((ts_type *)ts, sax, L / 16, 16, 256, 8);
}

/* sax.c:310, called as in hercules_query_engine.c:2189-2194 */
float shim_lb_sax(const float *paa, const unsigned char *sax, int L) {
  unsigned char card[16];
  memset(card, 8, sizeof card);
  return minidist_paa_to_isax_raw_SIMD((float *)paa, (sax_type *)sax, card, 8, 256, 16, MINVAL,
                                       MAXVAL, (float)(L / 16));
}

/* hercules_node.c:879 on a node holding only what the function reads */
float shim_lb_eapca(const float *q, int nseg, const short *points, const float *sk) {
  struct hercules_node node;
  memset(&node, 0, sizeof node);
  struct segment_sketch *sks = calloc(nseg, sizeof(struct segment_sketch));
  float *ind = malloc(sizeof(float) * 4 * nseg);
  memcpy(ind, sk, sizeof(float) * 4 * nseg);
  short *pts = malloc(sizeof(short) * nseg);
  memcpy(pts, points, sizeof(short) * nseg);
  for (int i = 0; i < nseg; ++i) {
    sks[i].indicators = ind + 4 * i;
    sks[i].num_indicators = 4;
  }
  node.node_points = pts;
  node.num_node_points = (short)nseg;
  node.node_segment_sketches = sks;
  float r = calculate_node_min_distance(NULL, &node, (ts_type *)q);
  free(sks);
  free(ind);
  free(pts);
  return r;
}

/* hercules_query_engine.c:4034: the node pointer field carries the row id */
void shim_topk_insert(float *dist, long long *id, unsigned *cur, unsigned k, float d, long long cid) {
  struct query_result *q = calloc(k, sizeof(struct query_result));
  for (unsigned i = 0; i < k; ++i) {
    q[i].distance = dist[i];
    q[i].node = (struct hercules_node *)(intptr_t)id[i];
  }
  struct query_result r;
  memset(&r, 0, sizeof r);
  r.distance = d;
  r.node = (struct hercules_node *)(intptr_t)cid;
  queue_bounded_sorted_insert(q, r, cur, k);
  for (unsigned i = 0; i < k; ++i) {
    dist[i] = q[i].distance;
    id[i] = (long long)(intptr_t)q[i].node;
  }
  free(q);
}

/* the 255 breakpoints of cardinality 256 (sax.c:113, offset (c-1)(c-2)/2) */
void shim_breakpoints(float *out) { memcpy(out, &sax_breakpoints[32385], sizeof(float) * 255); }
