/*
 * hercules_oracle.c -- CPU restatement of the Hercules exact k-NN query path.
 *
 * TEST INFRASTRUCTURE ONLY (the parity checker; see hercules_oracle.h).
 *
 * Compiled with -O2 -ffp-contract=off: every float expression below is
 * evaluated exactly as written, one IEEE-754 binary32 rounding per operation,
 * in the order the reference's AVX2 code performs it.  Each function names
 * the reference function and lines it restates.
 */
#include "hercules_oracle.h"

#include <float.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

/* ---------------------------------------------------------------------- */
/* primitives                                                              */
/* ---------------------------------------------------------------------- */

/* Sum of one 8-float chunk in the order of two _mm256_hadd_ps followed by
 * lane0 + lane4 (ts.c:99-102, calc_utils.c:75-78):
 *   ((v0+v1)+(v2+v3)) + ((v4+v5)+(v6+v7)). */
static inline float hsum8(const float v[8]) {
  float a = v[0] + v[1];
  float b = v[2] + v[3];
  float c = v[4] + v[5];
  float d = v[6] + v[7];
  float lo = a + b;
  float hi = c + d;
  return lo + hi;
}

/* ts.c:83-109.  The abandon test runs before every chunk, so an abandoned
 * call returns the partial sum reached so far. */
float or_ed(const float *t, const float *s, int L, float bound) {
  float distance = 0.0f;
  int i = 0;
  int size = L;
  while (size > 0 && distance < bound) {
    float d[8];
    for (int j = 0; j < 8; ++j) {
      float v = t[i + j] - s[i + j];
      d[j] = v * v;
    }
    size -= 8;
    i += 8;
    float c = hsum8(d);
    distance = distance + c;
  }
  return distance;
}

/* calc_utils.c:48-112 with masked_read_8 (:129-150): the tail chunk is
 * zero-padded to 8 values; stdev = sqrt((double)(sumsq/n)) rounded to float,
 * which equals the correctly rounded float square root. */
void or_mean_stdev(const float *series, int start, int end, float *mean, float *stdev) {
  *mean = 0.0f;
  *stdev = 0.0f;
  if (start >= end) return; /* the reference prints an error and leaves 0, 0 */
  int count = end - start;
  int d = count;
  const float *x = series + start;
  float sum = 0.0f, sumsq = 0.0f;
  while (d > 0) {
    float v[8], v2[8];
    int n = d >= 8 ? 8 : d;
    for (int j = 0; j < 8; ++j) v[j] = j < n ? x[j] : 0.0f;
    for (int j = 0; j < 8; ++j) v2[j] = v[j] * v[j];
    sum = sum + hsum8(v);
    sumsq = sumsq + hsum8(v2);
    x += n;
    d -= n;
  }
  float fc = (float)count;
  *mean = sum / fc;
  sumsq = sumsq - ((sum * sum) / fc);
  *stdev = (float)sqrt((double)(sumsq / fc));
}

/* sax.c:46-56: sequential float sum over L/16 values, then a division. */
void or_paa(const float *ts, float *paa, int L) {
  int per = L / OR_PAA_SEGMENTS;
  for (int s = 0; s < OR_PAA_SEGMENTS; ++s) {
    float acc = 0.0f;
    for (int i = 0; i < per; ++i) acc = acc + ts[s * per + i];
    paa[s] = acc / (float)per;
  }
}

/* sax.c:86-135 with the bsearch comparator of sax.c:28-41.  The comparator
 * selects s with bp[s-1] < paa <= bp[s]; with 255 sorted breakpoints this is
 * the number of breakpoints strictly below paa (0 for NaN, 255 above the
 * last breakpoint). */
void or_sax(const float *ts, unsigned char *sax, int L, const float *bp255) {
  float paa[OR_PAA_SEGMENTS];
  or_paa(ts, paa, L);
  for (int s = 0; s < OR_PAA_SEGMENTS; ++s) {
    int lo = 0, hi = OR_SAX_CARD - 1; /* count of bp < paa, binary search */
    while (lo < hi) {
      int mid = (lo + hi) / 2;
      if (bp255[mid] < paa[s]) lo = mid + 1; else hi = mid;
    }
    sax[s] = (unsigned char)lo;
  }
}

/* sax.c:310-479 with every segment at the full 8-bit cardinality:
 * region_lower = region_upper = symbol; MINVAL/MAXVAL (globals.h:66-67) for
 * the open ends; per-lane distance, then (d_j + d_{j+8}), two hadds and
 * lane0 + lane4; finally times mindist_sqrt = L/16 (hercules_index.c:106). */
float or_lb_sax(const float *paa, const unsigned char *sax, int L, const float *bp255) {
  float dl[16];
  for (int j = 0; j < 16; ++j) {
    int v = sax[j];
    float lo = (v == 0) ? (float)-2000000 : bp255[v - 1];
    float hi = (v == OR_SAX_CARD - 1) ? (float)2000000 : bp255[v];
    float p = paa[j];
    float d = 0.0f;
    if (lo > p) {
      float t = lo - p;
      d = t * t;
    } else if (hi < p) {
      float t = hi - p;
      d = t * t;
    }
    dl[j] = d;
  }
  float s[8];
  for (int j = 0; j < 8; ++j) s[j] = dl[j] + dl[j + 8];
  float ratio = (float)(L / OR_PAA_SEGMENTS);
  return hsum8(s) * ratio;
}

static inline int seg_start(const short *points, int i) { return i == 0 ? 0 : points[i - 1]; }
static inline int seg_len(const short *points, int i) {
  return i == 0 ? points[0] : points[i] - points[i - 1];
}

/* hercules_node.c:879-924.  fmin/fabs run in double on float arguments,
 * which is exact, so they are restated as float min/abs. */
float or_lb_eapca(const float *q, int nseg, const short *points, const float *sk) {
  float sum = 0.0f;
  int start = 0;
  for (int i = 0; i < nseg; ++i) {
    float mq, sq;
    or_mean_stdev(q, start, points[i], &mq, &sq);
    start = points[i];
    const float *ind = sk + 4 * i;
    float temp_dist = 0.0f;
    if ((sq - ind[2]) * (sq - ind[3]) > 0) {
      float a = fabsf(sq - ind[2]), b = fabsf(sq - ind[3]);
      float t = a < b ? a : b;
      temp_dist = temp_dist + t * t;
    }
    if ((mq - ind[0]) * (mq - ind[1]) > 0) {
      float a = fabsf(mq - ind[0]), b = fabsf(mq - ind[1]);
      float t = a < b ? a : b;
      temp_dist = temp_dist + t * t;
    }
    sum = sum + temp_dist * (float)seg_len(points, i);
  }
  return sum;
}

/* hercules_query_engine.c:4034-4082 */
void or_topk_insert(float *dist, int64_t *id, uint64_t *aux, int *cur, int k,
                    float d, int64_t cid, uint64_t caux, int tie_lowest) {
  for (int i = 0; i < *cur; ++i) {
    if (dist[i] == d) {
      if (tie_lowest && cid < id[i]) {
        id[i] = cid;
        if (aux) aux[i] = caux;
      }
      return;
    }
  }
  int pos;
  if (*cur == k) {
    pos = k - 1;
  } else {
    pos = *cur;
    ++(*cur);
  }
  dist[pos] = d;
  id[pos] = cid;
  if (aux) aux[pos] = caux;
  for (int j = pos; j > 0 && dist[j - 1] > dist[j]; --j) {
    float td = dist[j];
    dist[j] = dist[j - 1];
    dist[j - 1] = td;
    int64_t ti = id[j];
    id[j] = id[j - 1];
    id[j - 1] = ti;
    if (aux) {
      uint64_t ta = aux[j];
      aux[j] = aux[j - 1];
      aux[j - 1] = ta;
    }
  }
}

/* ---------------------------------------------------------------------- */
/* tree                                                                    */
/* ---------------------------------------------------------------------- */

typedef struct or_node {
  struct or_node *left, *right, *parent;
  int is_leaf, is_left;
  unsigned level;
  int nseg;
  short *points;
  int nhs;
  short *hs_points;
  float *sk;    /* nseg x 4: mean max, mean min, stdev max, stdev min */
  float *hs_sk; /* nhs x 4 */
  /* split policy (hercules_node_split.h:21-34) */
  short split_from, split_to;
  int split_idx;
  float split_value;
  unsigned node_size;
  uint32_t *members;
  unsigned cap;
  char *filename;
  uint64_t file_pos;
  int leaf_index;
} or_node;

struct or_index {
  int L;
  int leaf_size;
  uint64_t n;
  const float *data; /* build: the caller's dataset */
  or_node *root;
  int num_nodes;
  int num_leaves;
  or_node **leaves; /* DFS (left first) order */
  float *rows;      /* leaf-ordered rows (NULL after or_build_mt without rows) */
  int64_t *ids;     /* dataset id per leaf-ordered row */
  int owns_rows;
  int threads;      /* or_build_mt: worker threads (0 = the sequential build) */
};

/* calc_hs_split_points, hercules_node_split.c:371-396 (min_length = 1) */
static int calc_hs_points(short *hs, const short *points, int nseg) {
  int c = 0;
  for (int i = 0; i < nseg; ++i) {
    short length = points[i];
    if (i > 0) length = (short)(points[i] - points[i - 1]);
    if (length >= 2) {
      int start = i > 0 ? points[i - 1] : 0;
      hs[c++] = (short)(start + (length / 2));
    }
    hs[c++] = points[i];
  }
  return c;
}

static void init_sketch(float *s, int n) {
  for (int i = 0; i < n; ++i) {
    s[4 * i + 0] = -FLT_MAX;
    s[4 * i + 1] = FLT_MAX;
    s[4 * i + 2] = -FLT_MAX;
    s[4 * i + 3] = FLT_MAX;
  }
}

/* hercules_leaf_node_init + node_init_segments, hercules_node.c:84-225 */
static or_node *new_leaf(const short *points, int nseg) {
  or_node *n = (or_node *)calloc(1, sizeof(or_node));
  n->is_leaf = 1;
  n->nseg = nseg;
  n->points = (short *)malloc(sizeof(short) * nseg);
  memcpy(n->points, points, sizeof(short) * nseg);
  n->hs_points = (short *)malloc(sizeof(short) * nseg * 2);
  n->nhs = calc_hs_points(n->hs_points, points, nseg);
  n->sk = (float *)malloc(sizeof(float) * 4 * nseg);
  n->hs_sk = (float *)malloc(sizeof(float) * 4 * n->nhs);
  init_sketch(n->sk, nseg);
  init_sketch(n->hs_sk, n->nhs);
  n->split_idx = 0;
  return n;
}

/* create_hercules_node_filename, hercules_node.c:441-486 */
static void make_filename(or_node *n, const or_node *parent) {
  char buf[512];
  int l = sprintf(buf, "%02d", n->nseg);
  if (n->level) {
    l += sprintf(buf + l, "%s", n->is_left ? "_L" : "_R");
    l += sprintf(buf + l, "%s", parent->split_idx ? "_1" : "_0");
    l += sprintf(buf + l, "_(%d,%d,%g)", parent->split_from, parent->split_to,
                 (double)parent->split_value);
  }
  sprintf(buf + l, "_%d", n->level);
  n->filename = strdup(buf);
}

/* node_segment_sketch_update_sketch_parallel, hercules_node_split.c:86-120 */
static void sketch_update(float *ind, const float *x, int from, int to) {
  float m, s;
  or_mean_stdev(x, from, to, &m, &s);
  ind[0] = fmaxf(ind[0], m);
  ind[1] = fminf(ind[1], m);
  ind[2] = fmaxf(ind[2], s);
  ind[3] = fminf(ind[3], s);
}

/* update_node_statistics_parallel, hercules_node.c:523-555 */
static void update_stats(or_node *n, const float *x) {
  for (int i = 0; i < n->nseg; ++i) sketch_update(n->sk + 4 * i, x, seg_start(n->points, i), n->points[i]);
  for (int i = 0; i < n->nhs; ++i)
    sketch_update(n->hs_sk + 4 * i, x, seg_start(n->hs_points, i), n->hs_points[i]);
  ++n->node_size;
}

static void append_member(or_node *n, uint32_t id) {
  if (n->node_size > n->cap) {
    n->cap = n->cap ? n->cap * 2 : 64;
    while (n->cap < n->node_size) n->cap *= 2;
    n->members = (uint32_t *)realloc(n->members, sizeof(uint32_t) * n->cap);
  }
  n->members[n->node_size - 1] = id;
}

/* node_split_policy_route_to_left, hercules_node_split.c:172-193 */
static int route_left(const or_node *n, const float *x) {
  float m, s;
  or_mean_stdev(x, n->split_from, n->split_to, &m, &s);
  float v = n->split_idx ? s : m;
  return v < n->split_value;
}

/* range_calc, hercules_node_split.c:337-345 */
static float range_calc(const float *ind, int len) {
  float mean_width = ind[0] - ind[1];
  float stdev_upper = ind[2];
  return (float)len * (mean_width * mean_width + stdev_upper * stdev_upper);
}

/* The two split policies of hercules_node_split.c:22-71 evaluated for one
 * segment sketch: returns diff_value and the split value. */
static float policy_diff(const float *ind, int len, int policy, float *value) {
  float child[2][4];
  memcpy(child[0], ind, sizeof(float) * 4);
  memcpy(child[1], ind, sizeof(float) * 4);
  float v;
  if (policy == 0) {
    v = (ind[0] + ind[1]) / 2;
    child[0][1] = v;
    child[1][0] = v;
  } else {
    v = (ind[2] + ind[3]) / 2;
    child[0][2] = v;
    child[1][3] = v;
  }
  *value = v;
  float r0 = range_calc(child[0], len);
  float r1 = range_calc(child[1], len);
  float mean = 0.0f; /* calc_mean, calc_utils.c:165-188 */
  mean = mean + r0;
  mean = mean + r1;
  mean = mean / (float)2;
  float node_range = range_calc(ind, len);
  return node_range - mean;
}

static int cmp_short(const void *a, const void *b) {
  short x = *(const short *)a, y = *(const short *)b;
  return x < y ? -1 : (x > y ? 1 : 0);
}

/* hercules_index_split_node, hercules_node_split.c:1043-1345: the split
 * decision from the node's sketches and the two children, left empty. */
static void split_decide(or_index *ix, or_node *n) {
  float max_diff = -FLT_MAX;
  int hs_split_point = -1;
  short from = 0, to = 0;
  int idx = 0;
  float value = 0.0f;
  for (int i = 0; i < n->nseg; ++i) {
    int len = seg_len(n->points, i);
    for (int j = 0; j < 2; ++j) {
      float v;
      float diff = policy_diff(n->sk + 4 * i, len, j, &v);
      if (diff > max_diff) {
        max_diff = diff;
        from = (short)seg_start(n->points, i);
        to = n->points[i];
        idx = j;
        value = v;
      }
    }
  }
  max_diff = max_diff * 2;
  for (int i = 0; i < n->nhs; ++i) {
    int len = seg_len(n->hs_points, i);
    for (int j = 0; j < 2; ++j) {
      float v;
      float diff = policy_diff(n->hs_sk + 4 * i, len, j, &v);
      if (diff > max_diff) {
        max_diff = diff;
        from = (short)seg_start(n->hs_points, i);
        to = n->hs_points[i];
        idx = j;
        value = v;
        /* get_hs_split_point, hercules_node_split.c:296-313 */
        int found = 0;
        for (int p = 0; p < n->nseg; ++p)
          if (n->points[p] == to) found = 1;
        hs_split_point = found ? from : to;
      }
    }
  }
  n->split_from = from;
  n->split_to = to;
  n->split_idx = idx;
  n->split_value = value;

  int ncp = n->nseg + (hs_split_point >= 0 ? 1 : 0);
  short *cp = (short *)malloc(sizeof(short) * ncp);
  memcpy(cp, n->points, sizeof(short) * n->nseg);
  if (hs_split_point >= 0) {
    cp[ncp - 1] = (short)hs_split_point;
    qsort(cp, ncp, sizeof(short), cmp_short);
  }
  /* split_node_create_children, hercules_node_split.c:197-262 */
  or_node *l = new_leaf(cp, ncp), *r = new_leaf(cp, ncp);
  free(cp);
  l->parent = r->parent = n;
  l->level = r->level = n->level + 1;
  l->is_left = 1;
  make_filename(l, n);
  make_filename(r, n);
  n->left = l;
  n->right = r;
  ix->num_nodes += 2;
}

static void split_node(or_index *ix, or_node *n) {
  split_decide(ix, n);
  or_node *l = n->left, *r = n->right;
  /* redistribution in insertion order, :1294-1333 */
  for (unsigned m = 0; m < n->node_size; ++m) {
    uint32_t id = n->members[m];
    const float *x = ix->data + (uint64_t)id * ix->L;
    or_node *c = route_left(n, x) ? l : r;
    update_stats(c, x);
    append_member(c, id);
  }
  free(n->members);
  n->members = NULL;
  n->cap = 0;
  n->is_leaf = 0;
}

/* hercules_index_insert_series_to_node_parallel, hercules_index.c:2829-2927 */
static void insert(or_index *ix, uint32_t id) {
  const float *x = ix->data + (uint64_t)id * ix->L;
  or_node *n = ix->root;
  while (!n->is_leaf) n = route_left(n, x) ? n->left : n->right;
  update_stats(n, x);
  append_member(n, id);
  if (n->node_size >= (unsigned)ix->leaf_size) split_node(ix, n);
}

static void collect_leaves(or_index *ix, or_node *n, int *cnt) {
  if (!n->is_leaf) {
    collect_leaves(ix, n->left, cnt);
    collect_leaves(ix, n->right, cnt);
  } else {
    if (ix->leaves) ix->leaves[*cnt] = n;
    n->leaf_index = *cnt;
    ++(*cnt);
  }
}

/* update_node_ancestors_statistics_for_non_split_segments,
 * hercules_node.c:613-657.  split_segment stays -1 in the parallel build,
 * so segment i of a parent is merged with segment i of the child. */
static void merge_ancestors(or_node *leaf) {
  or_node *cn = leaf, *cp = leaf->parent;
  while (cp) {
    for (int i = 0; i < cp->nseg; ++i) {
      float *p = cp->sk + 4 * i;
      const float *c = cn->sk + 4 * i;
      p[0] = fmaxf(p[0], c[0]);
      p[1] = fminf(p[1], c[1]);
      p[2] = fmaxf(p[2], c[2]);
      p[3] = fminf(p[3], c[3]);
    }
    cn = cp;
    cp = cp->parent;
  }
}

static void finalize(or_index *ix) {
  int cnt = 0;
  collect_leaves(ix, ix->root, &cnt);
  ix->num_leaves = cnt;
  ix->leaves = (or_node **)malloc(sizeof(or_node *) * (cnt > 0 ? cnt : 1));
  cnt = 0;
  collect_leaves(ix, ix->root, &cnt);
  ix->rows = (float *)malloc(sizeof(float) * ix->L * (ix->n ? ix->n : 1));
  ix->ids = (int64_t *)malloc(sizeof(int64_t) * (ix->n ? ix->n : 1));
  ix->owns_rows = 1;
  uint64_t pos = 0;
  for (int i = 0; i < cnt; ++i) {
    or_node *lf = ix->leaves[i];
    lf->file_pos = pos;
    for (unsigned m = 0; m < lf->node_size; ++m) {
      uint32_t id = lf->members[m];
      memcpy(ix->rows + (pos + m) * ix->L, ix->data + (uint64_t)id * ix->L, sizeof(float) * ix->L);
      ix->ids[pos + m] = id;
    }
    pos += lf->node_size;
    merge_ancestors(lf);
  }
}

or_index *or_build(const float *data, uint64_t n, int L, int leaf_size) {
  if (L <= 0 || L % 16 != 0 || leaf_size <= 0) return NULL;
  or_index *ix = (or_index *)calloc(1, sizeof(or_index));
  ix->L = L;
  ix->leaf_size = leaf_size;
  ix->n = n;
  ix->data = data;
  short pt = (short)L; /* calc_split_points with init_segments = 1 */
  ix->root = new_leaf(&pt, 1);
  ix->root->filename = NULL;
  make_filename(ix->root, NULL);
  ix->num_nodes = 1;
  for (uint64_t i = 0; i < n; ++i) insert(ix, (uint32_t)i);
  finalize(ix);
  ix->data = NULL;
  return ix;
}

/* ---- the same build on several threads ----------------------------------
 * A node's sketches are the element-wise max / min of (mean, stdev) over the
 * series appended to it, and max / min do not depend on order; the
 * sequential build updates them per insert, this one computes them over the
 * member list when they are needed (at the node's split and, for the final
 * leaves, at the end), in parallel.  Routing, which depends on the tree at
 * the time of each insert, is done for a window of series at a time against
 * the current tree; a series whose cached leaf split before its turn is
 * routed on from that node.  The insertion order, the split decisions and
 * the redistribution order are those of or_build, so the tree, the leaf
 * order and every float are identical (tests check the index files). */

static void sketch_members(const or_index *ix, or_node *n, int threads) {
  const int nseg = n->nseg, nhs = n->nhs;
  init_sketch(n->sk, nseg);
  init_sketch(n->hs_sk, nhs);
  if (!n->node_size) return;
#ifdef _OPENMP
#pragma omp parallel num_threads(threads)
#endif
  {
    float *sk = (float *)malloc(sizeof(float) * 4 * (nseg + nhs));
    init_sketch(sk, nseg + nhs);
#ifdef _OPENMP
#pragma omp for schedule(static)
#endif
    for (int64_t m = 0; m < (int64_t)n->node_size; ++m) {
      const float *x = ix->data + (uint64_t)n->members[m] * ix->L;
      for (int i = 0; i < nseg; ++i) sketch_update(sk + 4 * i, x, seg_start(n->points, i), n->points[i]);
      for (int i = 0; i < nhs; ++i)
        sketch_update(sk + 4 * (nseg + i), x, seg_start(n->hs_points, i), n->hs_points[i]);
    }
#ifdef _OPENMP
#pragma omp critical
#endif
    {
      for (int i = 0; i < nseg; ++i) {
        float *p = n->sk + 4 * i;
        const float *c = sk + 4 * i;
        p[0] = fmaxf(p[0], c[0]);
        p[1] = fminf(p[1], c[1]);
        p[2] = fmaxf(p[2], c[2]);
        p[3] = fminf(p[3], c[3]);
      }
      for (int i = 0; i < nhs; ++i) {
        float *p = n->hs_sk + 4 * i;
        const float *c = sk + 4 * (nseg + i);
        p[0] = fmaxf(p[0], c[0]);
        p[1] = fminf(p[1], c[1]);
        p[2] = fmaxf(p[2], c[2]);
        p[3] = fminf(p[3], c[3]);
      }
    }
    free(sk);
  }
  (void)threads;
}

static void append_only(or_node *n, uint32_t id) {
  ++n->node_size;
  append_member(n, id);
}

static void split_node_mt(or_index *ix, or_node *n, unsigned char *flags) {
  sketch_members(ix, n, ix->threads);
  split_decide(ix, n);
  or_node *l = n->left, *r = n->right;
  const unsigned cnt = n->node_size;
#ifdef _OPENMP
#pragma omp parallel for schedule(static) num_threads(ix->threads)
#endif
  for (int64_t m = 0; m < (int64_t)cnt; ++m)
    flags[m] = (unsigned char)route_left(n, ix->data + (uint64_t)n->members[m] * ix->L);
  for (unsigned m = 0; m < cnt; ++m) append_only(flags[m] ? l : r, n->members[m]);
  free(n->members);
  n->members = NULL;
  n->cap = 0;
  n->is_leaf = 0;
}

or_index *or_build_mt(const float *data, uint64_t n, int L, int leaf_size, int threads, int keep_rows) {
  if (L <= 0 || L % 16 != 0 || leaf_size <= 0) return NULL;
#ifdef _OPENMP
  if (threads <= 0) threads = omp_get_max_threads();
#else
  threads = 1;
#endif
  or_index *ix = (or_index *)calloc(1, sizeof(or_index));
  ix->L = L;
  ix->leaf_size = leaf_size;
  ix->n = n;
  ix->data = data;
  ix->threads = threads;
  short pt = (short)L;
  ix->root = new_leaf(&pt, 1);
  make_filename(ix->root, NULL);
  ix->num_nodes = 1;
  const uint64_t W = (uint64_t)1 << 18;
  or_node **route = (or_node **)malloc(sizeof(or_node *) * W);
  unsigned char *flags = (unsigned char *)malloc((size_t)leaf_size + 1);
  for (uint64_t i0 = 0; i0 < n; i0 += W) {
    const uint64_t w = n - i0 < W ? n - i0 : W;
#ifdef _OPENMP
#pragma omp parallel for schedule(static, 256) num_threads(threads)
#endif
    for (int64_t j = 0; j < (int64_t)w; ++j) {
      const float *x = data + (i0 + (uint64_t)j) * L;
      or_node *nd = ix->root;
      while (!nd->is_leaf) nd = route_left(nd, x) ? nd->left : nd->right;
      route[j] = nd;
    }
    for (uint64_t j = 0; j < w; ++j) {
      const uint32_t id = (uint32_t)(i0 + j);
      const float *x = data + (uint64_t)id * L;
      or_node *nd = route[j];
      while (!nd->is_leaf) nd = route_left(nd, x) ? nd->left : nd->right;
      append_only(nd, id);
      if (nd->node_size >= (unsigned)leaf_size) split_node_mt(ix, nd, flags);
    }
  }
  free(route);
  free(flags);
  /* sketches of the final leaves, then the leaf order and the ancestor merge */
  int cnt = 0;
  collect_leaves(ix, ix->root, &cnt);
  ix->num_leaves = cnt;
  ix->leaves = (or_node **)malloc(sizeof(or_node *) * (cnt > 0 ? cnt : 1));
  cnt = 0;
  collect_leaves(ix, ix->root, &cnt);
  for (int i = 0; i < cnt; ++i) sketch_members(ix, ix->leaves[i], threads);
  ix->ids = (int64_t *)malloc(sizeof(int64_t) * (n ? n : 1));
  uint64_t pos = 0;
  for (int i = 0; i < cnt; ++i) {
    or_node *lf = ix->leaves[i];
    lf->file_pos = pos;
    for (unsigned m = 0; m < lf->node_size; ++m) ix->ids[pos + m] = lf->members[m];
    pos += lf->node_size;
    merge_ancestors(lf);
  }
  if (keep_rows) {
    ix->rows = (float *)malloc(sizeof(float) * L * (n ? n : 1));
    ix->owns_rows = 1;
#ifdef _OPENMP
#pragma omp parallel for schedule(static, 1024) num_threads(threads)
#endif
    for (int64_t r = 0; r < (int64_t)n; ++r)
      memcpy(ix->rows + (uint64_t)r * L, data + (uint64_t)ix->ids[r] * L, sizeof(float) * L);
    ix->data = NULL;
  }
  /* without rows, ix->data stays the caller's matrix until or_write */
  return ix;
}

/* ---------------------------------------------------------------------- */
/* on-disk format                                                          */
/* ---------------------------------------------------------------------- */

/* Leaf-ordered row r: the resident copy, or the caller's matrix after
 * or_build_mt without rows. */
static const float *leaf_row(const or_index *ix, uint64_t r) {
  return ix->rows ? ix->rows + r * ix->L : ix->data + (uint64_t)ix->ids[r] * ix->L;
}

static void write_node(or_index *ix, or_node *n, FILE *f, FILE *raw, FILE *sims, const float *bp,
                       uint64_t *leaves_written, const unsigned char *words) {
  unsigned char is_leaf = (unsigned char)n->is_leaf;
  fwrite(&is_leaf, 1, 1, f);
  fwrite(&n->level, 4, 1, f);
  if (!n->is_leaf) {
    write_node(ix, n->left, f, raw, sims, bp, leaves_written, words);
    write_node(ix, n->right, f, raw, sims, bp, leaves_written, words);
    fwrite(&n->node_size, 4, 1, f);
    short split_segment = -1;
    fwrite(&split_segment, 2, 1, f);
    /* struct node_split_policy, 48 bytes (hercules_node_split.h:21-34):
     * i16 from, i16 to, {f32 value, i32 idx}, i32 idx, f32 value, then
     * padding and a struct of two pointers whose bytes are not meaningful
     * (written as zeros here). */
    unsigned char pol[48];
    memset(pol, 0, sizeof pol);
    memcpy(pol + 0, &n->split_from, 2);
    memcpy(pol + 2, &n->split_to, 2);
    memcpy(pol + 4, &n->split_value, 4);
    memcpy(pol + 8, &n->split_idx, 4);
    memcpy(pol + 12, &n->split_idx, 4);
    memcpy(pol + 16, &n->split_value, 4);
    fwrite(pol, 1, 48, f);
    short ns = (short)n->nseg;
    fwrite(&ns, 2, 1, f);
    fwrite(n->points, 2, n->nseg, f);
    for (int i = 0; i < n->nseg; ++i) {
      int four = 4;
      fwrite(&four, 4, 1, f);
      fwrite(n->sk + 4 * i, 4, 4, f);
    }
  } else {
    fwrite(&n->node_size, 4, 1, f);
    int len = (int)strlen(n->filename);
    fwrite(&len, 4, 1, f);
    fwrite(n->filename, 1, len, f);
    short ns = (short)n->nseg;
    fwrite(&ns, 2, 1, f);
    fwrite(n->points, 2, n->nseg, f);
    for (int i = 0; i < n->nseg; ++i) {
      int four = 4;
      fwrite(&four, 4, 1, f);
      fwrite(n->sk + 4 * i, 4, 4, f);
    }
    fwrite(&n->file_pos, 8, 1, f);
    for (unsigned m = 0; m < n->node_size; ++m) {
      const float *x = leaf_row(ix, n->file_pos + m);
      fwrite(x, 4, ix->L, raw);
      if (words) {
        fwrite(words + (n->file_pos + m) * OR_PAA_SEGMENTS, 1, OR_PAA_SEGMENTS, sims);
      } else {
        unsigned char w[OR_PAA_SEGMENTS];
        or_sax(x, w, ix->L, bp);
        fwrite(w, 1, OR_PAA_SEGMENTS, sims);
      }
    }
    ++(*leaves_written);
  }
}

static FILE *open_in(const char *dir, const char *name, const char *mode) {
  char path[4096];
  snprintf(path, sizeof path, "%s%s", dir, name);
  return fopen(path, mode);
}

int or_write(or_index *ix, const char *dir, double buffer_mb, const float *bp255) {
  FILE *f = open_in(dir, "root.idx", "wb");
  FILE *raw = open_in(dir, "leaves_raw.idx", "wb");
  FILE *sims = open_in(dir, "leaves_sims.idx", "wb");
  if (!f || !raw || !sims) {
    if (f) fclose(f);
    if (raw) fclose(raw);
    if (sims) fclose(sims);
    return -1;
  }
  uint64_t leaves = 0;
  unsigned int L = ix->L, init_segments = 1, leaf = ix->leaf_size;
  int paa = OR_PAA_SEGMENTS, card = 8, serial = 1, sims_flag = 1;
  fwrite(&leaves, 8, 1, f);
  fwrite(&buffer_mb, 8, 1, f);
  fwrite(&L, 4, 1, f);
  fwrite(&init_segments, 4, 1, f);
  fwrite(&paa, 4, 1, f);
  fwrite(&card, 4, 1, f);
  fwrite(&leaf, 4, 1, f);
  fwrite(&serial, 4, 1, f);
  fwrite(&sims_flag, 4, 1, f);
  /* the multi-threaded build: iSAX words of every row in parallel first,
   * and large stdio buffers for the two data files */
  unsigned char *words = NULL;
  if (ix->threads > 0) {
    setvbuf(raw, NULL, _IOFBF, (size_t)1 << 24);
    setvbuf(sims, NULL, _IOFBF, (size_t)1 << 22);
    words = (unsigned char *)malloc((size_t)OR_PAA_SEGMENTS * (ix->n ? ix->n : 1));
#ifdef _OPENMP
#pragma omp parallel for schedule(static, 1024) num_threads(ix->threads)
#endif
    for (int64_t r = 0; r < (int64_t)ix->n; ++r)
      or_sax(leaf_row(ix, (uint64_t)r), words + (uint64_t)r * OR_PAA_SEGMENTS, ix->L, bp255);
  }
  write_node(ix, ix->root, f, raw, sims, bp255, &leaves, words);
  free(words);
  fseek(f, 0, SEEK_SET);
  fwrite(&leaves, 8, 1, f);
  fclose(f);
  fclose(raw);
  fclose(sims);
  return 0;
}

#define RD(ptr, sz, cnt) \
  do { if (fread((ptr), (sz), (cnt), f) != (size_t)(cnt)) return NULL; } while (0)

static or_node *read_node(or_index *ix, FILE *f, or_node *parent) {
  unsigned char is_leaf;
  or_node *n = (or_node *)calloc(1, sizeof(or_node));
  n->parent = parent;
  RD(&is_leaf, 1, 1);
  RD(&n->level, 4, 1);
  n->is_leaf = is_leaf;
  ix->num_nodes++;
  if (!is_leaf) {
    n->left = read_node(ix, f, n);
    n->right = read_node(ix, f, n);
    if (!n->left || !n->right) return NULL;
    short split_segment, ns;
    unsigned char pol[48];
    RD(&n->node_size, 4, 1);
    RD(&split_segment, 2, 1);
    RD(pol, 1, 48);
    memcpy(&n->split_from, pol + 0, 2);
    memcpy(&n->split_to, pol + 2, 2);
    memcpy(&n->split_idx, pol + 12, 4);
    memcpy(&n->split_value, pol + 16, 4);
    RD(&ns, 2, 1);
    n->nseg = ns;
    n->points = (short *)malloc(sizeof(short) * (ns > 0 ? ns : 1));
    RD(n->points, 2, ns);
    n->sk = (float *)malloc(sizeof(float) * 4 * (ns > 0 ? ns : 1));
    for (int i = 0; i < ns; ++i) {
      int ni;
      RD(&ni, 4, 1);
      if (ni != 4) return NULL;
      RD(n->sk + 4 * i, 4, 4);
    }
  } else {
    int len;
    RD(&n->node_size, 4, 1);
    RD(&len, 4, 1);
    if (len > 0) {
      n->filename = (char *)malloc(len + 1);
      RD(n->filename, 1, len);
      n->filename[len] = 0;
      short ns;
      RD(&ns, 2, 1);
      n->nseg = ns;
      n->points = (short *)malloc(sizeof(short) * (ns > 0 ? ns : 1));
      RD(n->points, 2, ns);
      n->sk = (float *)malloc(sizeof(float) * 4 * (ns > 0 ? ns : 1));
      for (int i = 0; i < ns; ++i) {
        int ni;
        RD(&ni, 4, 1);
        if (ni != 4) return NULL;
        RD(n->sk + 4 * i, 4, 4);
      }
      RD(&n->file_pos, 8, 1);
    } else {
      n->node_size = 0;
    }
  }
  return n;
}

or_index *or_read(const char *dir) {
  FILE *f = open_in(dir, "root.idx", "rb");
  if (!f) return NULL;
  or_index *ix = (or_index *)calloc(1, sizeof(or_index));
  uint64_t leaves;
  double buffer_mb;
  unsigned int L, init_segments, leaf;
  int paa, card, serial, sims;
  int ok = fread(&leaves, 8, 1, f) == 1 && fread(&buffer_mb, 8, 1, f) == 1 &&
           fread(&L, 4, 1, f) == 1 && fread(&init_segments, 4, 1, f) == 1 &&
           fread(&paa, 4, 1, f) == 1 && fread(&card, 4, 1, f) == 1 &&
           fread(&leaf, 4, 1, f) == 1 && fread(&serial, 4, 1, f) == 1 &&
           fread(&sims, 4, 1, f) == 1;
  if (!ok || paa != OR_PAA_SEGMENTS || card != 8 || L % 16 != 0) {
    fclose(f);
    free(ix);
    return NULL;
  }
  ix->L = (int)L;
  ix->leaf_size = (int)leaf;
  ix->root = read_node(ix, f, NULL);
  fclose(f);
  if (!ix->root) {
    free(ix);
    return NULL;
  }
  int cnt = 0;
  collect_leaves(ix, ix->root, &cnt);
  ix->num_leaves = cnt;
  ix->leaves = (or_node **)malloc(sizeof(or_node *) * (cnt > 0 ? cnt : 1));
  cnt = 0;
  collect_leaves(ix, ix->root, &cnt);
  uint64_t n = 0;
  for (int i = 0; i < cnt; ++i) n += ix->leaves[i]->node_size;
  ix->n = n;
  FILE *raw = open_in(dir, "leaves_raw.idx", "rb");
  if (!raw) {
    or_free(ix);
    return NULL;
  }
  ix->rows = (float *)malloc(sizeof(float) * L * (n ? n : 1));
  ix->owns_rows = 1;
  size_t got = fread(ix->rows, sizeof(float) * L, n, raw);
  fclose(raw);
  if (got != n) {
    or_free(ix);
    return NULL;
  }
  ix->ids = (int64_t *)malloc(sizeof(int64_t) * (n ? n : 1));
  for (uint64_t r = 0; r < n; ++r) ix->ids[r] = (int64_t)r;
  return ix;
}

static void free_node(or_node *n) {
  if (!n) return;
  free_node(n->left);
  free_node(n->right);
  free(n->points);
  free(n->hs_points);
  free(n->sk);
  free(n->hs_sk);
  free(n->members);
  free(n->filename);
  free(n);
}

void or_free(or_index *ix) {
  if (!ix) return;
  free_node(ix->root);
  free(ix->leaves);
  if (ix->owns_rows) free(ix->rows);
  free(ix->ids);
  free(ix);
}

int or_num_leaves(const or_index *ix) { return ix->num_leaves; }
int or_num_nodes(const or_index *ix) { return ix->num_nodes; }
int or_L(const or_index *ix) { return ix->L; }
uint64_t or_num_rows(const or_index *ix) { return ix->n; }
const float *or_rows(const or_index *ix) { return ix->rows; }

void or_leaf_info(const or_index *ix, int i, uint64_t *file_pos, uint32_t *size, int *nseg,
                  short *points, float *sk) {
  const or_node *lf = ix->leaves[i];
  if (file_pos) *file_pos = lf->file_pos;
  if (size) *size = lf->node_size;
  if (nseg) *nseg = lf->nseg;
  if (points) memcpy(points, lf->points, sizeof(short) * lf->nseg);
  if (sk) memcpy(sk, lf->sk, sizeof(float) * 4 * lf->nseg);
}

void or_row_ids(const or_index *ix, int64_t *ids_out) {
  memcpy(ids_out, ix->ids, sizeof(int64_t) * ix->n);
}

void or_leaf_lbs(const or_index *ix, const float *q, float *lb_out) {
  for (int i = 0; i < ix->num_leaves; ++i) {
    const or_node *lf = ix->leaves[i];
    lb_out[i] = or_lb_eapca(q, lf->nseg, lf->points, lf->sk);
  }
}

/* ---------------------------------------------------------------------- */
/* exact search                                                            */
/* ---------------------------------------------------------------------- */

typedef struct {
  float d;
  or_node *n;
} pq_item;

typedef struct {
  pq_item *a;
  int n, cap;
} pq_t;

static void pq_push(pq_t *q, pq_item it) {
  if (q->n == q->cap) {
    q->cap = q->cap ? q->cap * 2 : 64;
    q->a = (pq_item *)realloc(q->a, sizeof(pq_item) * q->cap);
  }
  int i = q->n++;
  q->a[i] = it;
  while (i > 0) {
    int p = (i - 1) / 2;
    if (q->a[p].d <= q->a[i].d) break;
    pq_item t = q->a[p];
    q->a[p] = q->a[i];
    q->a[i] = t;
    i = p;
  }
}

static int pq_pop(pq_t *q, pq_item *out) {
  if (q->n == 0) return 0;
  *out = q->a[0];
  q->a[0] = q->a[--q->n];
  int i = 0;
  for (;;) {
    int l = 2 * i + 1, r = l + 1, m = i;
    if (l < q->n && q->a[l].d < q->a[m].d) m = l;
    if (r < q->n && q->a[r].d < q->a[m].d) m = r;
    if (m == i) break;
    pq_item t = q->a[m];
    q->a[m] = q->a[i];
    q->a[i] = t;
    i = m;
  }
  return 1;
}

static int cmp_cand(const void *a, const void *b) {
  const pq_item *x = (const pq_item *)a, *y = (const pq_item *)b;
  return x->n->file_pos < y->n->file_pos ? -1 : (x->n->file_pos > y->n->file_pos ? 1 : 0);
}

/* One leaf of the scan (hercules_query_engine.c:2391-2425).  The list keys
 * are dataset ids (the tie rule compares them); aux carries the leaf-ordered
 * row. */
static void scan_leaf(const or_index *ix, const or_node *lf, const float *q, int k, int tie,
                      float *dist, int64_t *id, uint64_t *row, int *cur, float *kth_var) {
  for (unsigned m = 0; m < lf->node_size; ++m) {
    uint64_t r = lf->file_pos + m;
    float kth = dist[k - 1];
    *kth_var = kth;
    const float *x = ix->rows + r * ix->L;
    float d = or_ed(q, x, ix->L, kth);
    if (d < kth) {
      or_topk_insert(dist, id, row, cur, k, d, ix->ids[r], r, tie);
    } else if (tie && d == kth && *cur == k) {
      /* lowest-id rule: a row whose partial sum reached exactly kth may
       * still tie it */
      float full = or_ed(q, x, ix->L, FLT_MAX);
      if (full == kth) or_topk_insert(dist, id, row, cur, k, full, ix->ids[r], r, tie);
    }
  }
}

static uint64_t leaf_pos_of_row(const or_index *ix, uint64_t r) {
  int lo = 0, hi = ix->num_leaves - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) / 2;
    if (ix->leaves[mid]->file_pos <= r) lo = mid;
    else hi = mid - 1;
  }
  while (lo > 0 && ix->leaves[lo]->node_size == 0) --lo;
  return ix->leaves[lo]->file_pos;
}

/* hercules_query_engine.c:2215-2448 with epsilon = 0 and
 * approximate_knn_search (:176-222). */
int or_exact_knn(const or_index *ix, const float *q, int k, int tie_lowest, float *d_out,
                 int64_t *row_out, uint64_t *filepos_out, or_stats *st) {
  if (k <= 0 || !ix->root) return -1;
  float *dist = (float *)malloc(sizeof(float) * k);
  int64_t *id = (int64_t *)malloc(sizeof(int64_t) * k);
  uint64_t *row = (uint64_t *)malloc(sizeof(uint64_t) * k);
  for (int i = 0; i < k; ++i) {
    dist[i] = FLT_MAX;
    id[i] = -1;
    row[i] = UINT64_MAX;
  }
  int cur = 0;
  or_stats s;
  memset(&s, 0, sizeof s);
  float kth_var = FLT_MAX;

  /* approximate search: route to one leaf and scan it */
  or_node *n = ix->root;
  while (!n->is_leaf) n = route_left(n, q) ? n->left : n->right;
  const or_node *approx = n;
  scan_leaf(ix, n, q, k, tie_lowest, dist, id, row, &cur, &kth_var);
  s.loaded_leaves = 1;
  s.loaded_rows = n->node_size;
  s.approx_leaf = (uint32_t)n->leaf_index;
  /* the reference excludes knn_results[0].node, which is the approximate
   * leaf whenever that leaf produced a result */
  const or_node *approx_node = (cur > 0) ? approx : NULL;

  /* best-first LB_EAPCA traversal collecting candidate leaves */
  pq_t pq = {0, 0, 0};
  pq_item *cand = (pq_item *)malloc(sizeof(pq_item) * (ix->num_leaves + 1));
  int ncand = 0;
  pq_item root = {or_lb_eapca(q, ix->root->nseg, ix->root->points, ix->root->sk), ix->root};
  pq_push(&pq, root);
  pq_item it;
  while (pq_pop(&pq, &it)) {
    float kth = dist[k - 1];
    kth_var = kth;
    if (tie_lowest ? (it.d > kth) : (it.d > kth)) break;
    if (it.n->is_leaf) {
      cand[ncand++] = it;
    } else {
      or_node *ch[2] = {it.n->left, it.n->right};
      for (int c = 0; c < 2; ++c) {
        float lb = or_lb_eapca(q, ch[c]->nseg, ch[c]->points, ch[c]->sk);
        int pass = tie_lowest ? (lb <= kth) : (lb < kth);
        if (pass && ch[c] != approx_node) pq_push(&pq, (pq_item){lb, ch[c]});
      }
    }
  }
  free(pq.a);
  s.candidate_leaves = (uint32_t)ncand;
  qsort(cand, ncand, sizeof(pq_item), cmp_cand);
  for (int i = 0; i < ncand; ++i) {
    if (cand[i].d <= kth_var) {
      s.loaded_leaves++;
      s.loaded_rows += cand[i].n->node_size;
      scan_leaf(ix, cand[i].n, q, k, tie_lowest, dist, id, row, &cur, &kth_var);
    }
  }
  free(cand);
  for (int i = 0; i < k; ++i) {
    d_out[i] = dist[i];
    if (row_out) row_out[i] = i < cur ? (int64_t)row[i] : -1;
    if (filepos_out) filepos_out[i] = i < cur ? leaf_pos_of_row(ix, row[i]) : 0;
  }
  if (st) *st = s;
  free(dist);
  free(id);
  free(row);
  return cur;
}

/* The approximate searches of the reference's serial query path
 * (hercules_file_loaders.c:230-243 dispatch):
 *  - nprobes > 0: exact_ng_knn_search (hercules_query_engine.c:2623-2796):
 *    best-first over node LBs, a leaf scanned as soon as it is popped, at
 *    most nprobes leaves including the approximate one; stops when a popped
 *    node's LB exceeds the approximate search's best distance; children are
 *    pushed when LB < the current k-th distance;
 *  - else exact_de_knn_search with epsilon (:2215-2448): the traversal
 *    collects leaves with the k-th distance of the approximate leaf fixed
 *    (break when LB > kth/(1+eps), push when LB < kth/(1+eps)), then scans
 *    them in file_pos order, each only if LB <= kth/(1+eps) with the k-th
 *    distance of that moment.  r_delta is not used on this path.
 * The comparisons are the reference's in both tie modes; tie_lowest only
 * changes the top-k insert (lowest id on an exact FP32 tie). */
int or_approx_knn(const or_index *ix, const float *q, int k, int tie_lowest, float epsilon, int nprobes,
                  float *d_out, int64_t *row_out, uint64_t *filepos_out, or_stats *st) {
  if (k <= 0 || !ix->root) return -1;
  float *dist = (float *)malloc(sizeof(float) * k);
  int64_t *id = (int64_t *)malloc(sizeof(int64_t) * k);
  uint64_t *row = (uint64_t *)malloc(sizeof(uint64_t) * k);
  for (int i = 0; i < k; ++i) {
    dist[i] = FLT_MAX;
    id[i] = -1;
    row[i] = UINT64_MAX;
  }
  int cur = 0;
  or_stats s;
  memset(&s, 0, sizeof s);
  float kth_var = FLT_MAX;
  or_node *n = ix->root;
  while (!n->is_leaf) n = route_left(n, q) ? n->left : n->right;
  const or_node *approx = n;
  scan_leaf(ix, n, q, k, tie_lowest, dist, id, row, &cur, &kth_var);
  s.loaded_leaves = 1;
  s.loaded_rows = n->node_size;
  s.approx_leaf = (uint32_t)n->leaf_index;
  const or_node *approx_node = (cur > 0) ? approx : NULL;
  const float approx_best = dist[0];
  const float eps1 = 1.0f + epsilon;
  pq_t pq = {0, 0, 0};
  pq_item *cand = (pq_item *)malloc(sizeof(pq_item) * (ix->num_leaves + 1));
  int ncand = 0;
  pq_item root = {or_lb_eapca(q, ix->root->nseg, ix->root->points, ix->root->sk), ix->root};
  pq_push(&pq, root);
  pq_item it;
  if (nprobes > 0) {
    int probes = 1;
    while (pq_pop(&pq, &it) && probes < nprobes) {
      if (it.d > approx_best) break;
      if (it.n->is_leaf) {
        s.loaded_leaves++;
        s.loaded_rows += it.n->node_size;
        scan_leaf(ix, it.n, q, k, tie_lowest, dist, id, row, &cur, &kth_var);
        ++probes;
      } else {
        const float kth = dist[k - 1];
        or_node *ch[2] = {it.n->left, it.n->right};
        for (int c = 0; c < 2; ++c) {
          const float lb = or_lb_eapca(q, ch[c]->nseg, ch[c]->points, ch[c]->sk);
          if (lb < kth && ch[c] != approx_node) pq_push(&pq, (pq_item){lb, ch[c]});
        }
      }
    }
  } else {
    while (pq_pop(&pq, &it)) {
      const float kth = dist[k - 1];
      kth_var = kth;
      if (it.d > kth / eps1) break;
      if (it.n->is_leaf) {
        cand[ncand++] = it;
      } else {
        or_node *ch[2] = {it.n->left, it.n->right};
        for (int c = 0; c < 2; ++c) {
          const float lb = or_lb_eapca(q, ch[c]->nseg, ch[c]->points, ch[c]->sk);
          if (lb < kth / eps1 && ch[c] != approx_node) pq_push(&pq, (pq_item){lb, ch[c]});
        }
      }
    }
    s.candidate_leaves = (uint32_t)ncand;
    qsort(cand, ncand, sizeof(pq_item), cmp_cand);
    for (int i = 0; i < ncand; ++i) {
      if (cand[i].d <= kth_var / eps1) {
        s.loaded_leaves++;
        s.loaded_rows += cand[i].n->node_size;
        scan_leaf(ix, cand[i].n, q, k, tie_lowest, dist, id, row, &cur, &kth_var);
      }
    }
  }
  free(pq.a);
  free(cand);
  for (int i = 0; i < k; ++i) {
    d_out[i] = dist[i];
    if (row_out) row_out[i] = i < cur ? (int64_t)row[i] : -1;
    if (filepos_out) filepos_out[i] = i < cur ? leaf_pos_of_row(ix, row[i]) : 0;
  }
  if (st) *st = s;
  free(dist);
  free(id);
  free(row);
  return cur;
}

int or_pscan(const float *data, uint64_t n, int L, const float *q, int k, int tie_lowest,
             float *d_out, int64_t *id_out) {
  float *dist = (float *)malloc(sizeof(float) * k);
  int64_t *id = (int64_t *)malloc(sizeof(int64_t) * k);
  for (int i = 0; i < k; ++i) {
    dist[i] = FLT_MAX;
    id[i] = -1;
  }
  int cur = 0;
  for (uint64_t r = 0; r < n; ++r) {
    float kth = dist[k - 1];
    float d = or_ed(q, data + r * L, L, kth);
    if (d < kth) or_topk_insert(dist, id, NULL, &cur, k, d, (int64_t)r, 0, tie_lowest);
  }
  memcpy(d_out, dist, sizeof(float) * k);
  memcpy(id_out, id, sizeof(int64_t) * k);
  free(dist);
  free(id);
  return cur;
}
