/*
 * hercules_oracle.h -- CPU restatement of the Hercules exact k-NN query path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the parity checker for the
 * B200 implementation in hercules_b200/.  Only tests/, __graft_entry__.smoke()
 * and bench.py's cpu_baseline / --impl reference legs may load it; the
 * product path never calls into it.
 *
 * Every function restates one function of the reference C code
 * (karimaechihabi/hercules, code/hercules) in plain scalar C with the
 * reference's exact floating-point operation order.  The library is compiled
 * with -ffp-contract=off so that no multiply-add is fused: the result is the
 * literal ISO-C arithmetic of the reference source.  Parity is pinned by the
 * tests against the reference sources compiled from their own files
 * (oracle/Makefile, target `ref`).
 */
#ifndef HERCULES_ORACLE_H
#define HERCULES_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define OR_PAA_SEGMENTS 16
#define OR_SAX_CARD 256

/* --- primitives ------------------------------------------------------- */

/* ts_euclidean_distance_SIMD, code/hercules/src/ts.c:83-109 */
float or_ed(const float *t, const float *s, int L, float bound);

/* calc_mean_stdev_SIMD, code/hercules/src/calc_utils.c:48-112 */
void or_mean_stdev(const float *series, int start, int end, float *mean, float *stdev);

/* paa_from_ts, code/hercules/src/sax.c:46-56 (16 segments) */
void or_paa(const float *ts, float *paa, int L);

/* sax_from_ts, code/hercules/src/sax.c:86-135 (16 segments, 8 bits) */
void or_sax(const float *ts, unsigned char *sax, int L, const float *bp255);

/* minidist_paa_to_isax_raw_SIMD, code/hercules/src/sax.c:310-479 */
float or_lb_sax(const float *paa, const unsigned char *sax, int L, const float *bp255);

/* calculate_node_min_distance, code/hercules/src/hercules_node.c:879-924;
 * sk holds nseg x {mean_max, mean_min, stdev_max, stdev_min}. */
float or_lb_eapca(const float *q, int nseg, const short *points, const float *sk);

/* queue_bounded_sorted_insert, code/hercules/src/hercules_query_engine.c:4034-4082.
 * tie_lowest=0: reference rule (an equal distance is dropped).
 * tie_lowest=1: an equal distance keeps the lower id. */
void or_topk_insert(float *dist, int64_t *id, uint64_t *aux, int *cur, int k,
                    float d, int64_t cid, uint64_t caux, int tie_lowest);

/* --- index ------------------------------------------------------------ */

typedef struct or_index or_index;

/* hercules_index_build with one insert worker (hercules_index.c:2354-2927,
 * hercules_node_split.c:1043-1345).  data is row-major n x L. */
or_index *or_build(const float *data, uint64_t n, int L, int leaf_size);

/* or_build on `threads` threads (0 = every core): the same tree, leaf order
 * and floats.  keep_rows = 0 keeps no leaf-ordered copy of the rows: data
 * must then stay valid until or_write, which reads the rows from it. */
or_index *or_build_mt(const float *data, uint64_t n, int L, int leaf_size, int threads, int keep_rows);

/* hercules_index_write_sequential (hercules_index.c:1611-1692, 1967-2077,
 * hercules_file_buffer.c:539-583).  dir must end with '/'. */
int or_write(or_index *ix, const char *dir, double buffer_mb, const float *bp255);

/* hercules_index_read (hercules_index.c:1793-1905, 2188-2340) plus the
 * leaves_raw.idx content resident in memory. */
or_index *or_read(const char *dir);

void or_free(or_index *ix);

int or_num_leaves(const or_index *ix);
int or_num_nodes(const or_index *ix);
int or_L(const or_index *ix);
uint64_t or_num_rows(const or_index *ix);
/* leaf i in DFS order: file_pos and size */
void or_leaf_info(const or_index *ix, int i, uint64_t *file_pos, uint32_t *size,
                  int *nseg, short *points /* >= nseg */, float *sk /* >= 4*nseg */);
/* seeded synthetic data (oracle_gen.c): rows [first, first+n) of stream
 * seed -- random walks (unit = 0) or unit vectors (unit = 1) -- and noisy
 * queries whose base rows are regenerated from data_seed */
void or_gen_rows(uint64_t seed, uint64_t first, uint64_t n, int L, float *out, int unit, int threads);
void or_gen_queries(uint64_t data_seed, uint64_t seed, uint64_t n, int L, int nq, const double *sigma2, float *out,
                    uint64_t *base_ids, int unit);

/* dataset id of leaf-ordered row r (valid after or_build) */
void or_row_ids(const or_index *ix, int64_t *ids_out);
/* leaf-ordered raw rows (valid after or_build or or_read) */
const float *or_rows(const or_index *ix);

typedef struct {
  uint32_t loaded_leaves;     /* leaves scanned, approximate leaf included */
  uint64_t loaded_rows;       /* rows scanned */
  uint32_t candidate_leaves;  /* leaves collected by the LB_EAPCA traversal */
  uint32_t approx_leaf;       /* DFS index of the approximate-search leaf */
} or_stats;

/* exact_de_knn_search, hercules_query_engine.c:2215-2448 (epsilon = 0).
 * Outputs k squared distances (ascending), the leaf-ordered row of each
 * answer and its leaf's file_pos.  tie_lowest selects the tie rule. */
/* epsilon-approximate (nprobes == 0) or nprobes search of the reference's
 * serial path (exact_de_knn_search with epsilon, exact_ng_knn_search). */
int or_approx_knn(const or_index *ix, const float *q, int k, int tie_lowest, float epsilon, int nprobes,
                  float *d_out, int64_t *row_out, uint64_t *filepos_out, or_stats *st);
int or_exact_knn(const or_index *ix, const float *q, int k, int tie_lowest,
                 float *d_out, int64_t *row_out, uint64_t *filepos_out, or_stats *st);

/* LB_EAPCA of every leaf (DFS order) for query q */
void or_leaf_lbs(const or_index *ix, const float *q, float *lb_out);

/* PSCAN, code/pscan/src/parallel_scan_utils.c:205-481: scan all n rows in
 * file order with the early-abandoning distance and the top-k insert. */
int or_pscan(const float *data, uint64_t n, int L, const float *q, int k, int tie_lowest,
             float *d_out, int64_t *id_out);

#ifdef __cplusplus
}
#endif
#endif
