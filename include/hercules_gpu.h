/*
 * hercules_gpu.h -- C ABI of the B200-native Hercules exact k-NN path.
 *
 * libhercules_gpu.so replaces the exact k-NN query path of the Hercules C
 * library (karimaechihabi/hercules, code/hercules) with sm_100a kernels and
 * keeps its index format and semantics.  Each entry point names the
 * reference interface it replaces.  Plain C types and pointers only; every
 * call returns an hg_status and never exits the process; every device wait
 * is bounded.  A handle owns one CUDA stream and is not re-entrant: calls on
 * one handle must not overlap (the reference's query entry is not
 * re-entrant either, hercules_query_engine.c mutates index->stats).
 *
 * Conventions
 *   - series are float32 rows of length L (L a multiple of 16);
 *   - distances are squared Euclidean distances in float32, computed in the
 *     reference's summation order (ts_euclidean_distance_SIMD, ts.c:83-109);
 *   - a result list holds the k smallest DISTINCT distances; for each the
 *     row with the lowest dataset id among rows at exactly that distance;
 *     missing entries (fewer than k rows) have distance +inf and id -1.
 */
#ifndef HERCULES_GPU_H
#define HERCULES_GPU_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define HG_API __attribute__((visibility("default")))
#else
#define HG_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef int hg_status;
#define HG_OK 0
#define HG_ERR_ARG (-1)      /* invalid argument */
#define HG_ERR_IO (-2)       /* file missing, short read or write */
#define HG_ERR_FORMAT (-3)   /* root.idx not in the reference's format */
#define HG_ERR_CUDA (-4)     /* CUDA runtime error (no device, launch failure) */
#define HG_ERR_NOMEM (-5)    /* host or device allocation failed */
#define HG_ERR_TIMEOUT (-6)  /* a bounded device wait gave up */
#define HG_ERR_LIMIT (-7)    /* a size beyond a documented limit */

typedef struct hg_index hg_index;

/* Index-wide facts (hercules_index_settings, hercules_index.h). */
typedef struct {
  uint64_t num_series;    /* dataset size */
  uint32_t ts_length;     /* timeseries_size */
  uint32_t leaf_size;     /* max_leaf_size */
  uint32_t num_leaves;    /* leaf_nodes_count */
  uint32_t num_nodes;     /* total nodes */
  uint32_t max_segments;  /* most EAPCA segments in any leaf */
  uint32_t has_ids;       /* 1 when row -> dataset id is known */
  uint64_t device_bytes;  /* HBM held by the index */
} hg_index_info;

/* Per-call query counters (the Query_* TSV fields of print_query_stats,
 * hercules_query_engine.c:3558-3918, that this path defines). */
typedef struct {
  uint64_t queries;
  uint64_t leaves_scanned;    /* Query_total_loaded_nodes_count, summed */
  uint64_t rows_visited;      /* rows whose distance computation started */
  uint64_t rows_lbsax_pruned; /* rows of candidate leaves skipped by LB_SAX */
  uint64_t chunks_loaded;     /* 32-byte chunks of raw data read by the scan */
  uint64_t candidate_leaves;  /* leaves with LB_EAPCA <= k-th bound */
  double device_ms;           /* device time of the call (CUDA events) */
  uint64_t rows_completed;    /* rows whose full distance was computed */
  uint64_t scan_launches;     /* distance-kernel launches (profile = 1) */
  double scan_ms;             /* their summed device time (profile = 1) */
  uint64_t rows_considered;   /* rows of candidate leaves seen by the LB_SAX filter */
  uint64_t filter_launches;   /* LB_SAX filter launches (profile = 1) */
  double filter_ms;           /* their summed device time (profile = 1) */
  /* batched path (HG_MODE_BATCH, hg_knn_batch) */
  uint64_t bf16_pairs;        /* (query, row) pairs through the BF16 filter */
  uint64_t survivors;         /* pairs kept by the certified filter */
  uint64_t fallback_queries;  /* queries answered by the plain path instead */
  uint64_t retried_queries;   /* filter passes repeated with a tighter bound (bucket overflow) */
  double bound_ms;            /* device time: BF16 pass over the approximate leaves + bound */
  double gemm_ms;             /* device time: BF16 filter over every row */
  double rerank_ms;           /* device time: exact re-rank of the survivors */
  double fallback_ms;         /* device time: plain path for the fallback queries */
  uint64_t kernel_launches;   /* kernels this library launched for the call */
  /* batched path: the certified error bound err(q, item) of the filter pass
   * over every row, over its (work item, query) pairs with a finite bound */
  double err_mean;            /* mean err */
  double err_max;             /* largest err */
  double err_over_bound;      /* mean err / B_q (B_q > 0) */
  uint64_t leaf_pairs;        /* batched path: (query, non-empty leaf) pairs */
  uint64_t leaf_pairs_kept;   /* of those, the pairs LB_EAPCA keeps for the filter
                                 (LB <= the query's bound) */
} hg_query_stats;

/* Search mode. */
#define HG_MODE_PLAIN 0    /* exact_de_knn_search per query */
#define HG_MODE_PSCAN 1    /* parallel scan of every row (code/pscan) */
#define HG_MODE_BATCH 2    /* all queries at once: BF16 tensor-core filter with a
                              certified error bound + exact FP32 re-rank */

typedef struct {
  int mode;           /* HG_MODE_* */
  int use_lb_sax;     /* 1: per-row LB_SAX filter before the distance */
  int profile;        /* 1: time every leaf-scan launch with CUDA events */
  int approx_blocks;  /* blocks of the approximate-leaf scan (0 = two per SM) */
  int bucket_cap;     /* HG_MODE_BATCH: filter survivors kept per query before the
                         query falls back to the plain path (0 = 65536) */
  int dense_filter;   /* HG_MODE_BATCH: 1 = filter every row against every query
                         (no LB_EAPCA leaf pruning before the filter) */
  float epsilon;      /* HG_MODE_PLAIN, > 0: epsilon-approximate search of
                         exact_de_knn_search (hercules_query_engine.c:2215-2448):
                         leaves pruned at LB > kth / (1 + epsilon) */
  int nprobes;        /* HG_MODE_PLAIN, > 0: exact_ng_knn_search (:2623-2796):
                         at most nprobes leaves, best-first; takes precedence
                         over epsilon like the reference's dispatch */
  int approx_leaves;  /* HG_MODE_PLAIN exact search, > 1: greedy seeding with
                         L_max = approx_leaves leaves (the paper's L_max;
                         approximate_greedy_knn_search, :70-174, with
                         --approx-stop-condition): after the routed leaf, the
                         approx_leaves - 1 other leaves of smallest LB_EAPCA
                         are scanned first, best-first, so the k-th distance
                         the remaining candidates are filtered against is
                         tighter.  0 or 1: the routed leaf only, as the
                         reference's serial exact search.  The answers do not
                         depend on it. */
} hg_knn_opts;

/* ---- status ----------------------------------------------------------- */

/* Text for a status code. */
HG_API const char *hg_status_string(hg_status s);

/* Text of the last CUDA/runtime error seen on this thread. */
HG_API const char *hg_last_error(void);

/* ---- index construction ----------------------------------------------- */

/* Builds the index from a raw float32 file of at least n series of length L.
 * Replaces hercules_index_settings_init + hercules_index_init +
 * hercules_root_node_init + hercules_index_build
 * (hercules.c:355-420, hercules_index.c:32-153, 2354-2634) run with one
 * insert worker: the EAPCA tree, leaf order and envelopes are those of the
 * reference.  Routing, envelopes and iSAX words run on `device`. */
HG_API hg_status hg_index_build_file(const char *dataset, uint64_t n, uint32_t L, uint32_t leaf_size,
                              int device, hg_index **out);

/* Same from memory.  data is n x L row-major float32; data_on_device = 1
 * when it already lives on `device` (it is not freed and may be released
 * after the call). */
HG_API hg_status hg_index_build(const float *data, int data_on_device, uint64_t n, uint32_t L,
                         uint32_t leaf_size, int device, hg_index **out);

/* Writes root.idx, leaves_raw.idx and leaves_sims.idx into dir (which must
 * end with '/') in the reference's format (hercules_index_write_sequential,
 * hercules_index.c:1611-1692, 1967-2077), plus leaves_ids.idx (u64 dataset
 * id per row, ignored by the reference).  buffer_mb is recorded in the
 * header like --buffer-size. */
HG_API hg_status hg_index_write(hg_index *ix, const char *dir, double buffer_mb);

/* Loads an index written by the reference or by hg_index_write and makes
 * it resident on `device` (hercules_index_read, hercules_index.c:1793-1905;
 * leaves_raw.idx replaces the per-leaf fread of get_all_time_series_in_node).
 * Without leaves_ids.idx the dataset id of a row is its leaves_raw.idx row. */
HG_API hg_status hg_index_read(const char *dir, int device, hg_index **out);

/* Frees host and device memory (hercules_index_destroy, hercules_index.c:1056). */
HG_API void hg_index_destroy(hg_index *ix);

HG_API hg_status hg_index_info_get(const hg_index *ix, hg_index_info *info);

/* Leaf i (DFS order): first row (file_pos), size and EAPCA segment count. */
HG_API hg_status hg_index_leaf(const hg_index *ix, uint32_t i, uint64_t *file_pos, uint32_t *size,
                        uint32_t *num_segments);

/* Copies leaf i's segment ends (short[num_segments]) and envelopes
 * (float[4*num_segments]: mean max, mean min, stdev max, stdev min). */
HG_API hg_status hg_index_leaf_envelope(const hg_index *ix, uint32_t i, short *points, float *envelope);

/* Copies the dataset id of every leaf-ordered row (int64[num_series]). */
HG_API hg_status hg_index_row_ids(const hg_index *ix, int64_t *ids);

/* Copies rows [first, first+count) of the leaf-ordered data (row-major) and
 * their iSAX words (uint8[count*16]); either output may be NULL. */
HG_API hg_status hg_index_rows(const hg_index *ix, uint64_t first, uint64_t count, float *rows,
                        uint8_t *sax);

/* ---- queries ---------------------------------------------------------- */

/* Exact k-NN for nq queries (row-major nq x L, HOST memory).  Replaces
 * exact_de_knn_search (hercules_query_engine.c:2215-2448) as called per
 * query by hercules_knn_query_binary_file (hercules_file_loaders.c:99-294).
 * Outputs nq x k squared distances (ascending), dataset ids and the
 * file_pos of each answer's leaf (Query_exact_node_file_pos).  Any output
 * pointer may be NULL.  stats may be NULL. */
HG_API hg_status hg_knn(hg_index *ix, const float *queries, uint32_t nq, uint32_t k,
                 const hg_knn_opts *opts, float *dist_out, int64_t *id_out,
                 uint64_t *leaf_pos_out, hg_query_stats *stats);

/* Same with every buffer in device memory of the index's device, ordered
 * on `stream` (a cudaStream_t, NULL = the handle's stream). */
HG_API hg_status hg_knn_device(hg_index *ix, const float *d_queries, uint32_t nq, uint32_t k,
                        const hg_knn_opts *opts, float *d_dist_out, int64_t *d_id_out,
                        void *stream, hg_query_stats *stats);

/* Batched exact k-NN: every query of the call at once, with per-query k.
 * Same answers as hg_knn (bit-identical distances and ids).  The reference
 * answers queries one at a time (hercules_knn_query_binary_file loops over
 * exact_de_knn_search, hercules_file_loaders.c:99-294); this entry point
 * replaces that loop.  A BF16 tensor-core pass computes |q|^2 + |x|^2 - 2 q.x
 * for every (query, row) pair against FP64 norms, keeps the pairs within a
 * certified rounding-error bound of an exact k-th-distance bound taken from
 * the query's approximate leaf, and re-ranks them in FP32 in the reference's
 * order; a query whose survivors overflow opts->bucket_cap goes through the
 * plain path.  ks: k of each query (HOST array, NULL = every query uses
 * kmax), each 1..kmax; outputs are nq x kmax (entries past a query's k are
 * +inf / -1).  HOST buffers; opts->mode is ignored. */
HG_API hg_status hg_knn_batch(hg_index *ix, const float *queries, uint32_t nq, const uint32_t *ks,
                              uint32_t kmax, const hg_knn_opts *opts, float *dist_out, int64_t *id_out,
                              hg_query_stats *stats);

/* Same with queries and outputs in device memory, ordered on `stream`
 * (NULL = the handle's stream); ks stays a host array; d_queries must be
 * 16-byte aligned. */
HG_API hg_status hg_knn_batch_device(hg_index *ix, const float *d_queries, uint32_t nq, const uint32_t *ks,
                                     uint32_t kmax, const hg_knn_opts *opts, float *d_dist_out,
                                     int64_t *d_id_out, void *stream, hg_query_stats *stats);

/* Diagnostics (no counterpart in the reference): the batched filter's
 * tensor-core products q~.x~ -- BF16 roundings of every query and row,
 * multiplied on the tensor cores with FP32 accumulation -- of nq device
 * queries against n device rows (both row-major float32, L a multiple of 16),
 * written to d_dots as nq x n float32 (row-major by query), ordered on
 * `stream`.  Allocates its own temporaries. */
HG_API hg_status hg_bf16_dots(const float *d_rows, uint64_t n, uint32_t L, const float *d_queries, uint32_t nq,
                              float *d_dots, void *stream);

/* Diagnostics (no counterpart in the reference): the failure path of the
 * tensor-core filter kernel.  Runs it once on a small internal problem (512
 * rows x 64 queries of length 64, on the current device, ordered on
 * `stream`) with every bounded wait shortened to wait_us microseconds
 * (1..2,000,000).  withhold = 1 withholds the first operand copy, so a
 * barrier phase never completes and the MMA warp's wait runs out: the kernel
 * then drains its copies and MMAs, frees its tensor memory, returns, and the
 * call reports HG_ERR_TIMEOUT with the device still usable.  withhold = 0
 * returns HG_OK.  Allocates its own temporaries. */
HG_API hg_status hg_filter_wait_check(uint32_t wait_us, int withhold, void *stream);

/* The same for the CTA-pair filter kernel (the screening pass on 2-CTA
 * clusters, cta_group::2): one pass over 1,024 rows x 64 queries of length 64
 * with no bounds.  withhold = 1 withholds the odd CTA's first row copy, so
 * the leader CTA's barrier phase never completes; both CTAs of every pair
 * then give up, the leader drains its copies and MMAs, both free their
 * tensor memory, and the call reports HG_ERR_TIMEOUT. */
HG_API hg_status hg_filter_pair_wait_check(uint32_t wait_us, int withhold, void *stream);

/* Launch parameters of the query kernels that depend on the data and the
 * GPU (no counterpart in the reference: its parallel search takes thread
 * counts and thresholds on the command line instead).  0 in a field means
 * "keep the current value". */
typedef struct {
  uint32_t filter_tiles_per_item;  /* batched filter: 128-row tiles per work item (8..128) */
  uint32_t bound_tiles_per_item;   /* batched bound pass: tiles per work item (2..64) */
  uint32_t rerank_blocks_per_sm;   /* batched re-rank: blocks of 8 warps per SM (1..16) */
  uint32_t approx_blocks_per_sm;   /* plain path: blocks per SM of the approximate-leaf scan (1..4) */
  uint32_t filter_cta_pair;        /* batched filter (L <= 256): 1 = CTA pairs (cta_group::2 MMAs of
                                      256 rows, half of the query tile per CTA), 2 = one CTA per 128 rows
                                      (the default) */
  double batch_ms;                 /* hg_autotune: device time of one batch with the chosen values */
  double plain_ms;                 /* hg_autotune: device time of the plain-path sample */
} hg_tuning;

/* Current launch parameters of a handle (defaults until tuned or set). */
HG_API hg_status hg_tuning_get(const hg_index *ix, hg_tuning *out);

/* Sets launch parameters (fields left 0 keep their value). */
HG_API hg_status hg_tuning_set(hg_index *ix, const hg_tuning *t);

/* Autotuner: times candidate launch parameters on a sample of the caller's
 * own queries (device memory, 16-byte aligned; nq of them with per-query k
 * from the host array ks, NULL = kmax), one parameter at a time, keeps the
 * fastest with the handle and returns them.  Answers do not depend on these
 * parameters; only the time does.  Allocates its own output buffers. */
HG_API hg_status hg_autotune(hg_index *ix, const float *d_queries, uint32_t nq, const uint32_t *ks, uint32_t kmax,
                             void *stream, hg_tuning *out);

/* The approximate leaf of each query: the leaf the query routes to
 * (approximate_knn_search's traversal, hercules_query_engine.c:176-222). */
HG_API hg_status hg_route(hg_index *ix, const float *queries, uint32_t nq, int32_t *leaf_out);

/* LB_EAPCA of one query against every leaf in DFS order
 * (calculate_node_min_distance, hercules_node.c:879-924). */
HG_API hg_status hg_leaf_lower_bounds(hg_index *ix, const float *query, float *lb_out);

/* ---- data ------------------------------------------------------------- */

/* Seeded z-normalised random walks: rows [first, first+n) of stream `seed`
 * (tools/Cgenerator semantics, steps from Philox4x32-10 + Box-Muller).
 * out_on_device = 1 writes device memory of `device`, else host memory
 * (computed on the host CPU, same bits). */
HG_API hg_status hg_generate_walks(uint64_t seed, uint64_t first, uint64_t n, uint32_t L, float *out,
                            int out_on_device, int device);

/* Noisy queries: query j = dataset row pick(j) plus N(0, sigma2[j]) noise,
 * z-normalised.  data (n x L) and out (nq x L) are both host or both device
 * memory.  base_ids (may be NULL) receives pick(j). */
HG_API hg_status hg_generate_queries(uint64_t seed, const float *data, uint64_t n, uint32_t L,
                              uint32_t nq, const double *sigma2, float *out, uint64_t *base_ids,
                              int on_device, int device);

/* Unit vectors: rows [first, first+n) of stream `seed`, each N(0, I) (the
 * same Philox + Box-Muller draws) then L2-normalised in float -- the
 * short-series vector shape of the benchmark configurations (no reference
 * counterpart: the reference generator makes random walks only). */
HG_API hg_status hg_generate_unit_vectors(uint64_t seed, uint64_t first, uint64_t n, uint32_t L, float *out,
                                          int out_on_device, int device);

/* hg_generate_queries for unit vectors: row pick(j) plus N(0, sigma2[j])
 * noise, then L2-normalised. */
HG_API hg_status hg_generate_unit_queries(uint64_t seed, const float *data, uint64_t n, uint32_t L, uint32_t nq,
                                          const double *sigma2, float *out, uint64_t *base_ids, int on_device,
                                          int device);

/* Noisy queries over a seeded collection that need not be resident: query j
 * = row pick(j) of the stream data_seed (a random walk, or with unit = 1 a
 * unit vector), regenerated, plus N(0, sigma2[j]) noise, then normalised as
 * hg_generate_queries / hg_generate_unit_queries do -- the same bits as
 * those entry points given the collection of data_seed.  For row-range
 * shards, where no process holds every row.  out (nq x L) is host or device
 * memory (on_device). */
HG_API hg_status hg_generate_queries_seeded(uint64_t data_seed, uint64_t seed, uint64_t n, uint32_t L, uint32_t nq,
                                            const double *sigma2, int unit, float *out, uint64_t *base_ids,
                                            int on_device, int device);

/* The 255 iSAX breakpoints of cardinality 256 used by this library. */
HG_API hg_status hg_sax_breakpoints(float *out255);

/* ---- allocation-free scan -------------------------------------------- */

/* Exact k-NN of one query by a scan of every row of a caller-owned device
 * matrix (row-major n x L float32, 16-byte aligned; the id of a row is its
 * index), with the distance and tie rule of hg_knn; outputs k squared
 * distances and ids in device memory, ordered on `stream`.  This entry point
 * has no counterpart in the reference.  It is for callers that cannot
 * allocate device memory -- code held to a fixed memory-pool budget, or a
 * plugin host that forbids cudaMalloc/cudaFree (and the synchronisation they
 * imply) on its query threads -- so it allocates nothing.  Its working
 * memory is one static device array of about 0.3 MB (8 KB of counters and
 * the top-k, plus 148 candidate lists of 256 entries) that every GPU loading
 * the library holds until exit; the first call on a device looks that
 * array's device address up (make that first call before any stream
 * capture).  Calls share the array: calls whose kernels overlap on the GPU
 * race, so serialise them.  Limits: 1 <= k <= 224, L a multiple of 16 up to
 * 16384, n < 2^32; beyond them the call returns HG_ERR_LIMIT. */
HG_API hg_status hg_pscan_noalloc(const float *d_rows, uint64_t n, uint32_t L, const float *d_query,
                                  uint32_t k, float *d_dist_out, int64_t *d_id_out, void *stream);

#ifdef __cplusplus
}
#endif
#endif
