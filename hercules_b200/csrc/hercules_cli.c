/*
 * hercules_cli.c -- bin/hercules with the reference's command line, on the GPU.
 *
 * Accepts the flags of the reference CLI (code/hercules/src/hercules.c:81-116,
 * getopt_long) and prints its TSV lines (`Name\tvalue\tqueryfile\tq\trank`,
 * print_query_stats, hercules_query_engine.c:3558-3918):
 *
 *   --mode 0   build the index from --dataset and write it to --index-path
 *              (which must not exist, as in hercules_index_settings_init)
 *   --mode 1   read the index and answer --queries-size exact k-NN queries
 *   --mode 2   both
 *
 * Flags that choose among the reference's CPU strategies (--num-threads,
 * --serial, --sims, --num-queues, --num-read-threads, --flush-threshold,
 * --num-write-threads, --initial-db-size, --eapca-threshold, --sax-threshold,
 * --buffer-size beyond recording it) are accepted and have no effect: the
 * exact answer does not depend on them.  --approx-stop-condition N, given
 * explicitly, seeds the exact search with N leaves best-first (the greedy
 * seeding of the reference's parallel path; the answers are the same).
 * --epsilon E
 * (> 0) runs the reference's epsilon-approximate search and --nprobes P its
 * nprobes search (hercules_file_loaders.c:230-243: nprobes first); --delta is
 * accepted and, as in the reference's serial path (which passes r_delta =
 * FLT_MAX), has no effect.  Modes the GPU path does not serve (--track-bsf,
 * --track-pruning, --max-policy, --incremental) are refused with a message
 * instead of silently running something else.
 *
 * Added flags: --gpu N (device, default 0), --pscan (scan every row instead
 * of the index), --no-lb-sax (skip the per-row LB_SAX filter).
 */
#define _GNU_SOURCE
#include <errno.h>
#include <float.h>
#include <getopt.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>
#include <sys/time.h>
#include <unistd.h>

#include "hercules_gpu.h"

static double now_s(void) {
  struct timeval t;
  gettimeofday(&t, NULL);
  return t.tv_sec + t.tv_usec * 1e-6;
}

static int check(hg_status s, const char *what) {
  if (s != HG_OK) {
    fprintf(stderr, "Error in hercules (%s): %s: %s\n", what, hg_status_string(s), hg_last_error());
    return 0;
  }
  return 1;
}

typedef struct {
  const char *dataset, *queries, *index_path;
  unsigned long long dataset_size;
  unsigned queries_size, queries_skip, ts_size, leaf_size, k;
  double buffer_mb;
  int mode, gpu, pscan, lb_sax;
  float epsilon, delta;
  unsigned nprobes;
  int approx_leaves; /* --approx-stop-condition: greedy seeding with L_max leaves */
  int track_bsf, track_pruning, max_policy, incremental;
} opts_t;

static int build_index(const opts_t *o, hg_index **ix) {
  /* hercules_index_settings_init refuses an existing directory */
  struct stat st;
  if (stat(o->index_path, &st) == 0) {
    fprintf(stderr, "WARNING! Target index directory already exists. Please delete or choose a new one.\n");
    return 0;
  }
  if (mkdir(o->index_path, 0777) != 0) {
    fprintf(stderr, "Error in hercules: cannot create %s: %s\n", o->index_path, strerror(errno));
    return 0;
  }
  double t0 = now_s();
  if (!check(hg_index_build_file(o->dataset, o->dataset_size, o->ts_size, o->leaf_size, o->gpu, ix), "build"))
    return 0;
  double t1 = now_s();
  if (!check(hg_index_write(*ix, o->index_path, o->buffer_mb), "write")) return 0;
  double t2 = now_s();
  hg_index_info info;
  hg_index_info_get(*ix, &info);
  printf("Index_building_total_time_secs\t%lf\t%s\t%d\n", t1 - t0, o->dataset, 0);
  printf("Index_writing_total_time_secs\t%lf\t%s\t%d\n", t2 - t1, o->dataset, 0);
  printf("Index_leaf_nodes_count\t%u\t%s\t%d\n", info.num_leaves, o->dataset, 0);
  printf("Index_total_nodes_count\t%u\t%s\t%d\n", info.num_nodes, o->dataset, 0);
  printf("Index_internal_nodes_count\t%u\t%s\t%d\n", info.num_nodes - info.num_leaves, o->dataset, 0);
  return 1;
}

/* The query file must hold --queries-skip + --queries-size series of the
 * index's length (root.idx header: timeseries_size at byte 16).  Checked
 * before the index is loaded, so a bad request fails fast with the
 * reference's messages and no device work. */
static int check_query_file(const opts_t *o) {
  char path[4096];
  snprintf(path, sizeof path, "%sroot.idx", o->index_path ? o->index_path : "");
  FILE *r = fopen(path, "rb");
  if (!r) return 1; /* hg_index_read reports it */
  unsigned char hdr[20];
  const size_t got = fread(hdr, 1, sizeof hdr, r);
  fclose(r);
  if (got != sizeof hdr) return 1;
  uint32_t L;
  memcpy(&L, hdr + 16, 4);
  if (L == 0) return 1;
  FILE *f = fopen(o->queries, "rb");
  if (!f) {
    fprintf(stderr, "File %s not found!\n", o->queries);
    return 0;
  }
  fseeko(f, 0, SEEK_END);
  const unsigned long long total = (unsigned long long)ftello(f) / (sizeof(float) * L);
  fclose(f);
  if (total < (unsigned long long)o->queries_size + o->queries_skip) {
    fprintf(stderr, "File %s has only %llu records!\n", o->queries, total);
    return 0;
  }
  return 1;
}

static int run_queries(const opts_t *o, hg_index *ix) {
  hg_index_info info;
  hg_index_info_get(ix, &info);
  const unsigned L = info.ts_length;
  FILE *f = fopen(o->queries, "rb");
  if (!f) {
    fprintf(stderr, "File %s not found!\n", o->queries);
    return 0;
  }
  fseek(f, 0, SEEK_END);
  unsigned long long total = (unsigned long long)ftell(f) / (sizeof(float) * L);
  if (total < (unsigned long long)o->queries_size + o->queries_skip) {
    fprintf(stderr, "File %s has only %llu records!\n", o->queries, total);
    fclose(f);
    return 0;
  }
  fseek(f, (long)o->queries_skip * L * sizeof(float), SEEK_SET);
  float *q = malloc(sizeof(float) * L);
  float *d = malloc(sizeof(float) * o->k);
  int64_t *id = malloc(sizeof(int64_t) * o->k);
  uint64_t *pos = malloc(sizeof(uint64_t) * o->k);
  hg_knn_opts ko;
  memset(&ko, 0, sizeof ko);
  ko.mode = o->pscan ? HG_MODE_PSCAN : HG_MODE_PLAIN;
  ko.use_lb_sax = o->lb_sax;
  ko.epsilon = o->epsilon;
  ko.nprobes = (int)o->nprobes;
  ko.approx_leaves = o->approx_leaves;
  int ok = 1;
  for (unsigned i = 0; i < o->queries_size && ok; ++i) {
    if (fread(q, sizeof(float), L, f) != L) {
      fprintf(stderr, "Error in hercules: short read in %s\n", o->queries);
      ok = 0;
      break;
    }
    const unsigned qn = o->queries_skip + i + 1; /* q_loaded is 1-based */
    hg_query_stats st;
    double t0 = now_s();
    if (!check(hg_knn(ix, q, 1, o->k, &ko, d, id, pos, &st), "query")) {
      ok = 0;
      break;
    }
    double wall = now_s() - t0;
    for (unsigned r = 0; r < o->k; ++r) {
      const unsigned rank = r + 1;
      if (r == 0) {
        printf("Query_total_time_secs\t%lf\t%s\t%u\t%u\n", wall, o->queries, qn, rank);
        printf("Query_total_device_time_secs\t%lf\t%s\t%u\t%u\n", st.device_ms / 1000.0, o->queries, qn, rank);
        printf("Query_total_loaded_nodes_count\t%llu\t%s\t%u\t%u\n", (unsigned long long)st.leaves_scanned + 1,
               o->queries, qn, rank);
        printf("Query_total_loaded_ts_count\t%llu\t%s\t%u\t%u\n", (unsigned long long)st.rows_visited,
               o->queries, qn, rank);
      }
      printf("Query_exact_distance\t%f\t%s\t%u\t%u\n", isfinite(d[r]) ? sqrtf(d[r]) : FLT_MAX, o->queries, qn,
             rank);
      printf("Query_exact_series_id\t%lld\t%s\t%u\t%u\n", (long long)id[r], o->queries, qn, rank);
      printf("Query_exact_node_file_pos\t%u\t%s\t%u\t%u\n", (unsigned)pos[r], o->queries, qn, rank);
    }
  }
  fclose(f);
  free(q);
  free(d);
  free(id);
  free(pos);
  return ok;
}

static void usage(void) {
  printf("Usage: hercules --mode 0|1|2 --dataset F --dataset-size N --timeseries-size L --leaf-size S\n"
         "                --index-path DIR/ --queries F --queries-size Q [--queries-skip S] --k K\n"
         "                [--buffer-size MB] [--gpu N] [--pscan] [--no-lb-sax]\n"
         "  CPU strategy flags of the reference are accepted and ignored.\n");
}

int main(int argc, char **argv) {
  opts_t o;
  memset(&o, 0, sizeof o);
  o.index_path = "out/";
  o.dataset_size = 1000;
  o.queries_size = 5;
  o.ts_size = 256;
  o.leaf_size = 100;
  o.buffer_mb = 6439.2;
  o.k = 1;
  o.lb_sax = 1;
  o.delta = 1;
  static struct option long_options[] = {
      {"buffer-size", required_argument, 0, 'b'},      {"epsilon", required_argument, 0, 'c'},
      {"dataset", required_argument, 0, 'd'},          {"delta", required_argument, 0, 'e'},
      {"queries-size", required_argument, 0, 'f'},     {"track-bsf", required_argument, 0, 'g'},
      {"incremental", no_argument, 0, 'h'},            {"track-pruning", required_argument, 0, 'i'},
      {"all-mindists", required_argument, 0, 'j'},     {"k", required_argument, 0, 'k'},
      {"leaf-size", required_argument, 0, 'l'},        {"max-policy", required_argument, 0, 'm'},
      {"dataset-hists", required_argument, 0, 'n'},    {"nprobes", required_argument, 0, 'o'},
      {"index-path", required_argument, 0, 'p'},       {"queries", required_argument, 0, 'q'},
      {"serial", required_argument, 0, 'r'},           {"minimum-distance", required_argument, 0, 's'},
      {"timeseries-size", required_argument, 0, 't'},  {"sax-cardinality", required_argument, 0, 'w'},
      {"paa-segments", required_argument, 0, 'x'},     {"num-queues", required_argument, 0, 'A'},
      {"num-threads", required_argument, 0, 'B'},      {"num-read-threads", required_argument, 0, 'C'},
      {"approx-stop-condition", required_argument, 0, 'D'}, {"mode", required_argument, 0, 'y'},
      {"dataset-size", required_argument, 0, 'z'},     {"sims", no_argument, 0, 'S'},
      {"queries-skip", required_argument, 0, 'Q'},     {"flush-threshold", required_argument, 0, 'F'},
      {"num-write-threads", required_argument, 0, 'G'}, {"eapca-threshold", required_argument, 0, 'H'},
      {"sax-threshold", required_argument, 0, 'I'},    {"initial-db-size", required_argument, 0, 'J'},
      {"gpu", required_argument, 0, 1001},             {"pscan", no_argument, 0, 1002},
      {"no-lb-sax", no_argument, 0, 1003},             {"help", no_argument, 0, '?'},
      {0, 0, 0, 0}};
  for (;;) {
    int oi = 0;
    int c = getopt_long(argc, argv, "", long_options, &oi);
    if (c == -1) break;
    switch (c) {
      case 'b': o.buffer_mb = atof(optarg); break;
      case 'c': o.epsilon = atof(optarg); break;
      case 'd': o.dataset = optarg; break;
      case 'e': o.delta = atof(optarg); break;
      case 'f': o.queries_size = (unsigned)atoi(optarg); break;
      case 'g': o.track_bsf = atoi(optarg); break;
      case 'h': o.incremental = 1; break;
      case 'i': o.track_pruning = atoi(optarg); break;
      case 'k': o.k = (unsigned)atoi(optarg); break;
      case 'l': o.leaf_size = (unsigned)atoi(optarg); break;
      case 'm': o.max_policy = atoi(optarg); break;
      case 'o': o.nprobes = (unsigned)atoi(optarg); break;
      case 'p': o.index_path = optarg; break;
      case 'q': o.queries = optarg; break;
      case 't': o.ts_size = (unsigned)atoi(optarg); break;
      case 'w':
        if (atoi(optarg) != 8) { fprintf(stderr, "Error in hercules: only --sax-cardinality 8 is supported\n"); return 1; }
        break;
      case 'x':
        if (atoi(optarg) != 16) { fprintf(stderr, "Error in hercules: only --paa-segments 16 is supported\n"); return 1; }
        break;
      case 'y': o.mode = atoi(optarg); break;
      case 'z': o.dataset_size = strtoull(optarg, NULL, 10); break;
      case 'Q': o.queries_skip = (unsigned)atoi(optarg); break;
      case 1001: o.gpu = atoi(optarg); break;
      case 1002: o.pscan = 1; break;
      case 1003: o.lb_sax = 0; break;
      case 'D': o.approx_leaves = (int)atof(optarg); break; /* the reference's L_max, read as a leaf count */
      case 'j': case 'n': case 'r': case 's': case 'A': case 'B': case 'C': case 'S':
      case 'F': case 'G': case 'H': case 'I': case 'J':
        break; /* CPU strategy knobs of the reference: no effect on the exact answer */
      case '?': usage(); return 0;
      default: return 1;
    }
  }
  if (o.track_bsf || o.track_pruning || o.max_policy || o.incremental) {
    fprintf(stderr, "Error in hercules: --track-bsf, --track-pruning, --max-policy and --incremental are not "
                    "served on the GPU\n");
    return 1;
  }
  if (o.epsilon < 0 || (o.pscan && (o.epsilon > 0 || o.nprobes))) {
    fprintf(stderr, "Error in hercules: --epsilon must not be negative and applies to the index search only\n");
    return 1;
  }
  if (o.index_path[strlen(o.index_path) - 1] != '/') {
    fprintf(stderr, "Error in hercules: --index-path must end with '/'\n");
    return 1;
  }
  hg_index *ix = NULL;
  int ok = 1;
  if (o.mode == 0 || o.mode == 2) {
    if (!o.dataset) { fprintf(stderr, "Error in hercules: --dataset is required\n"); return 1; }
    ok = build_index(&o, &ix);
  }
  if (ok && (o.mode == 1 || o.mode == 2)) {
    if (!o.queries) { fprintf(stderr, "Error in hercules: --queries is required\n"); return 1; }
    if (!ix && !check_query_file(&o)) return 1;
    if (!ix) {
      double t0 = now_s();
      ok = check(hg_index_read(o.index_path, o.gpu, &ix), "read");
      if (ok) {
        hg_index_info info;
        hg_index_info_get(ix, &info);
        printf("Index_reading_total_time_secs\t%lf\t%s\t%d\n", now_s() - t0, o.index_path, 0);
        printf("Index_leaf_nodes_count\t%u\t%s\t%d\n", info.num_leaves, o.index_path, 0);
        fprintf(stderr, ">>> Index loaded successfully from: %s\n", o.index_path);
      }
    }
    if (ok) ok = run_queries(&o, ix);
  }
  if (o.mode < 0 || o.mode > 2) {
    fprintf(stderr, "Error in hercules: --mode must be 0, 1 or 2\n");
    ok = 0;
  }
  hg_index_destroy(ix);
  return ok ? 0 : 1;
}
