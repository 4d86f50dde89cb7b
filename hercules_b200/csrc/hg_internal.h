// hg_internal.h -- host-side structures of the B200 Hercules index.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/hercules_gpu.h"
#include "hg_batch.h"
#include "hg_kernels.h"

namespace hg {

// One node of the EAPCA tree (struct hercules_node, hercules_node.h:19-64,
// reduced to what the build, the query path and root.idx need).
struct Node {
  int parent = -1, left = -1, right = -1;
  bool is_leaf = true, is_left = false;
  uint32_t level = 0;
  std::vector<short> points;     // vertical segment ends
  std::vector<short> hs_points;  // horizontal-split candidate ends
  std::vector<float> sk;         // points.size() x {mean max, mean min, stdev max, stdev min}
  // split policy of an internal node (hercules_node_split.h:21-34)
  short split_from = 0, split_to = 0;
  int split_idx = 0;
  float split_value = 0.0f;
  uint32_t node_size = 0;
  std::vector<uint32_t> members;  // dataset rows of a leaf, insertion order
  std::string filename;
  uint64_t file_pos = 0;
  int leaf_index = -1;
};

// Device buffers sized by an index (one GPU per handle).
struct DeviceIndex {
  float* rows = nullptr;      // leaf-ordered rows, row-major (the leaves_raw.idx image)
  float* rows_rm = nullptr;   // optional row-major copy (write/export), may be null
  int64_t* ids = nullptr;     // dataset id of each leaf-ordered row
  uint8_t* sax = nullptr;     // iSAX word (16 symbols) of each leaf-ordered row
  float* bp = nullptr;        // 255 breakpoints of cardinality 256
  // leaves (DFS order)
  uint64_t* leaf_start = nullptr;
  uint32_t* leaf_size = nullptr;
  int* leaf_seg_off = nullptr;  // CSR offsets into leaf_points / leaf_sk
  short* leaf_points = nullptr;
  float* leaf_sk = nullptr;
  // routing tree (internal nodes; a child < 0 is the leaf ~child, DFS index)
  DNode* nodes = nullptr;
  int root = 0;
};

// Per-query scratch for the plain path (sized for the largest k).
struct QueryScratch {
  int kmax = 0;
  int nparts = 0;
  float* q = nullptr;             // L
  float* lb = nullptr;            // leaves
  int* approx_leaf = nullptr;     // 1
  int* cand = nullptr;            // leaves
  float* cand_lb = nullptr;       // leaves
  int* cand_count = nullptr;      // 1
  uint32_t* unit_prefix = nullptr;  // leaves + 1 (tiles per candidate, exclusive scan)
  uint32_t* counters = nullptr;   // work counter, misc
  uint32_t* bound = nullptr;      // float bits of the current k-th distance bound
  unsigned long long* parts = nullptr;  // nparts x kmax keys (d bits << 32 | id)
  int* part_count = nullptr;      // nparts
  unsigned long long* topk = nullptr;   // kmax keys
  int* topk_count = nullptr;
  uint64_t* topk_row = nullptr;   // kmax leaf-ordered rows of the answers
  float* paa = nullptr;           // 16
  float* sax_tab = nullptr;       // 16 x 256 LB_SAX terms of the current query
  uint32_t* sort_keys = nullptr;  // 4 x leaves: candidate sort above kMaxLeavesSort leaves
  unsigned long long* stats = nullptr;  // see ScanArgs
  uint32_t* list = nullptr;       // LB_SAX survivors (rows), n entries
  int* err = nullptr;             // device error flag
  uint32_t* actl = nullptr;       // approximate searches: [0] stale k-th bound bits, [1] gate flag
};

// Batched path: BF16 copy of the rows and their norms, built on the first
// batched call and kept with the index.
struct BatchData {
  void* xbf = nullptr;          // n x L BF16, row-major, leaf order
  float4* xmeta = nullptr;      // per row: |x|^2, |x~|, |x - x~| (FP64, rounded up)
  float4* tile_meta = nullptr;  // per 128-row tile: maxima of xmeta
  CUtensorMap rows_map;         // TMA descriptor of xbf (64 x 128 boxes, 128-byte swizzle)
};

// Batched path scratch, grown to the largest batch seen.
struct BatchScratch {
  uint32_t nq_cap = 0, bucket_cap = 0, bm_cap = 0, items_cap = 0;
  void* qbf = nullptr;
  float4* qmeta = nullptr;
  uint32_t* qperm = nullptr;
  int* approx = nullptr;
  uint32_t* kq = nullptr;
  uint32_t* slots = nullptr;
  BatchItem* items = nullptr;
  unsigned long long* bm = nullptr;
  float* bound = nullptr;
  unsigned long long* init = nullptr;
  int* init_cnt = nullptr;
  uint32_t* bucket = nullptr;
  uint32_t* bucket_cnt = nullptr;
  unsigned long long* pairs = nullptr;  // filter survivors before they are bucketed
  uint32_t pairs_cap = 0;
  int* ok = nullptr;
  unsigned long long* stats = nullptr;
  uint32_t* heads = nullptr;
  uint32_t parts_kmax = 0;
  uint32_t* qlist = nullptr;  // queries of a retry round
  uint32_t* seg_rows = nullptr;
  uint32_t* seg_prefix = nullptr;
  uint32_t* qbound = nullptr;
  unsigned long long* parts = nullptr;
  int* part_cnt = nullptr;
  // device-side control of a batch
  uint32_t* qlist2 = nullptr;    // second retry list (rounds alternate)
  uint32_t* ctrl = nullptr;      // [0] bound items [3] unverified queries [4 + r] queries of round r
  float* qin = nullptr;          // the batch's queries (fixed address for the graph)
  float* out_dist = nullptr;     // the batch's answers before they are copied out
  int64_t* out_id = nullptr;
  uint32_t out_kmax = 0;
  // bound-pass plan per leaf, for the `want` slots it was made for
  LeafPlan* leaf_plan = nullptr;
  uint32_t* group_cnt = nullptr;  // 2 x leaves: query grouping above kMaxLeavesSort leaves
  uint32_t* leaf_qoff = nullptr;
  uint32_t* leaf_qcnt = nullptr;
  uint32_t* item_off = nullptr;
  uint64_t plan_want = 0;
  uint32_t plan_bm_cap = 0, plan_max_use = 0;
  uint64_t gen = 0;              // bumped whenever a buffer above moves
  // the captured batch pipeline and the key it was captured for
  cudaGraphExec_t graph = nullptr;
  uint64_t graph_key[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  uint64_t graph_launches = 0;   // kernels in the captured pipeline
  unsigned long long* stamps = nullptr;  // [16] global-timer stamps at the phase boundaries
  double* errstat = nullptr;             // [5] certified bounds of the first filter pass (BatchGemm::errstat)
  uint32_t* queues = nullptr;            // [8] work-item counters of the filter launches
  // pruned filter: the (leaf, query) pairs LB_EAPCA keeps, their query panel
  // (each leaf's queries contiguous, BF16) and work items
  uint32_t prune_nq = 0;                 // queries the buffers hold (0: not allocated)
  uint32_t* leaf_cnt = nullptr;          // [leaves] kept queries
  uint32_t* leaf_q = nullptr;            // [leaves][prune_nq] their ids
  uint32_t* leaf_poff = nullptr;         // [leaves] panel offset
  uint32_t* leaf_ioff = nullptr;         // [leaves] item offset
  uint32_t* panel_list = nullptr;        // [panel_cap] query of each panel row
  void* panel_bf = nullptr;              // [panel_cap][L] BF16
  BatchItem* items3 = nullptr;           // [items3_cap]
  uint32_t panel_cap = 0, items3_cap = 0;
  uint32_t* pctl = nullptr;              // [4] items, panel rows, dense-pass queries
  unsigned long long* ppairs = nullptr;  // (query, row) pairs of the pruned pass
  CUtensorMap panel_map;                 // TMA descriptor of panel_bf (64 x 256 boxes)
  CUtensorMap panel_map_half;            // the same with 64 x 128 boxes (the CTA-pair filter)
  // distinct leaf segments (shared by many leaves) and the queries' mean and
  // stdev over each
  int nu = 0;
  short* useg_start = nullptr;
  short* useg_end = nullptr;
  int* seg_uid = nullptr;                // per leaf segment (leaf_points order): its distinct segment
  float2* segstats = nullptr;            // [prune_nq][nu]
};

}  // namespace hg

struct hg_index {
  int device = 0;
  uint32_t L = 0;
  uint32_t leaf_size = 0;
  uint64_t n = 0;
  double buffer_mb = 0.0;
  std::vector<hg::Node> nodes;  // nodes[0] is the root
  std::vector<int> leaves;      // node id of each leaf, DFS order
  std::vector<int64_t> ids;     // host copy of the row -> dataset id map
  bool has_ids = false;         // false for an index built by the reference
  hg::DeviceIndex d;
  hg::QueryScratch s;
  hg::BatchData bd;
  hg::BatchScratch bs;
  cudaStream_t stream = nullptr;
  int max_seg = 0;
  hg_tuning tune = {32, 8, 8, 2, 2, 0.0, 0.0};  // launch parameters (hg_autotune)
};
