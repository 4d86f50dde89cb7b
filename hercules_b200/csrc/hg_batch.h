// hg_batch.h -- launchers and argument blocks of the batched BF16 filter path.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "hg_kernels.h"

namespace hg {

constexpr int kBatchTileRows = 128;   // rows per tensor-core tile (and per tile norm)
constexpr int kBatchQueryTile = 256;  // queries per tensor-core tile (filter pass)
constexpr int kBatchBoundQueries = 64;  // queries per tile in the bound pass (MMA N = 64)
constexpr int kBatchMaxSlots = 4096;  // bound slots per query (sorted in one block)
constexpr int kBatchMaxSeg = 64;      // re-rank segments per query
constexpr int kBatchSegMin = 256;     // rows per re-rank segment, at least

// One work item of the bound pass: tiles [tile_lo, tile_hi) of the rows
// [row_begin, row_end) (one approximate leaf) against queries
// qperm[q_off .. q_off + q_cnt).
struct BatchItem {
  uint64_t row_begin, row_end;  // tile t covers rows row_begin + 128 t .. +127, valid below row_end
  uint32_t q_off, q_cnt;
  uint32_t tile_lo, tile_hi;
  uint32_t sub;       // bound slots per tile: 1, 2, 4, 8 or 16 (bound pass)
  uint32_t row_skip;  // rows of the first tile before the item's rows (pruned filter: tiles on the 128-row grid)
};

// Rows of one leaf and its bound-pass plan (slots per tile and tiles used).
struct LeafPlan {
  uint64_t start;
  uint32_t size, use_tiles, sub, pad;
};

// Arguments of the tensor-core filter (hg_umma.cu); the BF16 rows and the
// BF16 queries (in tile order) reach it as TMA descriptors.
struct BatchGemm {
  int L;
  uint64_t nrows;
  const float4* xmeta;      // per row: |x|^2, |x~|, |x - x~|, 0 (FP64, rounded up)
  const float4* tile_meta;  // per 128-row tile: the maxima of xmeta
  const float4* qmeta;      // per query: |q|^2, |q~|, |q - q~|, 0
  const uint32_t* qperm;   // query of each tile column (position in the BF16 query matrix)
  int nq;
  int mode;  // 0: bound pass over the items; 1: filter over every row; 2: raw products;
             // 3: filter over the items (leaves x the queries whose LB_EAPCA is within their bound)
  int qtile; // modes 1 and 2: queries per tile (MMA N): 64, 128, 256, or 0 = by the query count
  const uint32_t* nq_dev;   // if set: the query count (<= nq) read on the device
  // mode 0
  const BatchItem* items;
  uint32_t nitems;
  const uint32_t* nitems_dev;  // if set: the item count read on the device
  unsigned long long* bm;  // [q][bm_cap] (ordered d~ << 32 | row), ~0 before the launch
  uint32_t bm_cap;
  // mode 1
  uint32_t tiles_per_item;
  float c_acc, c_sq;       // error-bound coefficients: L 2^-20 and (L/8 + 16) 2^-22
  const float* bound;      // B_q
  unsigned long long* pairs;  // survivors (query << 32 | row) in blocks reserved per warp; ~0 = empty slot
  uint32_t* pairs_cnt;        // slots reserved; 0 before the launch, may end above pairs_cap
  uint32_t pairs_cap;
  int* err;                // raised (1) when a bounded wait gave up
  uint32_t* queue;         // if set: the work-item counter (0 before the launch); else a static round robin
  // if set (mode 1): the certified bounds used, [0] sum of err, [1] sum of
  // err / B_q (B_q > 0), [2] (item, query) pairs, [3] pairs with B_q > 0,
  // [4] the largest err; zeroed before the launch
  double* errstat;
  // mode 2 (diagnostics): raw dot products q~.x~, [query position][dots_ld]
  float* dots;
  uint64_t dots_ld;
  uint64_t wait_ns;         // each bounded wait gives up after this (0: 2 s)
  int withhold_first_copy;  // diagnostics: the first operand copy is never issued
};

struct BatchRank {
  const float* rows;  // FP32 rows, row-major, leaf order
  const int64_t* ids;
  const float* Q;     // FP32 queries
  int L;
  int nq;
  const uint32_t* kq;  // k of each query
  int kmax;            // output stride
  const unsigned long long* bm;
  uint32_t bm_cap;
  const uint32_t* slots_of_query;  // filled slots of the query's approximate leaf
  float* bound;                    // B_q (+inf: none)
  unsigned long long* init;        // [q][kMaxK] exact keys of the bound rows
  int* init_cnt;
  const uint32_t* bucket;
  const uint32_t* bucket_cnt;
  uint32_t bucket_cap;
  float* dist_out;  // [q][kmax]
  int64_t* id_out;
  int* ok_out;                // 1 verified, 0 retry with the lowered bound, -1 plain path
  unsigned long long* stats;  // [0] rows re-ranked [1] chunks [2] filter survivors
  // re-rank of the queries qlist[0 .. nlist) (qlist null: 0 .. nlist)
  const uint32_t* qlist;
  int nlist;                  // the list's size, or its capacity when nlist_dev is set
  const uint32_t* nlist_dev;  // if set: the list's size read on the device
  uint32_t* seg_rows;         // [list position] rows per segment
  uint32_t* seg_prefix;       // [nlist + 1] exclusive prefix of segments
  uint32_t* qbound;           // [q] running k-th distance (float bits)
  unsigned long long* parts;  // [segment][kmax] compacted lists
  int* part_cnt;              // [segment]
  uint32_t* heads;            // [0] segment counter
};

// n_dev (optional): the row count read on the device, at most n
cudaError_t launch_rows_to_bf16(const float* rows, const uint32_t* idx, uint64_t n, int L, void* out, float4* meta,
                                cudaStream_t s, const uint32_t* n_dev = nullptr);
cudaError_t launch_group_queries(const int* approx, int nq, const LeafPlan* plan, int nleaves, uint32_t btpi,
                                 uint32_t* perm, uint32_t* slots, uint32_t* leaf_qoff, uint32_t* leaf_qcnt,
                                 uint32_t* item_off, uint32_t* nitems, BatchItem* items, cudaStream_t s,
                                 uint32_t* gcnt = nullptr);  // 2 x nleaves words above kMaxLeavesSort leaves
// the pruned filter's query panel list and work items from the kept
// (leaf, query) pairs (k_group_pruned, k_emit_pruned); ctl[2] = the query
// count (*nq_dev if set, else nq) when the panel or the items do not fit
cudaError_t launch_group_pruned(const uint32_t* leaf_cnt, const uint32_t* leaf_q, uint32_t stride,
                                const LeafPlan* plan, int nleaves, uint32_t tpi, uint32_t panel_cap,
                                uint32_t items_cap, uint32_t nq, uint32_t* leaf_poff, uint32_t* leaf_ioff,
                                uint32_t* ctl, unsigned long long* pairs, uint32_t* panel_list, BatchItem* items,
                                cudaStream_t s, const uint32_t* nq_dev = nullptr);
cudaError_t launch_collect_retry(const int* ok, const uint32_t* list, uint32_t n, const uint32_t* n_dev,
                                 uint32_t* out, uint32_t* out_n, cudaStream_t s);
cudaError_t launch_count_unverified(const int* ok, uint32_t nq, uint32_t* out, cudaStream_t s);
cudaError_t launch_stamp(unsigned long long* slot, cudaStream_t s);  // global-timer stamp (ns)
cudaError_t launch_tile_norms(const float4* meta, uint64_t n, float4* tile_meta, cudaStream_t s);
cudaError_t launch_bound_select(const BatchRank& r, cudaStream_t s);
size_t umma_filter_smem();
// modes 1 and 3 on CTA pairs (cta_group::2, L <= 256): q_half_map has boxes
// of 128 queries (half of the query tile per CTA); blocks is rounded down to
// an even count
size_t umma_pair_smem();
cudaError_t launch_umma_pair(const CUtensorMap& rows_map, const CUtensorMap& q_half_map, const BatchGemm& g,
                             int blocks, cudaStream_t s);
// q_map: boxes of 256 queries, except for the bound pass (mode 0) with L <= 256:
// boxes of kBatchBoundQueries
cudaError_t launch_umma_filter(const CUtensorMap& rows_map, const CUtensorMap& q_map, const BatchGemm& g, int blocks,
                               cudaStream_t s);
cudaError_t launch_rerank(const BatchRank& r, int part_blocks, cudaStream_t s);
// Distributes the filter's survivor pairs into per-query buckets
// (bucket_cnt[q] counts every pair of q, also beyond bucket_cap); when the
// pair list overflowed, every query of the round is marked overflowed.
cudaError_t launch_scatter_pairs(const unsigned long long* pairs, const uint32_t* pairs_cnt, uint32_t pairs_cap,
                                 const uint32_t* qlist, int nlist, const uint32_t* nlist_dev, uint32_t* bucket,
                                 uint32_t* bucket_cnt, uint32_t bucket_cap, cudaStream_t s);

}  // namespace hg
