// hg_batch.h -- launchers and argument blocks of the batched BF16 filter path.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "hg_kernels.h"

namespace hg {

constexpr int kBatchTileRows = 128;   // rows per tensor-core tile (and per tile norm)
constexpr int kBatchMaxSlots = 4096;  // bound slots per query (sorted in one block)

// One work item of the bound pass: tiles [tile_lo, tile_hi) of the rows
// [row_begin, row_end) (one approximate leaf) against queries
// qperm[q_off .. q_off + q_cnt).
struct BatchItem {
  uint64_t row_begin, row_end;
  uint32_t q_off, q_cnt;
  uint32_t tile_lo, tile_hi;
  uint32_t sub;  // bound slots per tile: 1, 2, 4, 8 or 16
  uint32_t pad;
};

struct BatchGemm {
  const void* xbf;  // BF16 rows, row-major, leaf order
  const void* qbf;  // BF16 queries
  int L;
  uint64_t nrows;
  const float* xn2;        // |x|^2 rounded up
  const float* tile_n2;    // per 128-row tile: max |x|^2
  const float* tile_norm;  //                   max |x|
  const float* qn2;        // |q|^2 rounded up
  const float* qnorm;      // |q| rounded up
  const uint32_t* qperm;   // queries in tile order
  int nq;
  int mode;  // 0: bound pass over the items; 1: filter over every row
  // mode 0
  const BatchItem* items;
  uint32_t nitems;
  unsigned long long* bm;  // [q][bm_cap] (ordered d~ << 32 | row), ~0 before the launch
  uint32_t bm_cap;
  // mode 1
  uint32_t tiles_per_item;
  float c_dot, c_sq;       // error-bound coefficients
  const float* bound;      // B_q
  uint32_t* bucket;        // [q][bucket_cap] surviving rows
  uint32_t* bucket_cnt;    // 0 before the launch
  uint32_t bucket_cap;
  uint32_t* work_head;     // 0 before the launch
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
  int* ok_out;                // 1: verified; 0: take the plain path
  unsigned long long* stats;  // [0] rows re-ranked [1] chunks [2] filter survivors
};

cudaError_t launch_rows_to_bf16(const float* rows, uint64_t n, int L, void* out, float* n2, float* norm,
                                cudaStream_t s);
cudaError_t launch_tile_norms(const float* n2, uint64_t n, float* tile_n2, float* tile_norm, cudaStream_t s);
size_t bf16_filter_smem();
cudaError_t launch_bf16_filter(const BatchGemm& g, int blocks, cudaStream_t s);
cudaError_t launch_bound_select(const BatchRank& r, cudaStream_t s);
cudaError_t launch_rerank(const BatchRank& r, cudaStream_t s);

}  // namespace hg
