// hg_kernels.h -- launchers of the sm_100a kernels (host side declarations).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>

namespace hg {

// Raises one kernel's dynamic shared-memory limit on the current device
// before its first launch there.  cudaFuncSetAttribute acts on the current
// device only, so the "done" state is one bit per device (devices 0..63;
// higher ones set the attribute on every launch).  Two host threads making
// their first call at once may both set it, which is harmless: the value is
// the same.  One instance per (kernel, limit) call site, as a function-local
// static.
class SmemLimit {
 public:
  cudaError_t ensure(const void* func, int bytes) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    const uint64_t bit = (dev >= 0 && dev < 64) ? (1ull << dev) : 0ull;
    if (bit && (done_.load(std::memory_order_acquire) & bit)) return cudaSuccess;
    e = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess && bit) done_.fetch_or(bit, std::memory_order_acq_rel);
    return e;
  }

 private:
  std::atomic<uint64_t> done_{0};
};

constexpr int kEdWarps = 8;  // warps per block of the distance stream
constexpr int kEdBlocksPerSm = 4;  // resident blocks per SM of the distance stream
constexpr int kWarpListCap = 256;  // per-warp candidate buffer (k <= kWarpListCap - 32)
constexpr int kMaxK = kWarpListCap - 32;
constexpr int kMaxLeavesSort = 8192;  // leaves whose sort / grouping arrays fit in shared memory
constexpr int kMergeCap = 8192;       // single-CTA bitonic merge capacity

// A routing node of the EAPCA tree: an internal node's split policy
// (hercules_node_split.h:21-34) and its children; a child < 0 is the leaf ~child.
struct DNode {
  int left, right;
  float value;
  short from, to;
  int idx;
  int pad;
};

struct Tree {
  const DNode* nodes;
  int root;  // >= 0 internal node, < 0 the leaf ~root
};

// Stage 1 of the leaf scan: candidate leaves -> LB_SAX survivors.
struct FilterArgs {
  const uint8_t* sax;
  const float* bp;
  int L;
  uint64_t nrows;
  const uint64_t* leaf_start;
  const uint32_t* leaf_size;
  const int* cand;
  const float* cand_lb;
  const int* cand_count;
  const uint32_t* unit_prefix;  // exclusive prefix of 32-row units per candidate
  const float* paa;
  const float* sax_tab;  // the query's 16 x 256 LB_SAX terms (k_leaf_lb), 16-byte aligned
  int use_lbsax;
  int cand_lo, cand_hi;  // candidates [cand_lo, cand_hi) of the sorted list; cand_hi <= 0: to the end
  const uint32_t* bound;
  uint32_t* list;        // surviving rows
  uint32_t* list_count;  // must be 0 before the launch
  unsigned long long* stats;  // [0] rows considered [2] rows pruned by LB_SAX [3] leaves visited
  int* err;                   // set to 1 when a bounded wait ran out (may be NULL)
};

// Stage 2: early-abandoning distances over a row list (or a row range).
struct EdArgs {
  const float* rows;  // leaf-ordered, row-major
  const int64_t* ids;
  int L;
  const uint32_t* list;        // rows; NULL: the range below
  const uint32_t* list_count;
  const int* ident_leaf;       // range = this leaf's rows (device pointer), else
  uint64_t ident_first;        //   [ident_first, ident_first + ident_count)
  uint64_t ident_count;
  const uint64_t* leaf_start;
  const uint32_t* leaf_size;
  uint32_t* head;              // batch counter, must be 0 before the launch
  const float* q;
  int k;
  uint32_t* bound;             // float bits of the running k-th bound (atomicMin)
  unsigned long long* parts;   // per-warp sorted lists (kWarpListCap stride)
  int* part_count;
  unsigned long long* stats;   // [1] chunks computed [4] rows completed [5] rows started
  const int* gate;             // if set and *gate == 0, the launch scans nothing
  int has_floor;               // 1: only rows at distance > floor enter the lists (the
  float floor;                 //   answers of k above kMaxK come in rounds above it)
};

int sm_count(int device);


// build
cudaError_t launch_route_rows(const float* X, int L, const uint32_t* rows, uint64_t first, uint32_t count,
                              Tree t, int* leaf_out, cudaStream_t s);
cudaError_t launch_sketch_members(const float* X, int L, const uint32_t* members, uint32_t count,
                                  const short* seg_from, const short* seg_to, int nsegs, int* keys_out,
                                  cudaStream_t s);
cudaError_t launch_route_flags(const float* X, int L, const uint32_t* members, uint32_t count, short from,
                               short to, int idx, float value, uint8_t* flags, cudaStream_t s);
cudaError_t launch_gather_rows(const float* X, int L, const uint32_t* perm, uint64_t n, float* rows,
                               cudaStream_t s);
cudaError_t launch_sax_rows(const float* rows, int L, uint64_t n, const float* bp, uint8_t* sax,
                            cudaStream_t s);

// queries
cudaError_t launch_query_prep(const float* q, int L, Tree t, const uint64_t* leaf_start,
                              const uint32_t* leaf_size, int* approx_leaf, float* paa, int* cand,
                              float* cand_lb, int* cand_count, uint32_t* unit_prefix, uint32_t* bound,
                              int* topk_count, uint32_t* counters, cudaStream_t s);
cudaError_t launch_route_queries(const float* Q, int nq, int L, Tree t, int* leaf_out, cudaStream_t s);
cudaError_t launch_leaf_lb(const float* q, int L, int nleaves, const int* seg_off, const short* points,
                           const float* sk, float* lb_out, cudaStream_t s, const float* paa = nullptr,
                           const float* bp = nullptr, float* sax_tab = nullptr);
// gkeys: 4 x nleaves words of global scratch, needed above kMaxLeavesSort leaves
cudaError_t launch_select_sort(const float* lb, int nleaves, const uint32_t* bound, const int* approx_leaf,
                               const uint64_t* leaf_start, const uint32_t* leaf_size, int* cand,
                               float* cand_lb, int* cand_count, uint32_t* unit_prefix, cudaStream_t s,
                               uint32_t* gkeys = nullptr);
cudaError_t launch_pscan_prep(uint64_t nrows, int* cand_count, uint32_t* unit_prefix, uint32_t* bound,
                              int* topk_count, uint32_t* counters, cudaStream_t s);
cudaError_t launch_lbsax_filter(const FilterArgs& a, int blocks, cudaStream_t s);  // blocks: one per SM
size_t lbsax_filter_smem();
cudaError_t launch_ed_stream(const EdArgs& a, int blocks, cudaStream_t s);
// batched path: the (leaf, query) pairs whose LB_EAPCA is within the query's
// bound (k_leaf_keep)
cudaError_t launch_leaf_keep(const float* Q, int L, int nq, const short* useg_start, const short* useg_end, int nu,
                             float2* segstats, const int* seg_off, const short* points, const int* seg_uid,
                             const float* sk, const uint32_t* leaf_size, int nleaves, const float* bound,
                             uint32_t* leaf_cnt, uint32_t* leaf_q, uint32_t stride, cudaStream_t s);
// the same over the queries qlist[0 .. *nq_dev) (nq: their most), with the
// segment statistics already computed
cudaError_t launch_leaf_keep_list(const float2* segstats, int nu, int L, int nq, const int* seg_off,
                                  const short* points, const int* seg_uid, const float* sk, const uint32_t* leaf_size,
                                  int nleaves, const float* bound, uint32_t* leaf_cnt, uint32_t* leaf_q,
                                  uint32_t stride, const uint32_t* qlist, const uint32_t* nq_dev, cudaStream_t s);
// epsilon search: *flag = (lb <= stale / eps1), the reference's test of a
// candidate leaf against its k-th distance of that moment; *scanned counts
// the leaves that pass
cudaError_t launch_leaf_gate(float lb, float eps1, const uint32_t* stale, int* flag, unsigned long long* scanned,
                             cudaStream_t s);
// *stale = *bound when *flag
cudaError_t launch_stale_copy(const int* flag, const uint32_t* bound, uint32_t* stale, cudaStream_t s);
// resident blocks per SM of the distance stream for series length L
int ed_blocks_per_sm(int L);
// the same with id = row index (EdArgs::ids unused)
cudaError_t launch_ed_stream_row_ids(const EdArgs& a, int blocks, cudaStream_t s);
cudaError_t launch_merge(const unsigned long long* parts, const int* part_count, int nparts, int k,
                         unsigned long long* topk, int* topk_count, uint32_t* bound, int* err,
                         cudaStream_t s);
cudaError_t launch_emit(const unsigned long long* topk, const int* topk_count, int k, float* dist_out,
                        int64_t* id_out, cudaStream_t s);

// data
// unit = 1: unit-normalised Gaussian rows / L2-normalised noisy queries
cudaError_t launch_generate_walks(uint64_t seed, uint64_t first, uint64_t n, int L, float* out,
                                  cudaStream_t s, int unit = 0);
cudaError_t launch_generate_queries(uint64_t seed, const float* data, uint64_t n, int L, int nq,
                                    const double* sigma2, float* out, uint64_t* base_ids, cudaStream_t s,
                                    int unit = 0, uint64_t data_seed = 0);  // data == nullptr: rows from data_seed

}  // namespace hg
