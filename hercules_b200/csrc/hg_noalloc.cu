// hg_noalloc.cu -- exact k-NN scan that allocates no memory.
//
// Some callers cannot allocate device memory: a caller held to a fixed
// memory-pool budget that must not grow, or a plugin host that forbids
// allocation (and the implicit synchronisation of cudaMalloc/cudaFree) on
// its query threads.  hg_pscan_noalloc serves them: it scans a caller-owned
// device matrix (the same early-abandoning distance and tie rule as hg_knn's
// scan mode) and keeps all of its working memory in the file-scope array
// below.
//
// That array lives on every GPU that loads this library, for as long as the
// process runs (kNoAllocScratchBytes: 8 KB of counters and the top-k, plus
// one 256-entry candidate list of 8 bytes per entry for each of the 148
// blocks of the scan, about 0.3 MB).  Calls share it and it keeps the
// previous call's contents; every call resets the counters it needs before
// use.  Two calls whose kernels overlap on the GPU (different streams, or
// several host threads) race on it and give wrong answers: serialise them.
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

#include <mutex>

#include "../../include/hercules_gpu.h"
#include "hg_kernels.h"

void hg_record_error(const char* msg);  // hg_index.cu: the text hg_last_error returns

namespace {

// 148 blocks of 8 warps; the scan reduces its warps' lists to one
// 256-entry candidate list per block, and the merge reads those 148 lists
constexpr int kNoAllocBlocks = 148;
constexpr int kNoAllocParts = kNoAllocBlocks;
constexpr size_t kListBytes = (size_t)kNoAllocParts * hg::kWarpListCap * sizeof(unsigned long long);
constexpr size_t kHeaderBytes = 8192;  // counters, bound, top-k, per-list counts
constexpr size_t kNoAllocScratchBytes = kHeaderBytes + kListBytes;

static __device__ __align__(256) unsigned char g_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
unsigned char* g_ptr[kMaxDevices] = {nullptr};

hg_status fail(hg_status s, const char* msg) {
  hg_record_error(msg);
  return s;
}

// Device address of g_scratch on the current device, looked up once per
// device (the first call on a device performs this set-up).
hg_status scratch_of(int dev, unsigned char** out) {
  if (dev < 0 || dev >= kMaxDevices) return fail(HG_ERR_LIMIT, "hg_pscan_noalloc: device index above 63");
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_ptr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
    if (e != cudaSuccess || !p) return fail(HG_ERR_CUDA, "hg_pscan_noalloc: cudaGetSymbolAddress failed");
    g_ptr[dev] = static_cast<unsigned char*>(p);
  }
  *out = g_ptr[dev];
  return HG_OK;
}

}  // namespace

extern "C" HG_API hg_status hg_pscan_noalloc(const float* d_rows, uint64_t n, uint32_t L, const float* d_query,
                                             uint32_t k, float* d_dist_out, int64_t* d_id_out, void* stream) {
  if (!d_rows || !d_query || (!d_dist_out && !d_id_out)) return fail(HG_ERR_ARG, "hg_pscan_noalloc: null pointer");
  if (n == 0 || L == 0 || L % 16 != 0) return fail(HG_ERR_ARG, "hg_pscan_noalloc: need n > 0, L a multiple of 16");
  if (L > 16384) return fail(HG_ERR_LIMIT, "hg_pscan_noalloc: L above 16384");
  if (n > 0xffffffffull) return fail(HG_ERR_LIMIT, "hg_pscan_noalloc: more than 2^32-1 rows");
  if (k == 0 || k > (uint32_t)hg::kMaxK) return fail(HG_ERR_LIMIT, "hg_pscan_noalloc: k must be 1..224");
  if (((uintptr_t)d_rows & 15) || ((uintptr_t)d_query & 15))
    return fail(HG_ERR_ARG, "hg_pscan_noalloc: rows and query must be 16-byte aligned");
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return fail(HG_ERR_CUDA, "hg_pscan_noalloc: no current device");
  unsigned char* base = nullptr;
  hg_status st = scratch_of(dev, &base);
  if (st != HG_OK) return st;
  // layout of the scratch
  uint32_t* counters = reinterpret_cast<uint32_t*>(base + 0);          // 8
  uint32_t* bound = reinterpret_cast<uint32_t*>(base + 64);            // 1
  int* cand_count = reinterpret_cast<int*>(base + 128);                // 1
  uint32_t* unit_prefix = reinterpret_cast<uint32_t*>(base + 192);     // 2
  int* topk_count = reinterpret_cast<int*>(base + 256);                // 1
  unsigned long long* stats = reinterpret_cast<unsigned long long*>(base + 512);  // 8
  unsigned long long* topk = reinterpret_cast<unsigned long long*>(base + 1024);  // kMaxK
  int* part_count = reinterpret_cast<int*>(base + 3072);              // kNoAllocParts
  unsigned long long* parts = reinterpret_cast<unsigned long long*>(base + kHeaderBytes);
  static_assert(1024 + sizeof(unsigned long long) * hg::kMaxK <= 3072, "scratch layout");
  static_assert(3072 + sizeof(int) * kNoAllocParts <= kHeaderBytes, "scratch layout");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // counters, bound and list counts start from zero / +inf on every call
  cudaError_t e = hg::launch_pscan_prep(n, cand_count, unit_prefix, bound, topk_count, counters, s);
  if (e == cudaSuccess) {
    hg::EdArgs a{};
    a.rows = d_rows;
    a.ids = nullptr;
    a.L = (int)L;
    a.list = nullptr;
    a.ident_leaf = nullptr;
    a.ident_first = 0;
    a.ident_count = n;
    a.head = counters;
    a.q = d_query;
    a.k = (int)k;
    a.bound = bound;
    a.parts = parts;
    a.part_count = part_count;
    a.stats = stats;
    e = hg::launch_ed_stream_row_ids(a, kNoAllocBlocks, s);
  }
  if (e == cudaSuccess) e = hg::launch_merge(parts, part_count, kNoAllocBlocks, (int)k, topk, topk_count, bound, nullptr, s);
  if (e == cudaSuccess) e = hg::launch_emit(topk, topk_count, (int)k, d_dist_out, d_id_out, s);
  if (e != cudaSuccess) return fail(HG_ERR_CUDA, cudaGetErrorString(e));
  return HG_OK;
}
