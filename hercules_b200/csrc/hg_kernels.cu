// hg_kernels.cu -- sm_100a kernels of the Hercules exact k-NN path.
//
// Data layout in HBM: the leaf-ordered rows, row-major -- the image of
// leaves_raw.idx.  A row of L floats is L/8 chunks of 32 bytes; the distance
// kernel reads a row four chunks (one 128-byte line) at a time and stops at
// the line where the row abandons.  Distances follow the reference's
// summation order exactly (hg_arith.cuh).
#include <cuda_runtime.h>
#include <stdint.h>

#include "hg_arith.cuh"
#include "hg_gen.cuh"
#include "hg_device.cuh"
#include "hg_kernels.h"

namespace hg {

// Mean and stdev of v[from, to) in the order of calc_mean_stdev_SIMD: the
// lanes compute the 8-chunk sums in parallel, then every lane accumulates
// them in chunk order (identical warp-uniform result).
__device__ void warp_mean_stdev(const float* v, int from, int to, float* mean, float* stdev) {
  const int lane = threadIdx.x & 31;
  const int count = to - from;
  if (count <= 0) {
    *mean = 0.0f;
    *stdev = 0.0f;
    return;
  }
  const int nch = (count + 7) >> 3;
  float sum = 0.0f, sumsq = 0.0f;
  for (int base = 0; base < nch; base += 32) {
    const int c = base + lane;
    float cs = 0.0f, cq = 0.0f;
    if (c < nch) {
      float x[8], x2[8];
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const int i = c * 8 + j;
        x[j] = i < count ? v[from + i] : 0.0f;
        x2[j] = __fmul_rn(x[j], x[j]);
      }
      cs = hg_hsum8(x[0], x[1], x[2], x[3], x[4], x[5], x[6], x[7]);
      cq = hg_hsum8(x2[0], x2[1], x2[2], x2[3], x2[4], x2[5], x2[6], x2[7]);
    }
    const int lim = min(32, nch - base);
    for (int j = 0; j < lim; ++j) {
      sum = __fadd_rn(sum, __shfl_sync(HG_FULL, cs, j));
      sumsq = __fadd_rn(sumsq, __shfl_sync(HG_FULL, cq, j));
    }
  }
  const float fc = (float)count;
  *mean = __fdiv_rn(sum, fc);
  sumsq = __fsub_rn(sumsq, __fdiv_rn(__fmul_rn(sum, sum), fc));
  *stdev = __fsqrt_rn(__fdiv_rn(sumsq, fc));
}

// Walks the tree from the root (node_split_policy_route_to_left,
// hercules_node_split.c:172-193).  Returns the leaf index.
__device__ int warp_route(const float* q, const Tree& t) {
  int node = t.root;
  while (node >= 0) {
    const DNode n = t.nodes[node];
    float m, s;
    warp_mean_stdev(q, n.from, n.to, &m, &s);
    const float v = n.idx ? s : m;
    node = (v < n.value) ? n.left : n.right;
  }
  return ~node;
}

__device__ __forceinline__ uint32_t tiles_of_leaf(uint64_t start, uint32_t size) {
  if (size == 0) return 0;
  return (uint32_t)(((start + size - 1) >> 5) - (start >> 5) + 1);
}

// ---------------------------------------------------------------------------
// block-wide helpers
// ---------------------------------------------------------------------------

template <int THREADS>
__device__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* tmp /* THREADS/32 + 1 */, uint32_t* total) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  uint32_t x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(HG_FULL, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) tmp[w] = x;
  __syncthreads();
  if (w == 0) {
    uint32_t s = lane < THREADS / 32 ? tmp[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(HG_FULL, s, o);
      if (lane >= o) s += y;
    }
    if (lane < THREADS / 32) tmp[lane] = s;
    if (lane == THREADS / 32 - 1) tmp[THREADS / 32] = s;
  }
  __syncthreads();
  const uint32_t excl = x - v + (w > 0 ? tmp[w - 1] : 0);
  if (total) *total = tmp[THREADS / 32];
  __syncthreads();
  return excl;
}

// ---------------------------------------------------------------------------
// build kernels
// ---------------------------------------------------------------------------

// One series per thread: walk the current tree to a leaf.
__global__ void k_route_rows(const float* __restrict__ X, int L, const uint32_t* __restrict__ rows, uint64_t first,
                             uint32_t count, Tree t, int* __restrict__ leaf_out) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const uint64_t r = rows ? rows[i] : first + i;
  const float* x = X + r * (uint64_t)L;
  int node = t.root;
  while (node >= 0) {
    const DNode n = t.nodes[node];
    float m, s;
    hg_mean_stdev(x, n.from, n.to, &m, &s);
    const float v = n.idx ? s : m;
    node = (v < n.value) ? n.left : n.right;
  }
  leaf_out[i] = ~node;
}

// Order-preserving int image of a float for atomicMax/atomicMin.
__device__ __forceinline__ int fkey(float f) {
  int b = __float_as_int(f);
  return b >= 0 ? b : b ^ 0x7fffffff;
}

// Segment sketches (min/max of per-series segment mean and stdev) over a
// member list: node_segment_sketch_update_sketch_parallel applied to every
// member (hercules_node_split.c:86-120).  Min/max are order independent and
// fmaxf/fminf ignore NaN, so skipping NaN gives the same envelope.
// keys_out: nsegs x 4 ints {max mean, min mean, max stdev, min stdev}.
__global__ void k_sketch_members(const float* __restrict__ X, int L, const uint32_t* __restrict__ members,
                                 uint32_t count, const short* __restrict__ seg_from,
                                 const short* __restrict__ seg_to, int nsegs, int* __restrict__ keys_out) {
  extern __shared__ int sk[];  // nsegs x 4
  for (int i = threadIdx.x; i < nsegs; i += blockDim.x) {
    sk[4 * i + 0] = INT_MIN;
    sk[4 * i + 1] = INT_MAX;
    sk[4 * i + 2] = INT_MIN;
    sk[4 * i + 3] = INT_MAX;
  }
  __syncthreads();
  for (uint32_t m = blockIdx.x * blockDim.x + threadIdx.x; m < count; m += gridDim.x * blockDim.x) {
    const float* x = X + (uint64_t)members[m] * L;
    for (int s = 0; s < nsegs; ++s) {
      float mean, sd;
      hg_mean_stdev(x, seg_from[s], seg_to[s], &mean, &sd);
      if (mean == mean) {
        atomicMax(&sk[4 * s + 0], fkey(mean));
        atomicMin(&sk[4 * s + 1], fkey(mean));
      }
      if (sd == sd) {
        atomicMax(&sk[4 * s + 2], fkey(sd));
        atomicMin(&sk[4 * s + 3], fkey(sd));
      }
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < nsegs; i += blockDim.x) {
    atomicMax(&keys_out[4 * i + 0], sk[4 * i + 0]);
    atomicMin(&keys_out[4 * i + 1], sk[4 * i + 1]);
    atomicMax(&keys_out[4 * i + 2], sk[4 * i + 2]);
    atomicMin(&keys_out[4 * i + 3], sk[4 * i + 3]);
  }
}

__global__ void k_route_flags(const float* __restrict__ X, int L, const uint32_t* __restrict__ members,
                              uint32_t count, short from, short to, int idx, float value,
                              uint8_t* __restrict__ flags) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  float m, s;
  hg_mean_stdev(X + (uint64_t)members[i] * L, from, to, &m, &s);
  flags[i] = ((idx ? s : m) < value) ? 1 : 0;
}

// rows[r] = X[perm[r]], one thread per 16 bytes (a row is L/4 of them).
__global__ void k_gather_rows(const float* __restrict__ X, int L, const uint32_t* __restrict__ perm, uint64_t n,
                              float* __restrict__ rows) {
  const int v4 = L >> 2;
  const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const uint64_t r = t / v4;
  if (r >= n) return;
  const int j = (int)(t % v4);
  reinterpret_cast<float4*>(rows + r * L)[j] = reinterpret_cast<const float4*>(X + (uint64_t)perm[r] * L)[j];
}

// iSAX word of every leaf-ordered row (sax_from_ts, sax.c:86-135).
__global__ void k_sax_rows(const float* __restrict__ rows, int L, uint64_t n, const float* __restrict__ bp,
                           uint8_t* __restrict__ sax) {
  __shared__ float sbp[256];
  for (int i = threadIdx.x; i < 255; i += blockDim.x) sbp[i] = bp[i];
  __syncthreads();
  const uint64_t row = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= n) return;
  const int per = L / HG_PAA_SEGMENTS;
  const float* x = rows + row * L;
  uint8_t w[16];
  for (int s = 0; s < HG_PAA_SEGMENTS; ++s) {
    float acc = 0.0f;
    for (int i = 0; i < per; ++i) acc = __fadd_rn(acc, x[s * per + i]);
    w[s] = (uint8_t)hg_sax_symbol(__fdiv_rn(acc, (float)per), sbp);
  }
  uint4 out;
  out.x = w[0] | (w[1] << 8) | (w[2] << 16) | ((uint32_t)w[3] << 24);
  out.y = w[4] | (w[5] << 8) | (w[6] << 16) | ((uint32_t)w[7] << 24);
  out.z = w[8] | (w[9] << 8) | (w[10] << 16) | ((uint32_t)w[11] << 24);
  out.w = w[12] | (w[13] << 8) | (w[14] << 16) | ((uint32_t)w[15] << 24);
  reinterpret_cast<uint4*>(sax)[row] = out;
}

// ---------------------------------------------------------------------------
// query kernels
// ---------------------------------------------------------------------------

// One warp: route the query (approximate_knn_search's traversal), compute
// its PAA, and set the first scan phase to the approximate leaf with an
// unbounded k-th distance.
__global__ void k_query_prep(const float* __restrict__ q, int L, Tree t, const uint64_t* __restrict__ leaf_start,
                             const uint32_t* __restrict__ leaf_size, int* approx_leaf, float* paa, int* cand,
                             float* cand_lb, int* cand_count, uint32_t* unit_prefix, uint32_t* bound,
                             int* topk_count, uint32_t* counters) {
  const int lane = threadIdx.x & 31;
  if (lane < 6) counters[lane] = 0;
  const int leaf = warp_route(q, t);
  if (lane < HG_PAA_SEGMENTS) {
    const int per = L / HG_PAA_SEGMENTS;
    float acc = 0.0f;
    for (int i = 0; i < per; ++i) acc = __fadd_rn(acc, q[lane * per + i]);
    paa[lane] = __fdiv_rn(acc, (float)per);
  }
  if (lane == 0) {
    *approx_leaf = leaf;
    cand[0] = leaf;
    cand_lb[0] = 0.0f;
    *cand_count = 1;
    unit_prefix[0] = 0;
    unit_prefix[1] = tiles_of_leaf(leaf_start[leaf], leaf_size[leaf]);
    *bound = 0x7f800000u;  // +inf
    *topk_count = 0;
  }
}

__global__ void k_route_queries(const float* __restrict__ Q, int nq, int L, Tree t, int* __restrict__ leaf_out) {
  const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (w >= nq) return;
  const int leaf = warp_route(Q + (uint64_t)w * L, t);
  if ((threadIdx.x & 31) == 0) leaf_out[w] = leaf;
}

// LB_EAPCA of every leaf (a warp per leaf).  With sax_tab set, the
// threads also write the query's LB_SAX term table for the filter:
// sax_tab[t * 256 + s] = hg_lb_sax_lane(paa[t], s) (reference arithmetic,
// sax.c:310-479), 4,096 entries, computed once per query.
__global__ void k_leaf_lb(const float* __restrict__ q, int L, int nleaves, const int* __restrict__ seg_off,
                          const short* __restrict__ points, const float* __restrict__ sk, float* __restrict__ lb,
                          const float* __restrict__ paa, const float* __restrict__ bp, float* __restrict__ sax_tab) {
  extern __shared__ float qs[];
  if (sax_tab) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < HG_PAA_SEGMENTS * HG_SAX_CARD;
         i += gridDim.x * blockDim.x)
      sax_tab[i] = hg_lb_sax_lane(paa[i >> 8], i & 255, bp);
  }
  for (int i = threadIdx.x; i < L; i += blockDim.x) qs[i] = q[i];
  __syncthreads();
  const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (w >= nleaves) return;
  const int off = seg_off[w], nseg = seg_off[w + 1] - off;
  float sum = 0.0f;
  int start = 0;
  for (int s = 0; s < nseg; ++s) {
    const int end = points[off + s];
    float m, sd;
    warp_mean_stdev(qs, start, end, &m, &sd);
    sum = __fadd_rn(sum, hg_eapca_term(m, sd, sk + 4 * (off + s), end - start));
    start = end;
  }
  if ((threadIdx.x & 31) == 0) lb[w] = sum;
}

// Mean and stdev of every query over every distinct leaf segment (leaves
// share most of their segments: a split refines its parent's), with the
// reference arithmetic of calculate_node_min_distance's calc_mean_stdev_SIMD:
// one block per query, a warp per segment (warp_mean_stdev for segments of 64
// points or more, else hg_mean_stdev on one lane).  out[q * nu + u].
__global__ void k_query_segstats(const float* __restrict__ Q, int L, int nq, const short* __restrict__ useg_start,
                                 const short* __restrict__ useg_end, int nu, float2* __restrict__ out) {
  extern __shared__ float qs[];
  const int q = blockIdx.x;
  if (q >= nq) return;
  for (int i = threadIdx.x; i < L; i += blockDim.x) qs[i] = Q[(uint64_t)q * L + i];
  __syncthreads();
  const int lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  for (int u = threadIdx.x >> 5; u < nu; u += nw) {
    const int start = useg_start[u], end = useg_end[u];
    float m, sd;
    if (end - start >= 64) {
      warp_mean_stdev(qs, start, end, &m, &sd);
    } else {
      hg_mean_stdev(qs, start, end, &m, &sd);  // every lane, the same values
    }
    if (lane == 0) out[(uint64_t)q * nu + u] = make_float2(m, sd);
  }
}

// Leaves each query of a batch must filter: a thread per (query, leaf) sums
// the LB_EAPCA terms of the leaf's segments in order (the plain path's
// k_leaf_lb arithmetic, segment statistics from k_query_segstats; the terms
// are >= 0, so the sum stops once it exceeds the limit) and keeps the leaf
// when
//     LB <= B_q (1 + 2^-10) + L 2^-20,
// B_q the query's bound (+inf keeps every leaf).  The plain path scans only
// leaves with LB <= its running bound <= B_q, so the kept leaves include
// every leaf it scans; the margins cover the rounding of B_q's product.
// Kept (leaf, query) pairs go to leaf_q[leaf * stride + i], counted in
// leaf_cnt[leaf].
// qlist (optional): the queries are qlist[0 .. *nq_dev) instead of 0 .. nq.
// A thread per (query, leaf) pair, grid-stride (a warp per pair, with the
// sum's order kept through shuffles, made the bound phase 0.33 ms longer per
// batch of 4,096 queries at 25M x 256).
__global__ void k_leaf_keep(const float2* __restrict__ segstats, int nu, int L, int nq,
                            const int* __restrict__ seg_off, const short* __restrict__ points,
                            const int* __restrict__ seg_uid, const float* __restrict__ sk,
                            const uint32_t* __restrict__ leaf_size, int nleaves, const float* __restrict__ bound,
                            uint32_t* leaf_cnt, uint32_t* leaf_q, uint32_t stride, const uint32_t* qlist,
                            const uint32_t* nq_dev) {
  const uint64_t n = (uint64_t)(nq_dev ? min((uint32_t)nq, *nq_dev) : (uint32_t)nq) * nleaves;
  const uint64_t nt = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; g < n; g += nt) {
    const int qi = (int)(g / nleaves), w = (int)(g % nleaves);
    const int q = qlist ? (int)qlist[qi] : qi;
    if (leaf_size[w] == 0) continue;
    const float B = bound[q];
    const float lim = B < __int_as_float(0x7f800000)
                          ? __fadd_ru(__fmul_ru(B, 1.0f + 0x1p-10f), __fmul_ru((float)L, 0x1p-20f))
                          : __int_as_float(0x7f800000);
    const int off = seg_off[w], nseg = seg_off[w + 1] - off;
    const float2* st = segstats + (uint64_t)q * nu;
    float sum = 0.0f;
    int start = 0;
    for (int s = 0; s < nseg; ++s) {
      const int end = points[off + s];
      const float2 ms = st[seg_uid[off + s]];
      sum = __fadd_rn(sum, hg_eapca_term(ms.x, ms.y, sk + 4 * (off + s), end - start));
      start = end;
      if (!(sum <= lim)) break;
    }
    if (sum <= lim) leaf_q[(uint64_t)w * stride + atomicAdd(&leaf_cnt[w], 1u)] = (uint32_t)q;
  }
}

// Candidate leaves: LB_EAPCA <= current bound, not the approximate leaf, not
// empty; ordered by LB with a stable LSD radix sort (4-bit digits, 8 passes)
// in one CTA; then the exclusive prefix of their tile counts.
constexpr int kSortThreads = 1024;
__global__ void __launch_bounds__(kSortThreads) k_select_sort(const float* __restrict__ lb, int nleaves,
                                                              const uint32_t* bound, const int* approx_leaf,
                                                              const uint64_t* __restrict__ leaf_start,
                                                              const uint32_t* __restrict__ leaf_size, int* cand,
                                                              float* cand_lb, int* cand_count,
                                                              uint32_t* unit_prefix, uint32_t* gkeys) {
  // keys and values (two buffers each) live in shared memory up to
  // kMaxLeavesSort leaves, else in gkeys (4 x nleaves words of global memory)
  extern __shared__ uint32_t sm[];
  uint32_t* cnt = sm;  // 16 x kSortThreads digit counts
  uint32_t* kbase = gkeys ? gkeys : sm + 16 * kSortThreads;
  const int cap = gkeys ? nleaves : kMaxLeavesSort;
  uint32_t* keys0 = kbase;
  uint32_t* vals0 = keys0 + cap;
  uint32_t* keys1 = vals0 + cap;
  uint32_t* vals1 = keys1 + cap;
  __shared__ uint32_t tmp[kSortThreads / 32 + 1];
  __shared__ uint32_t total;
  const int t = threadIdx.x;
  const float B = __int_as_float((int)ld_volatile(bound));
  const int approx = *approx_leaf;
  // 1. select the non-empty leaves within the bound, the approximate leaf
  //    excepted (it was scanned first), order preserving
  const int per = (nleaves + kSortThreads - 1) / kSortThreads;
  const int b0 = min(nleaves, t * per), b1 = min(nleaves, b0 + per);
  uint32_t mine = 0;
  for (int i = b0; i < b1; ++i) {
    const float l = lb[i];
    if (leaf_size[i] > 0 && i != approx && !(l > B)) ++mine;
  }
  uint32_t pos = block_exclusive_scan<kSortThreads>(mine, tmp, &total);
  const int n = (int)total;
  for (int i = b0; i < b1; ++i) {
    const float l = lb[i];
    if (leaf_size[i] > 0 && i != approx && !(l > B)) {
      keys0[pos] = (l == l) ? __float_as_uint(l) : 0u;  // a NaN bound never prunes
      vals0[pos] = (uint32_t)i;
      ++pos;
    }
  }
  __syncthreads();
  // 2. sort by LB.  Up to kSortThreads candidates (the usual case): one
  //    bitonic sort of (LB bits, leaf) keys; the leaves are in index order on
  //    input, so equal LBs end in the order the stable radix sort below gives
  //    them, which handles larger counts.
  const int per2 = (n + kSortThreads - 1) / kSortThreads;
  const int r0 = min(n, t * per2), r1 = min(n, r0 + per2);
  uint32_t *ki = keys0, *vi = vals0, *ko = keys1, *vo = vals1;
  if (n <= kSortThreads) {
    unsigned long long* kv = reinterpret_cast<unsigned long long*>(keys1);  // 8-byte aligned, 2 x cap words (n <= 1024)
    int np = 2;
    while (np < n) np <<= 1;
    for (int i = t; i < np; i += kSortThreads)
      kv[i] = i < n ? (((unsigned long long)keys0[i] << 32) | vals0[i]) : ~0ull;
    __syncthreads();
    for (int size = 2; size <= np; size <<= 1)
      for (int stride = size >> 1; stride > 0; stride >>= 1) {
        for (int i = t; i < np / 2; i += kSortThreads) {
          const int pos = 2 * i - (i & (stride - 1));
          const int partner = pos + stride;
          const bool asc = (pos & size) == 0;
          const unsigned long long x = kv[pos], y = kv[partner];
          if ((x > y) == asc) {
            kv[pos] = y;
            kv[partner] = x;
          }
        }
        __syncthreads();
      }
    for (int i = t; i < n; i += kSortThreads) {
      keys0[i] = (uint32_t)(kv[i] >> 32);
      vals0[i] = (uint32_t)kv[i];
    }
    __syncthreads();
  }
  for (int pass = 0; n > kSortThreads && pass < 8; ++pass) {
    const int shift = pass * 4;
    uint32_t c[16];
#pragma unroll
    for (int d = 0; d < 16; ++d) c[d] = 0;
    for (int i = r0; i < r1; ++i) ++c[(ki[i] >> shift) & 15];
    // flattened digit-major counts: index d * kSortThreads + t; scan them in
    // that order (thread t owns the 16 entries t*16 .. t*16+15 of the flat array)
#pragma unroll
    for (int d = 0; d < 16; ++d) cnt[d * kSortThreads + t] = c[d];
    __syncthreads();
    uint32_t s = 0;
    uint32_t loc[16];
#pragma unroll
    for (int j = 0; j < 16; ++j) {
      loc[j] = s;
      s += cnt[t * 16 + j];
    }
    const uint32_t base = block_exclusive_scan<kSortThreads>(s, tmp, nullptr);
#pragma unroll
    for (int j = 0; j < 16; ++j) cnt[t * 16 + j] = base + loc[j];
    __syncthreads();
    uint32_t off[16];
#pragma unroll
    for (int d = 0; d < 16; ++d) off[d] = cnt[d * kSortThreads + t];
    for (int i = r0; i < r1; ++i) {
      const int d = (ki[i] >> shift) & 15;
      const uint32_t p = off[d]++;
      ko[p] = ki[i];
      vo[p] = vi[i];
    }
    __syncthreads();
    uint32_t* x = ki;
    ki = ko;
    ko = x;
    x = vi;
    vi = vo;
    vo = x;
  }
  // 3. outputs and tile prefix
  uint32_t tiles = 0;
  for (int i = r0; i < r1; ++i) {
    const int leaf = (int)vi[i];
    cand[i] = leaf;
    cand_lb[i] = __uint_as_float(ki[i]);
    tiles += tiles_of_leaf(leaf_start[leaf], leaf_size[leaf]);
  }
  uint32_t tp = block_exclusive_scan<kSortThreads>(tiles, tmp, &total);
  for (int i = r0; i < r1; ++i) {
    const int leaf = (int)vi[i];
    unit_prefix[i] = tp;
    tp += tiles_of_leaf(leaf_start[leaf], leaf_size[leaf]);
  }
  if (t == 0) {
    unit_prefix[n] = total;
    *cand_count = n;
  }
}

__global__ void k_pscan_prep(uint64_t nrows, int* cand_count, uint32_t* unit_prefix, uint32_t* bound,
                             int* topk_count, uint32_t* counters) {
  if (threadIdx.x < 4) counters[threadIdx.x] = 0;
  if (threadIdx.x == 0) {
    *cand_count = 1;
    unit_prefix[0] = 0;
    unit_prefix[1] = (uint32_t)((nrows + 31) >> 5);
    *bound = 0x7f800000u;
    *topk_count = 0;
  }
}

// ---------------------------------------------------------------------------
// The leaf scan (exact_de_knn_search's refine loop, hercules_query_engine.c:
// 2391-2425, with the per-row LB_SAX test of the reference's SIMS path,
// :2183-2211) runs as two kernels: a streaming LB_SAX filter that turns the
// candidate leaves into a compact list of surviving rows, and a distance
// stream over that list.
// ---------------------------------------------------------------------------

// Stage 1.  Work: the candidate leaves in ascending LB_EAPCA order, cut into
// 32-row units (32-aligned rows; a unit's rows outside its leaf are skipped).
// One persistent block per SM owns a contiguous range of units, ending at the
// first leaf whose LB exceeds the bound (found by the producer warp while
// the consumers build the table).  Its producer lane bulk-copies the
// units' iSAX words (a leaf's units are contiguous in memory: one
// cp.async.bulk per leaf run, 512 bytes per unit) into kFiltStages stages of
// shared memory, each guarded by a full and an empty mbarrier; 20 consumer
// warps take 3 units of every stage each (lane = row), test the rows from
// shared memory and append the survivors with one atomicAdd per warp and
// stage.  Every wait is bounded: on timeout the block raises *err, the
// producer drains the copies it issued, and the call reports HG_ERR_TIMEOUT.
//
// The per-row test is a certified lower bound of the reference's LB_SAX
// (minidist_paa_to_isax_raw_SIMD, sax.c:310-479).  The query's 16 x 256
// table of per-segment terms (k_leaf_lb, reference arithmetic) is turned,
// per block, into 8-bit terms q = floor(term * 254 / T) (rounded down at
// every step, at most 255) against the pruning threshold
// T = (B (1 + 2^-10) + 1e-6) / (L / 16); a row is pruned when its 16 terms
// add up to at least 255, which implies (L / 16) * (sum of the terms) >=
// (255 / 254) (B (1 + 2^-10) + 1e-6): the reference's float LB_SAX exceeds
// the bound with room to spare for its rounding, so every row this test
// prunes is one the exact float test prunes too (never a true neighbour).
// The 8-bit table is laid out lane-private: byte b of word
// ((h * 256 + s) * 2 + g) * 32 + lane holds that lane's term of symbol s for
// segment t = 8 h + 4 g + b, so the byte of (t, s) sits at
// (t / 8) * 65536 + ((t / 4) & 1) * 128 + (t & 3) + 256 s + 4 lane: the 16
// data-dependent lookups of a row never conflict on a bank, and one byte
// permute of the row's word and 4 lane gives each lookup's address.
constexpr int kFiltConsumers = 20;                          // consumer warps
constexpr int kFilterThreads = 32 * (kFiltConsumers + 1);   // + the producer warp
constexpr int kUnitsPerWarp = 3;                            // units of a stage per consumer warp
constexpr int kStageUnits = kFiltConsumers * kUnitsPerWarp; // 60 units: 30 KB
constexpr int kFiltStages = 3;
constexpr uint32_t kUnitBytes = 32 * 16;
constexpr uint32_t kStageBytes = kStageUnits * kUnitBytes;
constexpr int kSaxTabWords = HG_PAA_SEGMENTS * HG_SAX_CARD / 4 * 32;  // 128 KB
constexpr uint32_t kFiltSmStage = kSaxTabWords * 4;                     // stages after the table
constexpr uint32_t kFiltSmBar = kFiltSmStage + kFiltStages * kStageBytes;  // 2 x kFiltStages mbarriers
constexpr uint32_t kFiltSmMeta = kFiltSmBar + 2 * kFiltStages * 8;  // end unit, abort flag, first candidate
constexpr uint64_t kFiltWaitNs = 2000000000ull;                           // 2 s per wait
size_t lbsax_filter_smem() { return kFiltSmMeta + 16; }

__device__ __forceinline__ uint32_t sax_qterm(float term, float scale) {
  const float p = __fmul_rd(term, scale);
  return p >= 255.0f ? 255u : (uint32_t)p;
}

__device__ __forceinline__ bool fl_try(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ uint64_t fl_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
// Bounded wait for the phase of `parity`: false when the block aborted or
// the wait ran out (then the block aborts and *err is raised).
__device__ __noinline__ bool fl_wait_slow(uint32_t bar, uint32_t parity, volatile int* abort_flag, int* err) {
  const uint64_t t0 = fl_ns();
  for (uint32_t i = 1;; ++i) {
    if (fl_try(bar, parity)) return true;
    if ((i & 63) == 0) {
      if (*abort_flag) return false;
      if (fl_ns() - t0 > kFiltWaitNs) {
        *abort_flag = 1;
        if (err) atomicExch(err, 1);
        return false;
      }
    }
  }
}

// the first test inline, the polling loop out of line
__device__ __forceinline__ bool fl_wait(uint32_t bar, uint32_t parity, volatile int* abort_flag, int* err) {
  return fl_try(bar, parity) || fl_wait_slow(bar, parity, abort_flag, err);
}

__global__ void __launch_bounds__(kFilterThreads, 1) k_lbsax_filter(FilterArgs a) {
  extern __shared__ __align__(16) unsigned char fsm[];
  uint32_t* qtab = reinterpret_cast<uint32_t*>(fsm);
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const uint32_t sbase = (uint32_t)__cvta_generic_to_shared(fsm);
  auto full_bar = [&](int st) { return sbase + kFiltSmBar + 8u * st; };
  auto empty_bar = [&](int st) { return sbase + kFiltSmBar + 8u * (kFiltStages + st); };
  volatile uint32_t* s_uend = reinterpret_cast<volatile uint32_t*>(fsm + kFiltSmMeta);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(fsm + kFiltSmMeta + 4);
  const float B = __int_as_float((int)ld_volatile(a.bound));
  // candidates [clo, chi) of the sorted list (all of them by default); this
  // block's contiguous range of their units
  const int ncand = *a.cand_count;
  const int clo = min(a.cand_lo, ncand);
  const int chi = a.cand_hi > 0 ? min(a.cand_hi, ncand) : ncand;
  const uint32_t ubase = clo < chi ? a.unit_prefix[clo] : 0u;
  const uint32_t total = clo < chi ? a.unit_prefix[chi] - ubase : 0u;
  const uint32_t per_block = (total + gridDim.x - 1) / gridDim.x;
  const uint32_t u0 = ubase + blockIdx.x * per_block;
  const uint32_t u1 = min(ubase + total, u0 + per_block);
  volatile int* s_c0 = reinterpret_cast<volatile int*>(fsm + kFiltSmMeta + 8);
  if (wib == kFiltConsumers) {
    // the producer warp finds the block's first candidate and where its
    // range ends -- at the first leaf whose LB exceeds the bound (LBs ascend
    // along the list, so every later unit is past it too) -- with 32-way
    // searches, sets up the barriers and hands both to the consumers
    // through named barrier 1, while they build the table
    int c0 = clo;
    uint32_t ue = u0;
    if (u0 < u1) {
      c0 = unit_candidate_warp(a.unit_prefix, ncand, clo, u0, lane);
      ue = u1;
      for (int cb = c0; cb < chi; cb += 32) {
        const int c = cb + lane;
        const bool in_range = c < chi && a.unit_prefix[c] < u1;
        const uint32_t past = __ballot_sync(HG_FULL, in_range && a.cand_lb[c] > B);
        if (past) {
          ue = max(u0, a.unit_prefix[cb + __ffs(past) - 1]);
          break;
        }
        if (!__all_sync(HG_FULL, in_range)) break;
      }
    }
    if (lane == 0) {
      *s_uend = ue;
      *s_c0 = c0;
      *abort_flag = 0;
      for (int st = 0; st < kFiltStages; ++st) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(full_bar(st)), "r"(1) : "memory");
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(empty_bar(st)), "r"(kFiltConsumers) : "memory");
      }
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncwarp();
    asm volatile("bar.arrive 1, %0;" ::"r"(kFilterThreads) : "memory");
  } else if (a.use_lbsax) {
    const float Bs = __fadd_rn(__fmul_rn(B, 1.0009765625f), 1e-6f);
    const float T = __fdiv_ru(Bs, (float)(a.L / HG_PAA_SEGMENTS));
    const float scale = __fdiv_rd(254.0f, T);  // 0 when the bound is +inf: nothing is pruned
    for (int g = threadIdx.x; g < kSaxTabWords / 32; g += 32 * kFiltConsumers) {
      // the terms of symbol s for segments t0 .. t0 + 3
      const int sym = (g >> 1) & (HG_SAX_CARD - 1), t0 = 8 * (g >> 9) + 4 * (g & 1);
      const float* col = a.sax_tab + t0 * HG_SAX_CARD + sym;
      const uint32_t packed = sax_qterm(col[0], scale) | (sax_qterm(col[HG_SAX_CARD], scale) << 8) |
                              (sax_qterm(col[2 * HG_SAX_CARD], scale) << 16) |
                              (sax_qterm(col[3 * HG_SAX_CARD], scale) << 24);
#pragma unroll 8
      for (int r = 0; r < 32; ++r) qtab[g * 32 + ((r + lane) & 31)] = packed;
    }
  }
  if (wib != kFiltConsumers) asm volatile("bar.sync 1, %0;" ::"r"(kFilterThreads) : "memory");
  const uint32_t uend = *s_uend;
  const int c0 = *s_c0;
  const uint32_t nstages = (uend - u0 + kStageUnits - 1) / kStageUnits;  // 0 when u0 == uend
  if (wib == kFiltConsumers) {
    // ---------------- producer: bulk copies of whole units, leaf by leaf
    if (lane == 0 && nstages) {
      int c = c0;
      uint32_t k = 0;
      bool ok = true;
      for (; k < nstages; ++k) {
        const int st = (int)(k % kFiltStages);
        ok = fl_wait(empty_bar(st), ((k / kFiltStages) & 1) ^ 1, abort_flag, a.err);
        if (!ok) break;
        const uint32_t us = u0 + k * kStageUnits, ue = min(uend, us + kStageUnits);
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(full_bar(st)),
                     "r"((ue - us) * kUnitBytes)
                     : "memory");
        for (uint32_t u = us; u < ue;) {
          while (c + 1 < ncand && a.unit_prefix[c + 1] <= u) ++c;
          const uint32_t run_end = min(ue, c + 1 < ncand ? a.unit_prefix[c + 1] : ue);
          const uint64_t first_row = ((a.leaf_start[a.cand[c]] >> 5) + (u - a.unit_prefix[c])) << 5;
          const unsigned char* src = a.sax + first_row * 16;
          const uint32_t dst = sbase + kFiltSmStage + (uint32_t)st * kStageBytes + (u - us) * kUnitBytes;
          asm volatile(
              "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
              "l"(reinterpret_cast<uint64_t>(src)), "r"((run_end - u) * kUnitBytes), "r"(full_bar(st))
              : "memory");
          u = run_end;
        }
      }
      // leaving early: the copies in flight land before the block exits
      if (!ok) {
        const uint32_t first = k > (uint32_t)kFiltStages ? k - kFiltStages : 0u;
        for (uint32_t kk = first; kk < k; ++kk) {
          const uint64_t t0 = fl_ns();
          while (!fl_try(full_bar((int)(kk % kFiltStages)), (kk / kFiltStages) & 1) && fl_ns() - t0 < kFiltWaitNs) {
          }
        }
      }
    }
  } else {
    // ---------------- consumers: lane = row of a unit
    const unsigned char* tb = fsm;
    const uint32_t lanev = (uint32_t)(4 * lane);  // byte 0: 4 lane, bytes 1..3: zero
    const uint32_t lt = (1u << lane) - 1;
    int c = c0;  // the body moves it forward to each unit's candidate
    uint32_t next_c = c + 1 < ncand ? a.unit_prefix[c + 1] : 0xffffffffu;
    int cur = -1;
    uint32_t lstart = 0, lend = 0, first_unit = 0;
    uint32_t n_rows = 0, n_pass = 0, n_leaves = 0;  // lane 0's counts
    for (uint32_t k = 0; k < nstages; ++k) {
      const int st = (int)(k % kFiltStages);
      int got = 1;
      if (lane == 0) got = fl_wait(full_bar(st), (k / kFiltStages) & 1, abort_flag, a.err) ? 1 : 0;
      if (!__shfl_sync(HG_FULL, got, 0)) break;
      const uint32_t us = u0 + k * kStageUnits, ue = min(uend, us + kStageUnits);
      const uint4* stage = reinterpret_cast<const uint4*>(fsm + kFiltSmStage + st * kStageBytes);
      uint32_t m[kUnitsPerWarp], rr[kUnitsPerWarp];
      uint32_t cnt = 0;
#pragma unroll
      for (int i = 0; i < kUnitsPerWarp; ++i) {
        const uint32_t slot = (uint32_t)(wib * kUnitsPerWarp + i), unit = us + slot;
        m[i] = 0;
        rr[i] = 0;
        if (unit >= ue) continue;  // uniform over the warp
        while (unit >= next_c) {
          ++c;
          next_c = c + 1 < ncand ? a.unit_prefix[c + 1] : 0xffffffffu;
        }
        if (c != cur) {
          cur = c;
          const int leaf = a.cand[c];
          lstart = (uint32_t)a.leaf_start[leaf];
          lend = lstart + a.leaf_size[leaf];
          first_unit = a.unit_prefix[c];
        }
        const uint32_t tile_in = unit - first_unit;
        n_leaves += tile_in == 0 ? 1u : 0u;
        rr[i] = (((lstart >> 5) + tile_in) << 5) + lane;
        bool pass = rr[i] >= lstart && rr[i] < lend;
        n_rows += (uint32_t)__popc(__ballot_sync(HG_FULL, pass));
        if (pass && a.use_lbsax) {
          // byte j of word q is the symbol s of segment t = 4 q + j; the
          // permute puts s in byte 1 and 4 lane in byte 0: 256 s + 4 lane,
          // the lookup's offset from segment t's fixed base
          const uint4 w = stage[slot * 32 + lane];
          const uint32_t ws[4] = {w.x, w.y, w.z, w.w};
          uint32_t sum = 0;
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            const int tq = (q >> 1) * 65536 + (q & 1) * 128;
            sum += (uint32_t)tb[tq + __byte_perm(ws[q], lanev, 0x5504)] +
                   (uint32_t)tb[tq + 1 + __byte_perm(ws[q], lanev, 0x5514)] +
                   (uint32_t)tb[tq + 2 + __byte_perm(ws[q], lanev, 0x5524)] +
                   (uint32_t)tb[tq + 3 + __byte_perm(ws[q], lanev, 0x5534)];
          }
          pass = sum < 255u;
        }
        m[i] = __ballot_sync(HG_FULL, pass);
        cnt += (uint32_t)__popc(m[i]);
      }
      // the stage's words are read: hand it back to the producer
      __syncwarp();
      if (lane == 0) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(empty_bar(st)) : "memory");
      n_pass += cnt;
      uint32_t pos = 0;
      if (lane == 0 && cnt) pos = atomicAdd(a.list_count, cnt);
      pos = __shfl_sync(HG_FULL, pos, 0);
#pragma unroll
      for (int i = 0; i < kUnitsPerWarp; ++i) {
        if ((m[i] >> lane) & 1u) a.list[pos + __popc(m[i] & lt)] = rr[i];
        pos += __popc(m[i]);
      }
    }
    // rows considered, pruned (considered minus survivors) and leaves visited
    if (lane == 0) {
      atomicAdd(&a.stats[0], (unsigned long long)n_rows);
      atomicAdd(&a.stats[2], (unsigned long long)(n_rows - n_pass));
      atomicAdd(&a.stats[3], (unsigned long long)n_leaves);
    }
  }
}

// Stage 2: the early-abandoning squared distance (ts_euclidean_distance_SIMD,
// ts.c:83-109) over a row list, or over a row range when there is no list.
//
// A warp works on 8 rows at a time, 4 lanes per row ("slot").  Per step the
// 4 lanes of a slot load one 128-byte line of their row (chunk ch + j in
// lane j), each computes its 8-float chunk sum, and the slot adds the 4 chunk
// sums to the running distance in chunk order (shuffles), testing the bound
// after each (a strict test: a row whose distance equals the bound finishes,
// so ties keep the lowest id).  A slot whose row abandoned or finished takes
// the next row of its warp's batch: warp w of W owns the 32-entry batches w,
// w + W, w + 2W, ... of the list, and the next batch's entries are loaded
// while the current one is consumed.  Finished rows within the bound enter
// the warp's top-k list, which lowers the global bound (atomicMin) once it
// holds k distances.  The query lives in shared memory in blocks of 32
// chunks (40 float4 pairs each): chunk r of a block sits at pair r + r / 4,
// so the slots of a warp, which sit at different 4-chunk positions, read
// different banks.
constexpr int kEdThreads = 256;
__device__ __forceinline__ int q4_index(int chunk, int half) {
  const int r = chunk & 31;
  return ((chunk >> 5) * 40 + r + (r >> 2)) * 2 + half;
}
// bytes of that layout for a series of L floats
__host__ __device__ inline size_t q4_bytes(int L) { return (size_t)((L / 8 + 31) / 32) * 40 * 2 * 16; }
// kRowIds: the id of a row is its row index (a matrix without an id map).
// kSlot: lanes per row (a slot); kLines: 32-byte chunks per lane of a row in
// flight per step, so a slot reads kSlot * kLines * 32 bytes of its row per
// step.  Short series use 4-lane slots (8 rows per warp, 128-byte lines);
// long series, few candidate rows per query, use wider slots.
template <int kSlot>
__host__ __device__ constexpr uint32_t slot_leaders() {
  return kSlot == 32 ? 0x1u : (kSlot == 16 ? 0x10001u : (kSlot == 8 ? 0x01010101u : 0x11111111u));
}
template <bool kRowIds, int kLines, int kSlot>
__global__ void __launch_bounds__(kEdThreads, kLines > 2 ? 3 : 4) k_ed_stream(EdArgs a) {
  constexpr int W = kEdThreads / 32;
  __shared__ unsigned long long lists[W][kWarpListCap];
  extern __shared__ float4 qs4[];  // the query, q4_bytes(L) bytes
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int slot_lead = lane & ~(kSlot - 1), j = lane & (kSlot - 1);
  if (a.gate && *a.gate == 0) {
    // a gated launch that did not pass: the block reports an empty list
    if (threadIdx.x == 0) a.part_count[blockIdx.x] = 0;
    return;
  }
  unsigned long long* list = lists[wib];
  for (int i = lane; i < kWarpListCap; i += 32) list[i] = ~0ull;
  for (int i = threadIdx.x; i < (a.L >> 2); i += blockDim.x)
    qs4[q4_index(i >> 1, i & 1)] = reinterpret_cast<const float4*>(a.q)[i];
  __syncthreads();
  const int nch = a.L >> 3;
  uint64_t first = a.ident_first;
  uint32_t total;
  if (a.list) {
    total = *a.list_count;
  } else if (a.ident_leaf) {
    const int leaf = *a.ident_leaf;
    first = a.leaf_start[leaf];
    total = a.leaf_size[leaf];
  } else {
    total = (uint32_t)a.ident_count;
  }
  const uint32_t nwarps = gridDim.x * W;
  const uint32_t gw = blockIdx.x * W + wib;
  const uint32_t leaders = slot_leaders<kSlot>();
  // batch b of this warp covers entries [(gw + b * nwarps) * bs, +bs): bs
  // spreads a short list over all warps (a few long rows keep every warp busy)
  const uint32_t per_warp = (uint32_t)(((uint64_t)total + nwarps - 1) / nwarps);
  const uint32_t bs = per_warp < 1u ? 1u : (per_warp > 32u ? 32u : per_warp);
  auto entry = [&](uint32_t batch) -> uint32_t {
    const uint64_t idx = (uint64_t)batch * bs + lane;
    if ((uint32_t)lane >= bs || idx >= total) return 0xffffffffu;
    return a.list ? a.list[idx] : (uint32_t)(first + idx);
  };
  auto count_of = [&](uint32_t batch) -> uint32_t {
    const uint64_t b0 = (uint64_t)batch * bs;
    return b0 < total ? (uint32_t)(total - b0 < bs ? total - b0 : bs) : 0u;
  };
  uint32_t batch = gw;
  uint32_t cur = entry(batch);  // lane i holds entry i of the current batch
  uint32_t cur_n = count_of(batch);
  uint32_t cur_used = 0;
  batch += nwarps;
  uint32_t nxt = entry(batch);
  uint32_t nxt_n = count_of(batch);

  int cnt = 0;
  float T = __int_as_float(0x7f800000);
  float B = __int_as_float((int)ld_volatile(a.bound));
  const float F = a.has_floor ? a.floor : -1.0f;  // distances are >= 0
  bool valid = false;  // slot-uniform
  uint32_t row = 0;
  int ch = 0;  // a multiple of kStep: the query offsets below stay inside one 32-chunk group
  float dist = 0.0f;
  const float4* x = nullptr;
  uint32_t n_chunks = 0, n_done = 0, n_rows = 0;  // this lane's (slot leaders only)
  constexpr int kStep = kSlot * kLines;  // chunks of a row per step
  static_assert(32 % kStep == 0, "a step stays inside one 32-chunk group of the staged query");
  // staged-query float4 index of chunk ch + kSlot l + j: base(ch) + qoff[l]
  int qoff[kLines];
#pragma unroll
  for (int l = 0; l < kLines; ++l) {
    const int o = kSlot * l + j;
    qoff[l] = 2 * (o + (o >> 2));
  }
  for (int iter = 1;; ++iter) {
    // refill the slots without a row
    uint32_t need = __ballot_sync(HG_FULL, !valid) & leaders;
    while (need) {
      if (cur_used == cur_n) {
        if (nxt_n == 0) break;
        cur = nxt;
        cur_n = nxt_n;
        cur_used = 0;
        batch += nwarps;
        nxt = entry(batch);  // loaded while the current batch is consumed
        nxt_n = count_of(batch);
      }
      const int take = min(__popc(need), (int)(cur_n - cur_used));
      const int r = __popc(need & ((1u << slot_lead) - 1));  // rank among the free slots
      const bool mine = ((need >> slot_lead) & 1u) && r < take;
      const uint32_t got = __shfl_sync(HG_FULL, cur, (cur_used + (mine ? r : 0)) & 31);
      if (mine) {
        row = got;
        valid = true;
        dist = 0.0f;
        ch = 0;
        x = reinterpret_cast<const float4*>(a.rows + (uint64_t)row * a.L) + 2 * j;
        if (j == 0) ++n_rows;
      }
      cur_used += take;
      need = __ballot_sync(HG_FULL, !valid) & leaders;
    }
    if (!__any_sync(HG_FULL, valid)) break;
    const uint32_t bnext = ((iter & 7) == 0) ? ld_volatile(a.bound) : 0x7f800000u;
    // kLines chunks of every owned row in flight: lane j computes chunks
    // ch + kSlot l + j (l < kLines); chunks past the row's end count as 0
    float4 xv[kLines][2];
    bool in[kLines];
#pragma unroll
    for (int l = 0; l < kLines; ++l) {
      in[l] = valid && ch + kSlot * l + j < nch;
      if (in[l]) {
        xv[l][0] = __ldcs(x + 2 * kSlot * l);
        xv[l][1] = __ldcs(x + 2 * kSlot * l + 1);
      }
    }
    // a slot without a row (its ch may equal nch) reads the first chunks:
    // every index stays inside the staged query
    const int cq = valid ? ch : 0;
    const int qb = 2 * ((cq >> 5) * 40 + (cq & 31) + ((cq & 31) >> 2));
    float dl[kLines];
#pragma unroll
    for (int l = 0; l < kLines; ++l) {
      const float4 q0 = qs4[qb + qoff[l]], q1 = qs4[qb + qoff[l] + 1];
      const float qa[8] = {q0.x, q0.y, q0.z, q0.w, q1.x, q1.y, q1.z, q1.w};
      const float xa[8] = {xv[l][0].x, xv[l][0].y, xv[l][0].z, xv[l][0].w,
                           xv[l][1].x, xv[l][1].y, xv[l][1].z, xv[l][1].w};
      const float d = hg_chunk_d2(qa, xa);
      dl[l] = in[l] ? d : 0.0f;
    }
    // the slot adds the step's chunk sums in order (adding 0 leaves a sum
    // unchanged); one abandon test per step, since the step's lines are
    // already loaded
    float part[kStep];
    float acc = dist;
#pragma unroll
    for (int t = 0; t < kStep; ++t) {
      acc = __fadd_rn(acc, __shfl_sync(HG_FULL, dl[t / kSlot], slot_lead + (t % kSlot)));
      part[t] = acc;
    }
    bool finished = false;
    if (valid) {
      if (acc > B) {
        // abandoned: the reference reads up to the first chunk whose sum
        // exceeds the bound (the partial sums never decrease)
        if (j == 0) {
          int used = 1;
#pragma unroll
          for (int t = 0; t < kStep; ++t) used += part[t] <= B ? 1 : 0;
          n_chunks += (uint32_t)(ch + used);
        }
        valid = false;
      } else {
        dist = acc;
        ch += kStep;
        x += 2 * kStep;
        if (ch >= nch) {
          finished = true;
          valid = false;
          if (j == 0) {
            n_chunks += (uint32_t)nch;
            ++n_done;
          }
        }
      }
    }
    const bool take = finished && j == 0 && dist <= B && dist <= T && dist > F;
    warp_list_add(list, cnt, T, a.k, a.bound, take, dist,
                  take ? (kRowIds ? row : (uint32_t)a.ids[row]) : 0u);
    B = fminf(fminf(B, T), __int_as_float((int)bnext));
  }
  cnt = warp_compact(list, cnt, a.k);
  if (cnt == a.k && lane == 0) atomicMin(a.bound, (uint32_t)(list[a.k - 1] >> 32));
  // the block's warp lists (each at most k entries) become one: the
  // entries are packed to the front (read to registers, a barrier, written
  // at the warp's offset), the next power of two of them sorted, the first
  // k distinct distances kept; the merge then reads one part per block
  __shared__ int s_cnt[W];
  if (lane == 0) s_cnt[wib] = cnt;
  constexpr int kPer = kWarpListCap / 32;  // entries per lane of a full list
  unsigned long long mine[kPer];
#pragma unroll
  for (int r = 0; r < kPer; ++r) mine[r] = list[lane + 32 * r];
  __syncthreads();
  int offset = 0, packed = 0;
#pragma unroll
  for (int w = 0; w < W; ++w) {
    offset += w < wib ? s_cnt[w] : 0;
    packed += s_cnt[w];
  }
  int nsort = 32;
  while (nsort < packed) nsort <<= 1;
  unsigned long long* flat = &lists[0][0];
  __syncthreads();
#pragma unroll
  for (int r = 0; r < kPer; ++r)
    if (lane + 32 * r < cnt) flat[offset + lane + 32 * r] = mine[r];
  for (int i = packed + (int)threadIdx.x; i < nsort; i += kEdThreads) flat[i] = ~0ull;
  __syncthreads();
  for (int size = 2; size <= nsort; size <<= 1)
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      for (int i = threadIdx.x; i < nsort / 2; i += kEdThreads) {
        const int pos = 2 * i - (i & (stride - 1));
        const int partner = pos + stride;
        const bool asc = (pos & size) == 0;
        const unsigned long long x = flat[pos], y = flat[partner];
        if ((x > y) == asc) {
          flat[pos] = y;
          flat[partner] = x;
        }
      }
      __syncthreads();
    }
  if (wib == 0) {
    const int bc = warp_dedup_sorted(flat, packed, a.k, 0);
    unsigned long long* out = a.parts + (uint64_t)blockIdx.x * kWarpListCap;
    for (int i = lane; i < bc; i += 32) out[i] = flat[i];
    if (lane == 0) {
      a.part_count[blockIdx.x] = bc;
      if (bc == a.k) atomicMin(a.bound, (uint32_t)(flat[a.k - 1] >> 32));
    }
  }
  unsigned long long s_chunks = n_chunks, s_done = n_done, s_rows = n_rows;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    s_chunks += __shfl_xor_sync(HG_FULL, s_chunks, o);
    s_done += __shfl_xor_sync(HG_FULL, s_done, o);
    s_rows += __shfl_xor_sync(HG_FULL, s_rows, o);
  }
  if (lane == 0) {
    atomicAdd(&a.stats[1], s_chunks);
    atomicAdd(&a.stats[4], s_done);
    atomicAdd(&a.stats[5], s_rows);
  }
}

// Merges the per-block lists (and the current top-k, passed as part -1) into
// the k smallest distinct distances, lowest id per distance.  Only entries
// <= the final bound can belong to the answer.
constexpr int kMergeThreads = 1024;
__global__ void __launch_bounds__(kMergeThreads) k_merge(const unsigned long long* __restrict__ parts,
                                                         const int* __restrict__ part_count, int nparts, int k,
                                                         unsigned long long* topk, int* topk_count,
                                                         uint32_t* bound, int* err) {
  extern __shared__ unsigned long long buf[];  // kMergeCap
  __shared__ unsigned long long best[kMaxK];
  __shared__ uint32_t tmp[kMergeThreads / 32 + 1];
  __shared__ uint32_t total;
  __shared__ int nbest;
  const int t = threadIdx.x;
  const uint32_t B = ld_volatile(bound);
  // previous top-k
  if (t == 0) nbest = *topk_count;
  __syncthreads();
  for (int i = t; i < kMaxK; i += kMergeThreads) best[i] = (i < nbest) ? topk[i] : ~0ull;
  __syncthreads();
  // count entries <= B per part (lists are sorted ascending)
  const int per = (nparts + kMergeThreads - 1) / kMergeThreads;
  const int p0 = min(nparts, t * per), p1 = min(nparts, p0 + per);
  uint32_t mine = 0;
  for (int p = p0; p < p1; ++p) {
    const unsigned long long* l = parts + (uint64_t)p * kWarpListCap;
    int lo = 0, hi = part_count[p];
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if ((uint32_t)(l[mid] >> 32) <= B) lo = mid + 1;
      else hi = mid;
    }
    mine += lo;
  }
  const uint32_t start = block_exclusive_scan<kMergeThreads>(mine, tmp, &total);
  const uint32_t M = total;
  const int room = kMergeCap - k;
  for (uint32_t r0 = 0; r0 < M || r0 == 0; r0 += room) {
    // this round takes global positions [r0, r0 + room) after the current best
    const uint32_t rem = M > r0 ? M - r0 : 0u;
    const uint32_t m = rem < (uint32_t)room ? rem : (uint32_t)room;
    int nsort = 32;
    while (nsort < k + (int)m) nsort <<= 1;
    for (int i = t; i < nsort; i += kMergeThreads) buf[i] = (i < k) ? best[i] : ~0ull;
    __syncthreads();
    uint32_t g = start;
    for (int p = p0; p < p1; ++p) {
      const unsigned long long* l = parts + (uint64_t)p * kWarpListCap;
      const int cntp = part_count[p];
      for (int j = 0; j < cntp; ++j) {
        const unsigned long long v = l[j];
        if ((uint32_t)(v >> 32) > B) break;
        if (g >= r0 && g < r0 + room) buf[k + (g - r0)] = v;
        ++g;
      }
    }
    __syncthreads();
    // bitonic sort of nsort keys
    for (int size = 2; size <= nsort; size <<= 1) {
      for (int stride = size >> 1; stride > 0; stride >>= 1) {
        for (int i = t; i < nsort / 2; i += kMergeThreads) {
          const int pos = 2 * i - (i & (stride - 1));
          const int partner = pos + stride;
          const bool asc = (pos & size) == 0;
          const unsigned long long x = buf[pos], y = buf[partner];
          if ((x > y) == asc) {
            buf[pos] = y;
            buf[partner] = x;
          }
        }
        __syncthreads();
      }
    }
    // dedup by distance, keep k (thread 0; at most kMergeCap steps, exits at k)
    if (t == 0) {
      int out = 0;
      uint32_t prev = 0;
      for (int i = 0; i < nsort && out < k; ++i) {
        const unsigned long long v = buf[i];
        if (v == ~0ull) break;
        const uint32_t d = (uint32_t)(v >> 32);
        if (out > 0 && d == prev) continue;
        best[out++] = v;
        prev = d;
      }
      for (int i = out; i < kMaxK; ++i) best[i] = ~0ull;
      nbest = out;
    }
    __syncthreads();
    if (M == 0) break;
  }
  for (int i = t; i < k; i += kMergeThreads) topk[i] = best[i];
  if (t == 0) {
    *topk_count = nbest;
    if (nbest == k) atomicMin(bound, (uint32_t)(best[k - 1] >> 32));
    (void)err;
  }
}

__global__ void k_emit(const unsigned long long* topk, const int* topk_count, int k, float* dist_out,
                       int64_t* id_out) {
  const int i = threadIdx.x + blockIdx.x * blockDim.x;
  if (i >= k) return;
  const int n = *topk_count;
  if (i < n) {
    const unsigned long long v = topk[i];
    if (dist_out) dist_out[i] = __uint_as_float((uint32_t)(v >> 32));
    if (id_out) id_out[i] = (int64_t)(uint32_t)v;
  } else {
    if (dist_out) dist_out[i] = __int_as_float(0x7f800000);
    if (id_out) id_out[i] = -1;
  }
}

// ---------------------------------------------------------------------------
// data generation
// ---------------------------------------------------------------------------

__global__ void k_generate_walks(uint64_t seed, uint64_t first, uint64_t n, int L, float* out, int unit) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  // each thread writes its own row; the L2 merges the partial sectors
  if (unit) gaussian_unit(seed, first + i, L, out + i * (uint64_t)L);
  else random_walk(seed, first + i, L, out + i * (uint64_t)L);
}

// data == nullptr: the base row is regenerated from data_seed into the
// query's own output row (the collection need not be resident), then the
// noise is added in place.
__global__ void k_generate_queries(uint64_t seed, const float* data, uint64_t n, int L, int nq,
                                   const double* sigma2, float* out, uint64_t* base_ids, int unit,
                                   uint64_t data_seed) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= nq) return;
  const uint64_t b = pick_row(seed, (uint64_t)j, n);
  if (base_ids) base_ids[j] = b;
  float* o = out + (uint64_t)j * L;
  const float* base = data + b * (uint64_t)L;
  if (!data) {
    if (unit) gaussian_unit(data_seed, b, L, o);
    else random_walk(data_seed, b, L, o);
    base = o;
  }
  noisy_query(seed, (uint64_t)j, base, L, sigma2[j], o, unit);
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------

static inline unsigned blocks_for(uint64_t n, int t) { return (unsigned)((n + t - 1) / t); }

int sm_count(int device) {
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  return sms;
}

cudaError_t launch_route_rows(const float* X, int L, const uint32_t* rows, uint64_t first, uint32_t count,
                              Tree t, int* leaf_out, cudaStream_t s) {
  if (!count) return cudaSuccess;
  k_route_rows<<<blocks_for(count, 128), 128, 0, s>>>(X, L, rows, first, count, t, leaf_out);
  return cudaGetLastError();
}

cudaError_t launch_sketch_members(const float* X, int L, const uint32_t* members, uint32_t count,
                                  const short* seg_from, const short* seg_to, int nsegs, int* keys_out,
                                  cudaStream_t s) {
  if (!count || !nsegs) return cudaSuccess;
  unsigned b = blocks_for(count, 256);
  if (b > 148 * 8) b = 148 * 8;
  k_sketch_members<<<b, 256, sizeof(int) * 4 * nsegs, s>>>(X, L, members, count, seg_from, seg_to, nsegs,
                                                           keys_out);
  return cudaGetLastError();
}

cudaError_t launch_route_flags(const float* X, int L, const uint32_t* members, uint32_t count, short from,
                               short to, int idx, float value, uint8_t* flags, cudaStream_t s) {
  if (!count) return cudaSuccess;
  k_route_flags<<<blocks_for(count, 256), 256, 0, s>>>(X, L, members, count, from, to, idx, value, flags);
  return cudaGetLastError();
}

cudaError_t launch_gather_rows(const float* X, int L, const uint32_t* perm, uint64_t n, float* rows,
                               cudaStream_t s) {
  const uint64_t threads = n * (L / 4);
  if (!threads) return cudaSuccess;
  k_gather_rows<<<blocks_for(threads, 256), 256, 0, s>>>(X, L, perm, n, rows);
  return cudaGetLastError();
}

cudaError_t launch_sax_rows(const float* rows, int L, uint64_t n, const float* bp, uint8_t* sax,
                            cudaStream_t s) {
  if (!n) return cudaSuccess;
  k_sax_rows<<<blocks_for(n, 128), 128, 0, s>>>(rows, L, n, bp, sax);
  return cudaGetLastError();
}

cudaError_t launch_query_prep(const float* q, int L, Tree t, const uint64_t* leaf_start,
                              const uint32_t* leaf_size, int* approx_leaf, float* paa, int* cand,
                              float* cand_lb, int* cand_count, uint32_t* unit_prefix, uint32_t* bound,
                              int* topk_count, uint32_t* counters, cudaStream_t s) {
  k_query_prep<<<1, 32, 0, s>>>(q, L, t, leaf_start, leaf_size, approx_leaf, paa, cand, cand_lb, cand_count,
                                unit_prefix, bound, topk_count, counters);
  return cudaGetLastError();
}

cudaError_t launch_route_queries(const float* Q, int nq, int L, Tree t, int* leaf_out, cudaStream_t s) {
  if (!nq) return cudaSuccess;
  k_route_queries<<<blocks_for((uint64_t)nq * 32, 128), 128, 0, s>>>(Q, nq, L, t, leaf_out);
  return cudaGetLastError();
}

cudaError_t launch_leaf_lb(const float* q, int L, int nleaves, const int* seg_off, const short* points,
                           const float* sk, float* lb_out, cudaStream_t s, const float* paa, const float* bp,
                           float* sax_tab) {
  if (!nleaves) return cudaSuccess;
  static SmemLimit attr;
  const cudaError_t ea = attr.ensure((const void*)k_leaf_lb, 65536);
  if (ea != cudaSuccess) return ea;
  unsigned grid = blocks_for((uint64_t)nleaves * 32, 256);
  if (sax_tab && grid < HG_PAA_SEGMENTS) grid = HG_PAA_SEGMENTS;  // 16 x 256 threads: one per table entry
  k_leaf_lb<<<grid, 256, sizeof(float) * L, s>>>(q, L, nleaves, seg_off, points, sk, lb_out, paa, bp, sax_tab);
  return cudaGetLastError();
}

cudaError_t launch_leaf_keep(const float* Q, int L, int nq, const short* useg_start, const short* useg_end, int nu,
                             float2* segstats, const int* seg_off, const short* points, const int* seg_uid,
                             const float* sk, const uint32_t* leaf_size, int nleaves, const float* bound,
                             uint32_t* leaf_cnt, uint32_t* leaf_q, uint32_t stride, cudaStream_t s) {
  if (nq <= 0 || nleaves <= 0) return cudaSuccess;
  static SmemLimit attr;
  const cudaError_t ea = attr.ensure((const void*)k_query_segstats, 65536);
  if (ea != cudaSuccess) return ea;
  k_query_segstats<<<nq, 256, sizeof(float) * L, s>>>(Q, L, nq, useg_start, useg_end, nu, segstats);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  return launch_leaf_keep_list(segstats, nu, L, nq, seg_off, points, seg_uid, sk, leaf_size, nleaves, bound,
                               leaf_cnt, leaf_q, stride, nullptr, nullptr, s);
}

cudaError_t launch_leaf_keep_list(const float2* segstats, int nu, int L, int nq, const int* seg_off,
                                  const short* points, const int* seg_uid, const float* sk, const uint32_t* leaf_size,
                                  int nleaves, const float* bound, uint32_t* leaf_cnt, uint32_t* leaf_q,
                                  uint32_t stride, const uint32_t* qlist, const uint32_t* nq_dev, cudaStream_t s) {
  if (nq <= 0 || nleaves <= 0) return cudaSuccess;
  // grid-stride over the (query, leaf) pairs: at most 64 blocks of 256 threads per SM
  int dev = 0;
  const cudaError_t ed = cudaGetDevice(&dev);
  if (ed != cudaSuccess) return ed;
  const uint64_t want = blocks_for((uint64_t)nq * nleaves, 256);
  const uint64_t cap = 64ull * (uint64_t)sm_count(dev);
  k_leaf_keep<<<(unsigned)(want < cap ? want : cap), 256, 0, s>>>(
      segstats, nu, L, nq, seg_off, points, seg_uid, sk, leaf_size, nleaves, bound, leaf_cnt, leaf_q, stride, qlist,
      nq_dev);
  return cudaGetLastError();
}

__global__ void k_leaf_gate(float lb, float eps1, const uint32_t* stale, int* flag, unsigned long long* scanned) {
  const float kth = __uint_as_float(*stale);
  const int pass = lb <= __fdiv_rn(kth, eps1) ? 1 : 0;
  *flag = pass;
  if (pass) ++*scanned;
}
__global__ void k_stale_copy(const int* flag, const uint32_t* bound, uint32_t* stale) {
  if (*flag) *stale = *bound;
}
cudaError_t launch_leaf_gate(float lb, float eps1, const uint32_t* stale, int* flag, unsigned long long* scanned,
                             cudaStream_t s) {
  k_leaf_gate<<<1, 1, 0, s>>>(lb, eps1, stale, flag, scanned);
  return cudaGetLastError();
}
cudaError_t launch_stale_copy(const int* flag, const uint32_t* bound, uint32_t* stale, cudaStream_t s) {
  k_stale_copy<<<1, 1, 0, s>>>(flag, bound, stale);
  return cudaGetLastError();
}

static size_t select_smem(bool global_keys) {
  return sizeof(uint32_t) * 16 * kSortThreads + (global_keys ? 0 : sizeof(uint32_t) * 4 * kMaxLeavesSort);
}

cudaError_t launch_select_sort(const float* lb, int nleaves, const uint32_t* bound, const int* approx_leaf,
                               const uint64_t* leaf_start, const uint32_t* leaf_size, int* cand,
                               float* cand_lb, int* cand_count, uint32_t* unit_prefix, cudaStream_t s,
                               uint32_t* gkeys) {
  const bool global_keys = nleaves > kMaxLeavesSort;
  if (global_keys && !gkeys) return cudaErrorInvalidValue;
  static SmemLimit attr;
  const cudaError_t ea = attr.ensure((const void*)k_select_sort, (int)select_smem(false));
  if (ea != cudaSuccess) return ea;
  k_select_sort<<<1, kSortThreads, select_smem(global_keys), s>>>(lb, nleaves, bound, approx_leaf, leaf_start,
                                                                  leaf_size, cand, cand_lb, cand_count, unit_prefix,
                                                                  global_keys ? gkeys : nullptr);
  return cudaGetLastError();
}

cudaError_t launch_pscan_prep(uint64_t nrows, int* cand_count, uint32_t* unit_prefix, uint32_t* bound,
                              int* topk_count, uint32_t* counters, cudaStream_t s) {
  k_pscan_prep<<<1, 32, 0, s>>>(nrows, cand_count, unit_prefix, bound, topk_count, counters);
  return cudaGetLastError();
}

cudaError_t launch_lbsax_filter(const FilterArgs& a, int blocks, cudaStream_t s) {
  static SmemLimit attr;
  const cudaError_t ea = attr.ensure((const void*)k_lbsax_filter, (int)lbsax_filter_smem());
  if (ea != cudaSuccess) return ea;
  k_lbsax_filter<<<blocks, kFilterThreads, lbsax_filter_smem(), s>>>(a);
  return cudaGetLastError();
}

template <bool kRowIds, int kLines, int kSlot>
static cudaError_t launch_ed(const EdArgs& a, int blocks, cudaStream_t s) {
  static SmemLimit attr;
  const cudaError_t ea = attr.ensure((const void*)k_ed_stream<kRowIds, kLines, kSlot>, (int)q4_bytes(16384));
  if (ea != cudaSuccess) return ea;
  k_ed_stream<kRowIds, kLines, kSlot><<<blocks, kEdThreads, q4_bytes(a.L), s>>>(a);
  return cudaGetLastError();
}
// long series (L >= 4096): few candidate rows per query, each long, so
// more lanes per row keep more of each row in flight
#ifndef HG_ED_LONG_LINES
#define HG_ED_LONG_LINES 2
#endif
#ifndef HG_ED_LONG_SLOT
#define HG_ED_LONG_SLOT 8
#endif
#ifndef HG_ED_SHORT_LINES
#define HG_ED_SHORT_LINES 2
#endif
cudaError_t launch_ed_stream(const EdArgs& a, int blocks, cudaStream_t s) {
  return a.L >= 4096 ? launch_ed<false, HG_ED_LONG_LINES, HG_ED_LONG_SLOT>(a, blocks, s)
                     : launch_ed<false, HG_ED_SHORT_LINES, 4>(a, blocks, s);
}
cudaError_t launch_ed_stream_row_ids(const EdArgs& a, int blocks, cudaStream_t s) {
  return a.L >= 4096 ? launch_ed<true, HG_ED_LONG_LINES, HG_ED_LONG_SLOT>(a, blocks, s)
                     : launch_ed<true, HG_ED_SHORT_LINES, 4>(a, blocks, s);
}
int ed_blocks_per_sm(int L) {
  // shared memory per block: the staged query + 8 per-warp lists of 2 KB
  const size_t per_block = q4_bytes(L) + (size_t)kEdWarps * kWarpListCap * 8 + 1024;
  const int fit = (int)((size_t)227 * 1024 / per_block);
  // registers: more than two lines per step leave room for 3 blocks
  const int lines = L >= 4096 ? HG_ED_LONG_LINES : HG_ED_SHORT_LINES;
  const int cap = lines > 2 ? 3 : kEdBlocksPerSm;
  return fit < 1 ? 1 : (fit < cap ? fit : cap);
}

cudaError_t launch_merge(const unsigned long long* parts, const int* part_count, int nparts, int k,
                         unsigned long long* topk, int* topk_count, uint32_t* bound, int* err,
                         cudaStream_t s) {
  const int smem = sizeof(unsigned long long) * kMergeCap;
  static SmemLimit attr;
  const cudaError_t ea = attr.ensure((const void*)k_merge, smem);
  if (ea != cudaSuccess) return ea;
  k_merge<<<1, kMergeThreads, smem, s>>>(parts, part_count, nparts, k, topk, topk_count, bound, err);
  return cudaGetLastError();
}

cudaError_t launch_emit(const unsigned long long* topk, const int* topk_count, int k, float* dist_out,
                        int64_t* id_out, cudaStream_t s) {
  k_emit<<<blocks_for(k, 128), 128, 0, s>>>(topk, topk_count, k, dist_out, id_out);
  return cudaGetLastError();
}

cudaError_t launch_generate_walks(uint64_t seed, uint64_t first, uint64_t n, int L, float* out,
                                  cudaStream_t s, int unit) {
  if (!n) return cudaSuccess;
  k_generate_walks<<<blocks_for(n, 128), 128, 0, s>>>(seed, first, n, L, out, unit);
  return cudaGetLastError();
}

cudaError_t launch_generate_queries(uint64_t seed, const float* data, uint64_t n, int L, int nq,
                                    const double* sigma2, float* out, uint64_t* base_ids, cudaStream_t s, int unit,
                                    uint64_t data_seed) {
  if (!nq) return cudaSuccess;
  k_generate_queries<<<blocks_for(nq, 64), 64, 0, s>>>(seed, data, n, L, nq, sigma2, out, base_ids, unit,
                                                       data_seed);
  return cudaGetLastError();
}

}  // namespace hg
