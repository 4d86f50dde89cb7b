// hg_batch.cu -- batched exact k-NN: a BF16 tensor-core filter with a
// certified error bound, then an exact FP32 re-rank in the reference's
// summation order (ts_euclidean_distance_SIMD, ts.c:83-109).
//
// For thousands of queries at once the dot products q.x of every (query,
// row) pair are cheap on the tensor cores.  With q~, x~ the BF16 roundings of
// q and x, r_q = q - q~, r_x = x - x~ and FP32 accumulation,
//     d~(q, x) = |q|^2 + |x|^2 - 2 acc(q~ . x~)
// and q.x - q~.x~ = q~.r_x + r_q.x~ + r_q.r_x, so by Cauchy-Schwarz
//     |d~ - D| <= 2 (|q~| |r_x| + |r_q| |x~| + |r_q| |r_x|) + 2 L 2^-20 |q~| |x~|
// (the last term covers the tensor cores' FP32 accumulation), and D differs
// from the reference's FP32 sum by (L/8 + 4) 2^-24 D at most.  Per 128-row
// tile the row terms are replaced by their maxima:
//     err(q, tile) = 2 (1 + 2^-20) (|q~| R + r |X~| + r R + L 2^-20 |q~| X~)
//                    + c_sq (|q|^2 + max |x|^2 + B) + 1e-5,   c_sq = (L/8 + 16) 2^-22
// with |x|^2 and |q|^2 computed in FP64 and rounded up.  The pipeline:
//   1. route every query to its approximate leaf (approximate_knn_search's
//      traversal, hercules_query_engine.c:176-222);
//   2. bound: the tensor cores give the minimum d~ of every group of 8..128
//      rows of the approximate leaf; the k smallest groups' rows are ranked
//      exactly and their k-th distinct distance is B_q, an exact upper bound
//      of the query's k-th neighbour distance;
//   3. filter: every row against every query; (q, x) is kept when
//      d~ - err <= B_q, which holds for every row whose exact distance is <= B_q;
//   4. re-rank the kept rows exactly (early abandon at the running k-th
//      distance), merged with step 2's rows: k distinct distances, lowest id
//      per distance (queue_bounded_sorted_insert, hercules_query_engine.c:4034);
//   5. verify per query: B_q finite, k distances found, no bucket overflow;
//      a query that fails goes through the plain path.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "hg_arith.cuh"
#include "hg_batch.h"
#include "hg_device.cuh"

namespace hg {

constexpr int kBM = kBatchTileRows;

// ---------------------------------------------------------------------------
// preparation
// ---------------------------------------------------------------------------

// One warp per output row w: the BF16 copy of source row src = idx ? idx[w] : w
// (round to nearest) and, in FP64 rounded up, meta[src] = {|x|^2, |x~|,
// |x - x~|, 0} (x~ the BF16 row).
__global__ void k_rows_to_bf16(const float* __restrict__ rows, const uint32_t* __restrict__ idx, uint64_t n,
                               const uint32_t* n_dev, int L, __nv_bfloat16* __restrict__ out,
                               float4* __restrict__ meta) {
  const int lane = threadIdx.x & 31;
  if (n_dev) n = min(n, (uint64_t)*n_dev);  // at most the n the launch was sized for
  const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t w = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < n; w += nw) {
  const uint64_t src = idx ? idx[w] : w;
  const float4* x = reinterpret_cast<const float4*>(rows + src * L);
  __nv_bfloat162* o = reinterpret_cast<__nv_bfloat162*>(out + w * L);
  double a2 = 0.0, t2 = 0.0, r2 = 0.0;
  auto acc = [&](float v, float t) {
    const double dv = v, dt = t, dr = dv - dt;  // exact: both are floats
    a2 += dv * dv;
    t2 += dt * dt;
    r2 += dr * dr;
  };
  for (int i = lane; i < (L >> 2); i += 32) {
    const float4 v = x[i];
    const __nv_bfloat162 b0 = __floats2bfloat162_rn(v.x, v.y), b1 = __floats2bfloat162_rn(v.z, v.w);
    o[2 * i] = b0;
    o[2 * i + 1] = b1;
    const float2 f0 = __bfloat1622float2(b0), f1 = __bfloat1622float2(b1);
    acc(v.x, f0.x);
    acc(v.y, f0.y);
    acc(v.z, f1.x);
    acc(v.w, f1.y);
  }
#pragma unroll
  for (int s = 16; s > 0; s >>= 1) {
    a2 += __shfl_xor_sync(HG_FULL, a2, s);
    t2 += __shfl_xor_sync(HG_FULL, t2, s);
    r2 += __shfl_xor_sync(HG_FULL, r2, s);
  }
  if (lane == 0) {
    // FP64 sums of L non-negative terms: relative error below L 2^-53
    const double up = 1.0 + 1e-12;
    meta[src] = make_float4(__double2float_ru(a2 * up), __double2float_ru(sqrt(t2) * up),
                          __double2float_ru(sqrt(r2) * up), 0.0f);
  }
  }
}

// Per 128-row tile of the leaf-ordered rows: the maximum of each meta field.
__global__ void k_tile_norms(const float4* __restrict__ meta, uint64_t n, float4* __restrict__ tile_meta) {
  const uint64_t t = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  const uint64_t r0 = t * kBM;
  if (r0 >= n) return;
  float4 m = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  for (uint64_t r = r0 + lane; r < r0 + kBM && r < n; r += 32) {
    const float4 v = meta[r];
    m.x = fmaxf(m.x, v.x);
    m.y = fmaxf(m.y, v.y);
    m.z = fmaxf(m.z, v.z);
  }
#pragma unroll
  for (int s = 16; s > 0; s >>= 1) {
    m.x = fmaxf(m.x, __shfl_xor_sync(HG_FULL, m.x, s));
    m.y = fmaxf(m.y, __shfl_xor_sync(HG_FULL, m.y, s));
    m.z = fmaxf(m.z, __shfl_xor_sync(HG_FULL, m.z, s));
  }
  if (lane == 0) tile_meta[t] = m;
}

// ---------------------------------------------------------------------------
// bound, re-rank, verification
// ---------------------------------------------------------------------------

// Step 2: one block per query.  The slots' minima are distinct rows; the
// kMaxK smallest are ranked exactly (hg_ed, reference order) and the k-th
// distinct distance among them bounds the query's k-th neighbour distance
// (more rows than k: a tighter bound, and k distinct distances despite ties).
// squared distance of chunk c of x (8 floats) to the same chunk of q
__device__ __forceinline__ float chunk_d2_v4(const float* q, const float* x, int c) {
  const float4 x0 = reinterpret_cast<const float4*>(x)[2 * c], x1 = reinterpret_cast<const float4*>(x)[2 * c + 1];
  const float4 q0 = reinterpret_cast<const float4*>(q)[2 * c], q1 = reinterpret_cast<const float4*>(q)[2 * c + 1];
  const float qq[8] = {q0.x, q0.y, q0.z, q0.w, q1.x, q1.y, q1.z, q1.w};
  const float xx[8] = {x0.x, x0.y, x0.z, x0.w, x1.x, x1.y, x1.z, x1.w};
  return hg_chunk_d2(qq, xx);
}

constexpr int kSelThreads = 256;
__global__ void __launch_bounds__(kSelThreads) k_bound_select(BatchRank a) {
  extern __shared__ unsigned long long ssel[];
  unsigned long long* buf = ssel;                    // bm_pow2 keys
  __shared__ unsigned long long list[kWarpListCap];  // exact (distance, id) keys
  const int tid = threadIdx.x;
  const int q = blockIdx.x;
  const int k = (int)a.kq[q];
  const uint32_t ns = min(a.slots_of_query[q], a.bm_cap);
  int n = 32;
  while (n < (int)ns) n <<= 1;
  for (int i = tid; i < n; i += kSelThreads) buf[i] = i < (int)ns ? a.bm[(uint64_t)q * a.bm_cap + i] : ~0ull;
  __syncthreads();
  for (int size = 2; size <= n; size <<= 1)
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      for (int i = tid; i < (n >> 1); i += kSelThreads) {
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
  const float* qv = a.Q + (uint64_t)q * a.L;
  // a warp per row: lane c computes chunk c of a 32-chunk group (one
  // coalesced load), the chunk sums are added in chunk order
  // (ts_euclidean_distance_SIMD's order, no abandon)
  const int lane = tid & 31, nch = a.L >> 3;
  // the 2k + 32 best slots by d~ (at most kMaxK) are ranked exactly: the k-th
  // distinct exact distance among them bounds the query's k-th neighbour
  const int nrank = min(kMaxK, 2 * k + 32);
  for (int i = tid >> 5; i < kWarpListCap; i += kSelThreads / 32) {
    unsigned long long v = ~0ull;
    if (i < nrank && i < n && buf[i] != ~0ull) {  // uniform over the warp
      const uint32_t row = (uint32_t)buf[i];
      const float* xr = a.rows + (uint64_t)row * a.L;
      float d = 0.0f;
      for (int c0 = 0; c0 < nch; c0 += 32) {
        const float cd = c0 + lane < nch ? chunk_d2_v4(qv, xr, c0 + lane) : 0.0f;
        const int lim = min(32, nch - c0);
        for (int t = 0; t < lim; ++t) d = __fadd_rn(d, __shfl_sync(HG_FULL, cd, t));
      }
      v = ((unsigned long long)__float_as_uint(d) << 32) | (uint32_t)a.ids[row];
    }
    if (lane == 0) list[i] = v;
  }
  __syncthreads();
  if (tid < 32) {
    // the valid keys are a prefix (rows of the sorted prefix), the rest ~0
    int take = 0;
    for (int i = tid; i < kWarpListCap; i += 32) take += list[i] != ~0ull;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) take += __shfl_xor_sync(HG_FULL, take, o);
    const int cnt = warp_compact(list, take, k);
    if (tid == 0) {
      a.bound[q] = cnt == k ? __uint_as_float((uint32_t)(list[k - 1] >> 32)) : __int_as_float(0x7f800000);
      a.init_cnt[q] = cnt;
    }
    for (int i = tid; i < cnt; i += 32) a.init[(uint64_t)q * kMaxK + i] = list[i];
  }
}

// Steps 4-5 run in three kernels over the queries qlist[0 .. nlist) (all
// queries when qlist is null).  Plan: each query's surviving rows (the first
// bucket_cap of them when its bucket overflowed) are cut into at most
// kBatchMaxSeg segments of at least kBatchSegMin rows; segments are numbered
// over the list (exclusive prefix seg_prefix, by list position).
__global__ void __launch_bounds__(1024) k_rerank_plan(BatchRank a) {
  __shared__ uint32_t warp_sums[32];
  __shared__ uint32_t carry;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  if (tid == 0) carry = 0;
  __syncthreads();
  const float inf = __int_as_float(0x7f800000);
  const int nlist = a.nlist_dev ? (int)*a.nlist_dev : a.nlist;
  for (int base = 0; base < nlist; base += 1024) {
    const int i = base + tid;
    uint32_t nseg = 0, seg = 0;
    if (i < nlist) {
      const int q = a.qlist ? (int)a.qlist[i] : i;
      const uint32_t n = a.bound[q] < inf ? min(a.bucket_cnt[q], a.bucket_cap) : 0u;
      seg = max((uint32_t)kBatchSegMin, (n + kBatchMaxSeg - 1) / kBatchMaxSeg);
      nseg = (n + seg - 1) / seg;
      a.seg_rows[i] = seg;
      a.qbound[q] = __float_as_uint(a.bound[q]);
    }
    // block-wide exclusive scan of nseg
    uint32_t v = nseg;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t t = __shfl_up_sync(HG_FULL, v, o);
      if (lane >= o) v += t;
    }
    if (lane == 31) warp_sums[wid] = v;
    __syncthreads();
    if (wid == 0) {
      uint32_t w = warp_sums[lane];
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(HG_FULL, w, o);
        if (lane >= o) w += t;
      }
      warp_sums[lane] = w;
    }
    __syncthreads();
    const uint32_t excl = carry + (wid ? warp_sums[wid - 1] : 0u) + v - nseg;
    if (i < nlist) a.seg_prefix[i] = excl;
    __syncthreads();
    if (tid == 1023) carry = excl + nseg;
    __syncthreads();
  }
  if (tid == 0) {
    a.seg_prefix[nlist] = carry;
    a.heads[0] = 0;  // work counter of k_rerank_part
  }
}

// Squared distance of the 8-float chunk c of q and x (ts.c:83-109 order),
// both read as two float4.

// Segment re-rank: persistent warps take segments from a counter.  A warp
// starts from step 2's list, shares the query's running k-th distance through
// qbound (float bits, atomicMin) and writes its compacted list as one part.
// Within the warp, 32 / kSlot slots of kSlot lanes: lane j of a slot computes
// chunks ch + kSlot l + j (l < kLines) and every lane of the slot adds the
// step's kSlot * kLines chunk sums in order (ts_euclidean_distance_SIMD's
// order); one abandon test per step, as the step's lines are loaded already.
// Short series use 2-lane slots of four chunks per lane (16 rows per warp,
// 256 bytes of each per step: rows in flight matter more than lanes per row);
// long ones 8-lane slots of two (4 rows, 512 bytes).
constexpr int kRankWarps = 8;
template <int kSlot>
__host__ __device__ constexpr uint32_t rank_leaders() {
  return kSlot == 2 ? 0x55555555u : (kSlot == 4 ? 0x11111111u : (kSlot == 8 ? 0x01010101u : 0x00010001u));
}
template <int kSlot, int kLines>
__global__ void __launch_bounds__(kRankWarps * 32) k_rerank_part(BatchRank a) {
  __shared__ unsigned long long lists[kRankWarps][kWarpListCap];
  constexpr int kStep = kSlot * kLines;
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int slot_lead = lane & ~(kSlot - 1), j = lane & (kSlot - 1);
  unsigned long long* list = lists[wib];
  const float inf = __int_as_float(0x7f800000);
  const int nlist = a.nlist_dev ? (int)*a.nlist_dev : a.nlist;
  const uint32_t total_items = a.seg_prefix[nlist];
  const int nch = a.L >> 3;
  const uint32_t leaders = rank_leaders<kSlot>();
  unsigned long long n_rows = 0, n_chunks = 0;
  for (;;) {
    uint32_t item = 0;
    if (lane == 0) item = atomicAdd(&a.heads[0], 1u);
    item = __shfl_sync(HG_FULL, item, 0);
    if (item >= total_items) break;
    // list position of the item: the last i with seg_prefix[i] <= item
    int lo = 0, hi = nlist - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (a.seg_prefix[mid] <= item) lo = mid;
      else hi = mid - 1;
    }
    const int q = a.qlist ? (int)a.qlist[lo] : lo;
    const uint32_t seg = item - a.seg_prefix[lo];
    const uint32_t per = a.seg_rows[lo];
    const uint32_t first = seg * per;
    const uint32_t last = min(min(a.bucket_cnt[q], a.bucket_cap), first + per);  // an overflowed bucket holds bucket_cap rows
    const int k = (int)a.kq[q];
    const int c0 = a.init_cnt[q];
    for (int i = lane; i < kWarpListCap; i += 32) list[i] = i < c0 ? a.init[(uint64_t)q * kMaxK + i] : ~0ull;
    __syncwarp();
    int cnt = c0;
    float T = cnt == k ? __uint_as_float((uint32_t)(list[k - 1] >> 32)) : inf;
    float B = fminf(T, __uint_as_float(ld_volatile(&a.qbound[q])));
    const uint32_t* bk = a.bucket + (uint64_t)q * a.bucket_cap;
    const float* qv = a.Q + (uint64_t)q * a.L;
    uint32_t next = first;
    bool valid = false;
    uint32_t row = 0;
    int ch = 0;
    float dist = 0.0f;
    const float4* x = nullptr;
    const float4* qc = reinterpret_cast<const float4*>(qv) + 2 * j;
    for (;;) {
      const uint32_t need = __ballot_sync(HG_FULL, !valid) & leaders;
      if (need && next < last) {
        const int r = __popc(need & ((1u << slot_lead) - 1));
        const uint32_t avail = min(last - next, (uint32_t)(32 / kSlot));
        if (((need >> slot_lead) & 1u) && (uint32_t)r < avail) {
          row = bk[next + r];
          valid = true;
          dist = 0.0f;
          ch = 0;
          x = reinterpret_cast<const float4*>(a.rows + (uint64_t)row * a.L) + 2 * j;
          if (j == 0) ++n_rows;
        }
        next += min((uint32_t)__popc(need), avail);
        // the other warps of this query may have lowered its k-th distance
        B = fminf(B, __uint_as_float(ld_volatile(&a.qbound[q])));
      }
      if (!__any_sync(HG_FULL, valid)) break;
      // chunk ch + kSlot l + j of the row (0 past the row's end: adding it
      // leaves a sum unchanged)
      float dl[kLines];
#pragma unroll
      for (int l = 0; l < kLines; ++l) {
        const bool in = valid && ch + kSlot * l + j < nch;
        float4 x0, x1, q0, q1;
        if (in) {
          x0 = x[2 * kSlot * l];
          x1 = x[2 * kSlot * l + 1];
          q0 = qc[2 * ch + 2 * kSlot * l];
          q1 = qc[2 * ch + 2 * kSlot * l + 1];
        }
        const float qq[8] = {q0.x, q0.y, q0.z, q0.w, q1.x, q1.y, q1.z, q1.w};
        const float xx[8] = {x0.x, x0.y, x0.z, x0.w, x1.x, x1.y, x1.z, x1.w};
        const float d = hg_chunk_d2(qq, xx);
        dl[l] = in ? d : 0.0f;
      }
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
          // partial sums only grow: this row cannot enter; the reference
          // reads up to the first chunk whose sum exceeds the bound
          if (j == 0) {
            int used = 1;
#pragma unroll
            for (int t = 0; t < kStep; ++t) used += part[t] <= B ? 1 : 0;
            n_chunks += (unsigned long long)(ch + used);
          }
          valid = false;
        } else {
          dist = acc;
          ch += kStep;
          x += 2 * kStep;
          if (ch >= nch) {
            finished = true;
            valid = false;
            if (j == 0) n_chunks += (unsigned long long)nch;
          }
        }
      }
      const bool take = finished && j == 0;
      warp_list_add<true>(list, cnt, T, k, &a.qbound[q], take, dist, take ? (uint32_t)a.ids[row] : 0u);
      B = fminf(B, T);
    }
    cnt = warp_compact(list, cnt, k);
    unsigned long long* part = a.parts + (uint64_t)item * a.kmax;
    for (int i = lane; i < cnt; i += 32) part[i] = list[i];
    if (lane == 0) a.part_cnt[item] = cnt;
    __syncwarp();
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    n_rows += __shfl_xor_sync(HG_FULL, n_rows, o);
    n_chunks += __shfl_xor_sync(HG_FULL, n_chunks, o);
  }
  if (lane == 0 && n_rows) {
    atomicAdd(&a.stats[0], n_rows);
    atomicAdd(&a.stats[1], n_chunks);
  }
}

// Merge: one warp per query folds its starting list and its parts into the
// answer (k distinct distances, lowest id per distance) and verifies it:
//   ok 1: the filter kept every row within B_q and the k-th distance is <= B_q;
//   ok 0: the bucket overflowed but its first rows gave k distances below
//         B_q: B_q is lowered to the k-th, the list kept, the query retried;
//   ok -1: neither: the plain path answers it.
__global__ void __launch_bounds__(kRankWarps * 32) k_rerank_merge(BatchRank a) {
  __shared__ unsigned long long lists[kRankWarps][kWarpListCap];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int pos = blockIdx.x * kRankWarps + wib;
  if (pos >= (a.nlist_dev ? (int)*a.nlist_dev : a.nlist)) return;
  const int q = a.qlist ? (int)a.qlist[pos] : pos;
  unsigned long long* list = lists[wib];
  const int k = (int)a.kq[q];
  const float inf = __int_as_float(0x7f800000);
  const int c0 = a.init_cnt[q];
  for (int i = lane; i < kWarpListCap; i += 32) list[i] = i < c0 ? a.init[(uint64_t)q * kMaxK + i] : ~0ull;
  __syncwarp();
  int cnt = c0;
  float T = cnt == k ? __uint_as_float((uint32_t)(list[k - 1] >> 32)) : inf;
  // the segments shared the query's running k-th distance: no entry above
  // its final value can be among the k, and every part is sorted
  const float Tq = __uint_as_float(ld_volatile(&a.qbound[q]));
  const uint32_t p0 = a.seg_prefix[pos], p1 = a.seg_prefix[pos + 1];
  for (uint32_t p = p0; p < p1; ++p) {
    const int pc = max(0, min(a.part_cnt[p], a.kmax));
    const unsigned long long* part = a.parts + (uint64_t)p * a.kmax;
    for (int base = 0; base < pc; base += 32) {
      const unsigned long long v = base + lane < pc ? part[base + lane] : ~0ull;
      const float d = __uint_as_float((uint32_t)(v >> 32));
      const bool take = base + lane < pc && d <= Tq && d <= T;
      if (!__any_sync(HG_FULL, take)) break;  // sorted: nothing further qualifies
      warp_list_add<true>(list, cnt, T, k, nullptr, take, d, (uint32_t)v);
    }
  }
  cnt = warp_compact(list, cnt, k);
  const float Bq = a.bound[q];
  const uint32_t nb = a.bucket_cnt[q];
  const float dk = cnt == k ? __uint_as_float((uint32_t)(list[k - 1] >> 32)) : inf;
  const int ok = (Bq < inf && nb <= a.bucket_cap && dk <= Bq) ? 1 : ((Bq < inf && dk < Bq) ? 0 : -1);
  for (int i = lane; i < a.kmax; i += 32) {
    const bool have = i < cnt;
    a.dist_out[(uint64_t)q * a.kmax + i] = have ? __uint_as_float((uint32_t)(list[i] >> 32)) : inf;
    a.id_out[(uint64_t)q * a.kmax + i] = have ? (int64_t)(uint32_t)list[i] : -1;
  }
  if (ok == 0) {
    for (int i = lane; i < cnt; i += 32) a.init[(uint64_t)q * kMaxK + i] = list[i];
    if (lane == 0) {
      a.init_cnt[q] = cnt;
      a.bound[q] = dk;
    }
  }
  if (lane == 0) {
    a.ok_out[q] = ok;
    atomicAdd(&a.stats[2], (unsigned long long)nb);
  }
}

// Survivor pairs into their queries' buckets, 32 pairs per warp step: lanes
// holding the same query share one atomic (pairs of a query cluster, since
// the filter emits them tile by tile); empty slots (~0) are skipped.
__global__ void k_scatter_pairs(const unsigned long long* __restrict__ pairs, const uint32_t* pairs_cnt,
                                uint32_t pairs_cap, uint32_t* __restrict__ bucket, uint32_t* bucket_cnt,
                                uint32_t bucket_cap) {
  const uint32_t n = min(*pairs_cnt, pairs_cap);
  const int lane = threadIdx.x & 31;
  const uint32_t warps = gridDim.x * (blockDim.x >> 5);
  for (uint32_t base = (blockIdx.x * blockDim.x + threadIdx.x) & ~31u; base < n; base += warps * 32) {
    const uint32_t i = base + lane;
    const unsigned long long e = i < n ? pairs[i] : ~0ull;
    const bool valid = e != ~0ull;
    const uint32_t q = valid ? (uint32_t)(e >> 32) : 0xffffffffu;
    const uint32_t same = __match_any_sync(HG_FULL, q);
    const int leader = __ffs(same) - 1;
    uint32_t pos = 0;
    if (valid && lane == leader) pos = atomicAdd(&bucket_cnt[q], (uint32_t)__popc(same));
    pos = __shfl_sync(HG_FULL, pos, leader) + (uint32_t)__popc(same & ((1u << lane) - 1));
    if (valid && pos < bucket_cap) bucket[(uint64_t)q * bucket_cap + pos] = (uint32_t)e;
  }
}

// The pair list overflowed: every query of the round counts as overflowed.
__global__ void k_mark_overflow(const uint32_t* pairs_cnt, uint32_t pairs_cap, const uint32_t* qlist, int nlist,
                                const uint32_t* nlist_dev, uint32_t* bucket_cnt, uint32_t bucket_cap) {
  if (*pairs_cnt <= pairs_cap) return;
  if (nlist_dev) nlist = (int)*nlist_dev;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nlist; i += gridDim.x * blockDim.x) {
    const uint32_t q = qlist ? qlist[i] : (uint32_t)i;
    bucket_cnt[q] = max(bucket_cnt[q], bucket_cap + 1);
  }
}

// ---------------------------------------------------------------------------
// device-side control of a batch: grouping, retry lists, verification count
// ---------------------------------------------------------------------------

// Queries grouped by approximate leaf (one block): per leaf its query count
// and offset (counting sort; the order inside a leaf is arbitrary), each
// query's bound slots, and the bound pass's item offsets per leaf (groups of
// at most kBatchBoundQueries queries x chunks of btpi tiles).
constexpr int kGroupThreads = 1024;
__global__ void __launch_bounds__(kGroupThreads) k_group_queries(const int* __restrict__ approx, int nq,
                                                                 const LeafPlan* __restrict__ plan, int nleaves,
                                                                 uint32_t btpi, uint32_t* perm, uint32_t* slots,
                                                                 uint32_t* leaf_qoff, uint32_t* leaf_qcnt,
                                                                 uint32_t* item_off, uint32_t* nitems,
                                                                 uint32_t* gcnt) {
  // per-leaf counters in shared memory, or in gcnt (2 x nleaves words of
  // global memory) above kMaxLeavesSort leaves
  extern __shared__ uint32_t gsh[];
  uint32_t* cnt = gcnt ? gcnt : gsh;   // [nleaves]
  uint32_t* cur = cnt + nleaves;       // [nleaves]
  __shared__ uint32_t wsum[2][32];
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  for (int i = tid; i < nleaves; i += kGroupThreads) cnt[i] = cur[i] = 0;
  __syncthreads();
  for (int q = tid; q < nq; q += kGroupThreads) atomicAdd(&cnt[approx[q]], 1u);
  __syncthreads();
  // exclusive scans over the leaves of query counts and item counts; each
  // thread owns a run of consecutive leaves
  const int per = (nleaves + kGroupThreads - 1) / kGroupThreads;
  const int l0 = min(tid * per, nleaves), l1 = min(l0 + per, nleaves);
  auto items_of = [&](int l) -> uint32_t {
    const uint32_t c = cnt[l], use = plan[l].use_tiles;
    if (c == 0 || use == 0) return 0u;
    return ((c + kBatchBoundQueries - 1) / kBatchBoundQueries) * ((use + btpi - 1) / btpi);
  };
  uint32_t sq = 0, si = 0;
  for (int l = l0; l < l1; ++l) {
    sq += cnt[l];
    si += items_of(l);
  }
  uint32_t vq = sq, vi = si;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t x = __shfl_up_sync(HG_FULL, vq, o), y = __shfl_up_sync(HG_FULL, vi, o);
    if (lane >= o) {
      vq += x;
      vi += y;
    }
  }
  if (lane == 31) {
    wsum[0][wid] = vq;
    wsum[1][wid] = vi;
  }
  __syncthreads();
  if (wid == 0) {
    uint32_t x = wsum[0][lane], y = wsum[1][lane];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t x2 = __shfl_up_sync(HG_FULL, x, o), y2 = __shfl_up_sync(HG_FULL, y, o);
      if (lane >= o) {
        x += x2;
        y += y2;
      }
    }
    wsum[0][lane] = x;
    wsum[1][lane] = y;
  }
  __syncthreads();
  uint32_t oq = (wid ? wsum[0][wid - 1] : 0u) + vq - sq, oi = (wid ? wsum[1][wid - 1] : 0u) + vi - si;
  for (int l = l0; l < l1; ++l) {
    leaf_qoff[l] = oq;
    leaf_qcnt[l] = cnt[l];
    item_off[l] = oi;
    oq += cnt[l];
    oi += items_of(l);
  }
  if (tid == kGroupThreads - 1) *nitems = oi;
  __syncthreads();
  for (int q = tid; q < nq; q += kGroupThreads) {
    const int l = approx[q];
    const uint32_t pos = atomicAdd(&cur[l], 1u);
    perm[leaf_qoff[l] + pos] = (uint32_t)q;
    slots[q] = plan[l].use_tiles * plan[l].sub;
  }
}

// The bound pass's work items, one warp per leaf.
__global__ void k_group_items(const LeafPlan* __restrict__ plan, int nleaves, uint32_t btpi,
                              const uint32_t* __restrict__ leaf_qoff, const uint32_t* __restrict__ leaf_qcnt,
                              const uint32_t* __restrict__ item_off, BatchItem* items) {
  const int l = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
  if (l >= nleaves) return;
  const LeafPlan p = plan[l];
  const uint32_t c = leaf_qcnt[l], use = p.use_tiles;
  if (c == 0 || use == 0) return;
  const uint32_t per_group = (use + btpi - 1) / btpi;
  const uint32_t n = ((c + kBatchBoundQueries - 1) / kBatchBoundQueries) * per_group;
  for (uint32_t i = lane; i < n; i += 32) {
    const uint32_t g = i / per_group, tb = i % per_group;
    BatchItem it;
    it.row_begin = p.start;
    it.row_end = p.start + p.size;
    it.q_off = leaf_qoff[l] + g * kBatchBoundQueries;
    it.q_cnt = min((uint32_t)kBatchBoundQueries, c - g * kBatchBoundQueries);
    it.tile_lo = tb * btpi;
    it.tile_hi = min(use, tb * btpi + btpi);
    it.sub = p.sub;
    it.row_skip = 0;
    items[item_off[l] + i] = it;
  }
}

// The pruned filter's layout (one block): per leaf, its kept queries get a
// run of the query panel (exclusive scan of the counts) and its work items
// a run of the item list (query tiles of kBatchQueryTile x chunks of tpi
// 128-row tiles on the global tile grid).  ctl[0] = items, ctl[1] = panel
// rows, ctl[2] = the dense pass's query count: 0, or nq when the panel or
// the item list would overflow (the dense pass then filters every row),
// ctl[3] = the kept (leaf, query) pairs.
// pairs = sum over leaves of kept queries x leaf rows.
__global__ void __launch_bounds__(kGroupThreads) k_group_pruned(const uint32_t* __restrict__ leaf_cnt,
                                                                const LeafPlan* __restrict__ plan, int nleaves,
                                                                uint32_t tpi, uint32_t panel_cap, uint32_t items_cap,
                                                                uint32_t nq, const uint32_t* nq_dev,
                                                                uint32_t* leaf_poff, uint32_t* leaf_ioff,
                                                                uint32_t* ctl, unsigned long long* pairs) {
  __shared__ unsigned long long wsum[3][32];
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  auto items_of = [&](int l) -> unsigned long long {
    const uint32_t c = leaf_cnt[l];
    if (c == 0 || plan[l].size == 0) return 0ull;
    const uint64_t t0 = plan[l].start / kBM, t1 = (plan[l].start + plan[l].size + kBM - 1) / kBM;
    return (unsigned long long)((c + kBatchQueryTile - 1) / kBatchQueryTile) * ((t1 - t0 + tpi - 1) / tpi);
  };
  const int per = (nleaves + kGroupThreads - 1) / kGroupThreads;
  const int l0 = min(tid * per, nleaves), l1 = min(l0 + per, nleaves);
  unsigned long long sq = 0, si = 0, sp = 0;
  for (int l = l0; l < l1; ++l) {
    sq += leaf_cnt[l];
    si += items_of(l);
    sp += (unsigned long long)leaf_cnt[l] * plan[l].size;
  }
  unsigned long long v[3] = {sq, si, sp};
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      const unsigned long long x = __shfl_up_sync(HG_FULL, v[i], o);
      if (lane >= o) v[i] += x;
    }
  }
  if (lane == 31)
    for (int i = 0; i < 3; ++i) wsum[i][wid] = v[i];
  __syncthreads();
  if (wid == 0) {
    unsigned long long x[3] = {wsum[0][lane], wsum[1][lane], wsum[2][lane]};
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        const unsigned long long y = __shfl_up_sync(HG_FULL, x[i], o);
        if (lane >= o) x[i] += y;
      }
    }
    for (int i = 0; i < 3; ++i) wsum[i][lane] = x[i];
  }
  __syncthreads();
  unsigned long long oq = (wid ? wsum[0][wid - 1] : 0ull) + v[0] - sq;
  unsigned long long oi = (wid ? wsum[1][wid - 1] : 0ull) + v[1] - si;
  for (int l = l0; l < l1; ++l) {
    leaf_poff[l] = (uint32_t)oq;
    leaf_ioff[l] = (uint32_t)oi;
    oq += leaf_cnt[l];
    oi += items_of(l);
  }
  if (tid == kGroupThreads - 1) {
    const unsigned long long tq = wsum[0][31], ti = wsum[1][31], tp = wsum[2][31];
    const bool fits = tq <= panel_cap && ti <= items_cap;
    ctl[0] = fits ? (uint32_t)ti : 0u;
    ctl[1] = fits ? (uint32_t)tq : 0u;
    ctl[2] = fits ? 0u : (nq_dev ? *nq_dev : nq);
    ctl[3] = (uint32_t)tq;  // kept (leaf, query) pairs
    *pairs = fits ? tp : 0ull;
  }
}

// The pruned filter's panel list and work items, one block per leaf.
__global__ void k_emit_pruned(const uint32_t* __restrict__ leaf_cnt, const uint32_t* __restrict__ leaf_q,
                              uint32_t stride, const uint32_t* __restrict__ leaf_poff,
                              const uint32_t* __restrict__ leaf_ioff, const LeafPlan* __restrict__ plan, uint32_t tpi,
                              const uint32_t* __restrict__ ctl, uint32_t* panel_list, BatchItem* items) {
  const int l = blockIdx.x;
  const uint32_t c = leaf_cnt[l];
  if (ctl[0] == 0 || c == 0 || plan[l].size == 0) return;
  const uint32_t po = leaf_poff[l], io = leaf_ioff[l];
  for (uint32_t i = threadIdx.x; i < c; i += blockDim.x) panel_list[po + i] = leaf_q[(uint64_t)l * stride + i];
  const uint64_t start = plan[l].start, end = start + plan[l].size;
  const uint64_t t0 = start / kBM, t1 = (end + kBM - 1) / kBM;
  const uint32_t ntile = (uint32_t)(t1 - t0), nch = (ntile + tpi - 1) / tpi;
  const uint32_t nqt = (c + kBatchQueryTile - 1) / kBatchQueryTile;
  for (uint32_t i = threadIdx.x; i < nch * nqt; i += blockDim.x) {
    const uint32_t ch = i / nqt, qt = i % nqt;
    BatchItem it;
    it.row_begin = t0 * kBM;
    it.row_end = end;
    it.q_off = po + qt * kBatchQueryTile;
    it.q_cnt = min((uint32_t)kBatchQueryTile, c - qt * kBatchQueryTile);
    it.tile_lo = ch * tpi;
    it.tile_hi = min(ntile, ch * tpi + tpi);
    it.sub = 1;
    it.row_skip = (uint32_t)(start - t0 * kBM);
    items[io + i] = it;
  }
}

// Queries of a round (list, or 0 .. n) still to retry (ok == 0) go to out.
__global__ void k_collect_retry(const int* __restrict__ ok, const uint32_t* list, uint32_t n, const uint32_t* n_dev,
                                uint32_t* out, uint32_t* out_n) {
  if (n_dev) n = *n_dev;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint32_t q = list ? list[i] : i;
    if (ok[q] == 0) out[atomicAdd(out_n, 1u)] = q;
  }
}

// Phase boundary of a batch: the global timer (ns) into a slot.
__global__ void k_stamp(unsigned long long* slot) {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  *slot = t;
}

// Queries the batch did not verify (ok != 1): the plain path answers them.
__global__ void k_count_unverified(const int* __restrict__ ok, uint32_t nq, uint32_t* out) {
  uint32_t c = 0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nq; i += gridDim.x * blockDim.x) c += ok[i] != 1;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(HG_FULL, c, o);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(out, c);
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------

static inline unsigned nblk(uint64_t n, int t) { return (unsigned)((n + t - 1) / t); }

cudaError_t launch_rows_to_bf16(const float* rows, const uint32_t* idx, uint64_t n, int L, void* out, float4* meta,
                                cudaStream_t s, const uint32_t* n_dev) {
  if (!n) return cudaSuccess;
  // a warp per row, grid-stride: a count read on the device (often far below
  // n) costs no launch of n warps
  uint64_t blocks = nblk(n * 32, 256);
  if (n_dev) {
    int dev = 0;
    const cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    const uint64_t cap = 32ull * (uint64_t)sm_count(dev);
    if (blocks > cap) blocks = cap;
  }
  k_rows_to_bf16<<<(unsigned)blocks, 256, 0, s>>>(rows, idx, n, n_dev, L, static_cast<__nv_bfloat16*>(out), meta);
  return cudaGetLastError();
}

cudaError_t launch_tile_norms(const float4* meta, uint64_t n, float4* tile_meta, cudaStream_t s) {
  const uint64_t nt = (n + kBM - 1) / kBM;
  if (!nt) return cudaSuccess;
  k_tile_norms<<<nblk(nt * 32, 256), 256, 0, s>>>(meta, n, tile_meta);
  return cudaGetLastError();
}

cudaError_t launch_scatter_pairs(const unsigned long long* pairs, const uint32_t* pairs_cnt, uint32_t pairs_cap,
                                 const uint32_t* qlist, int nlist, const uint32_t* nlist_dev, uint32_t* bucket,
                                 uint32_t* bucket_cnt, uint32_t bucket_cap, cudaStream_t s) {
  // grid-stride, enough threads in flight to hide the bucket atomics' latency
  k_scatter_pairs<<<2048, 256, 0, s>>>(pairs, pairs_cnt, pairs_cap, bucket, bucket_cnt, bucket_cap);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess || nlist == 0) return e;
  k_mark_overflow<<<nblk(nlist, 256), 256, 0, s>>>(pairs_cnt, pairs_cap, qlist, nlist, nlist_dev, bucket_cnt,
                                                   bucket_cap);
  return cudaGetLastError();
}

cudaError_t launch_group_queries(const int* approx, int nq, const LeafPlan* plan, int nleaves, uint32_t btpi,
                                 uint32_t* perm, uint32_t* slots, uint32_t* leaf_qoff, uint32_t* leaf_qcnt,
                                 uint32_t* item_off, uint32_t* nitems, BatchItem* items, cudaStream_t s,
                                 uint32_t* gcnt) {
  const bool global_cnt = nleaves > kMaxLeavesSort;
  if (global_cnt && !gcnt) return cudaErrorInvalidValue;
  const size_t smem = global_cnt ? 0 : sizeof(uint32_t) * 2 * (size_t)nleaves;
  static SmemLimit attr;
  const cudaError_t ea = attr.ensure((const void*)k_group_queries, (int)(sizeof(uint32_t) * 2 * kMaxLeavesSort));
  if (ea != cudaSuccess) return ea;
  k_group_queries<<<1, kGroupThreads, smem, s>>>(approx, nq, plan, nleaves, btpi, perm, slots, leaf_qoff, leaf_qcnt,
                                                 item_off, nitems, global_cnt ? gcnt : nullptr);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  k_group_items<<<nblk((uint64_t)nleaves * 32, 256), 256, 0, s>>>(plan, nleaves, btpi, leaf_qoff, leaf_qcnt,
                                                                 item_off, items);
  return cudaGetLastError();
}

cudaError_t launch_group_pruned(const uint32_t* leaf_cnt, const uint32_t* leaf_q, uint32_t stride,
                                const LeafPlan* plan, int nleaves, uint32_t tpi, uint32_t panel_cap,
                                uint32_t items_cap, uint32_t nq, uint32_t* leaf_poff, uint32_t* leaf_ioff,
                                uint32_t* ctl, unsigned long long* pairs, uint32_t* panel_list, BatchItem* items,
                                cudaStream_t s, const uint32_t* nq_dev) {
  k_group_pruned<<<1, kGroupThreads, 0, s>>>(leaf_cnt, plan, nleaves, tpi, panel_cap, items_cap, nq, nq_dev,
                                             leaf_poff, leaf_ioff, ctl, pairs);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess || nleaves == 0) return e;
  k_emit_pruned<<<nleaves, 256, 0, s>>>(leaf_cnt, leaf_q, stride, leaf_poff, leaf_ioff, plan, tpi, ctl, panel_list,
                                        items);
  return cudaGetLastError();
}

cudaError_t launch_collect_retry(const int* ok, const uint32_t* list, uint32_t n, const uint32_t* n_dev,
                                 uint32_t* out, uint32_t* out_n, cudaStream_t s) {
  if (!n) return cudaSuccess;
  const unsigned g = nblk(n, 256) < 1024 ? nblk(n, 256) : 1024;
  k_collect_retry<<<g, 256, 0, s>>>(ok, list, n, n_dev, out, out_n);
  return cudaGetLastError();
}

cudaError_t launch_stamp(unsigned long long* slot, cudaStream_t s) {
  k_stamp<<<1, 1, 0, s>>>(slot);
  return cudaGetLastError();
}

cudaError_t launch_count_unverified(const int* ok, uint32_t nq, uint32_t* out, cudaStream_t s) {
  if (!nq) return cudaSuccess;
  const unsigned g = nblk(nq, 256) < 1024 ? nblk(nq, 256) : 1024;
  k_count_unverified<<<g, 256, 0, s>>>(ok, nq, out);
  return cudaGetLastError();
}

cudaError_t launch_bound_select(const BatchRank& r, cudaStream_t s) {
  if (!r.nq) return cudaSuccess;
  int n = 32;
  while (n < (int)r.bm_cap) n <<= 1;
  static SmemLimit attr;
  const cudaError_t ea = attr.ensure((const void*)k_bound_select, (int)(sizeof(unsigned long long) * kBatchMaxSlots));
  if (ea != cudaSuccess) return ea;
  k_bound_select<<<r.nq, kSelThreads, sizeof(unsigned long long) * n, s>>>(r);
  return cudaGetLastError();
}

cudaError_t launch_rerank(const BatchRank& r, int part_blocks, cudaStream_t s) {
  if (!r.nlist) return cudaSuccess;
  k_rerank_plan<<<1, 1024, 0, s>>>(r);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  if (r.L >= 4096) k_rerank_part<8, 2><<<part_blocks, kRankWarps * 32, 0, s>>>(r);
  else k_rerank_part<2, 4><<<part_blocks, kRankWarps * 32, 0, s>>>(r);
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  k_rerank_merge<<<nblk(r.nlist, kRankWarps), kRankWarps * 32, 0, s>>>(r);
  return cudaGetLastError();
}

}  // namespace hg
