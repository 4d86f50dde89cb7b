// hg_device.cuh -- device helpers shared by the query kernels.
#pragma once

#include <stdint.h>

#include "hg_kernels.h"

namespace hg {

#define HG_FULL 0xffffffffu

__device__ __forceinline__ uint32_t ld_volatile(const uint32_t* p) {
  return *(const volatile uint32_t*)p;
}

// --- warp candidate list -----------------------------------------------------
// A warp keeps its candidates as 64-bit keys (distance bits << 32 | id) in a
// shared buffer of kWarpListCap entries.  Compaction sorts the buffer
// (bitonic), keeps the first entry of each distinct distance (the lowest id,
// the tie rule) and the k smallest distances.

static __device__ void warp_sort(unsigned long long* a, int n) {
  const int lane = threadIdx.x & 31;
  for (int size = 2; size <= n; size <<= 1) {
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      for (int i = lane; i < (n >> 1); i += 32) {
        const int pos = 2 * i - (i & (stride - 1));
        const int partner = pos + stride;
        const bool asc = (pos & size) == 0;
        const unsigned long long x = a[pos], y = a[partner];
        if ((x > y) == asc) {
          a[pos] = y;
          a[partner] = x;
        }
      }
      __syncwarp();
    }
  }
}

// list[0..cnt) sorted ascending by (distance, id): keeps the first entry of
// each distance, at most k, at the front; sets list[out..cap) to ~0ull;
// returns the count (warp-uniform).
static __device__ int warp_dedup_sorted(unsigned long long* list, int cnt, int k, int cap) {
  const int lane = threadIdx.x & 31;
  int out = 0;
  uint32_t prev_d = 0xffffffffu;
  bool have_prev = false;
  for (int base = 0; base < cnt && out < k; base += 32) {
    const int i = base + lane;
    const unsigned long long v = i < cnt ? list[i] : ~0ull;
    const uint32_t d = (uint32_t)(v >> 32);
    uint32_t dprev = __shfl_up_sync(HG_FULL, d, 1);
    if (lane == 0) dprev = have_prev ? prev_d : ~d;
    const bool keep = i < cnt && d != dprev;
    const uint32_t m = __ballot_sync(HG_FULL, keep);
    const int r = __popc(m & ((1u << lane) - 1));
    __syncwarp();
    if (keep && out + r < k) list[out + r] = v;
    prev_d = __shfl_sync(HG_FULL, d, 31);
    have_prev = true;
    out = min(k, out + __popc(m));
    __syncwarp();
  }
  for (int i = out + lane; i < cap; i += 32) list[i] = ~0ull;
  __syncwarp();
  return out;
}

// Sorts list[0..cnt), dedups by distance, keeps at most k; returns the new
// count (warp-uniform).  Entries beyond cnt must be ~0ull on entry.
static __device__ int warp_compact(unsigned long long* list, int cnt, int k) {
  int n = 32;
  while (n < cnt) n <<= 1;
  warp_sort(list, n);
  return warp_dedup_sorted(list, cnt, k, kWarpListCap);
}

// Appends (key, id) candidates of the lanes in `take` to the warp's list and
// compacts it once it holds k entries; returns the warp's k-th distance T
// (+inf until k distinct distances are held) and lowers the global bound.
// kLazy: compact only when the list may not hold another 32 entries (fewer
// sorts; T and the global bound are lowered at each compaction only).
template <bool kLazy = false>
__device__ __forceinline__ void warp_list_add(unsigned long long* list, int& cnt, float& T, int k, uint32_t* bound,
                                              bool take, float dist, uint32_t id) {
  const int lane = threadIdx.x & 31;
  const uint32_t m = __ballot_sync(HG_FULL, take);
  if (!m) return;
  if (take) {
    const int r = __popc(m & ((1u << lane) - 1));
    list[cnt + r] = ((unsigned long long)__float_as_uint(dist) << 32) | id;
  }
  cnt += __popc(m);
  __syncwarp();
  if (kLazy ? cnt > kWarpListCap - 32 : cnt >= k) {
    cnt = warp_compact(list, cnt, k);
    if (cnt == k) {
      const float nt = __uint_as_float((uint32_t)(list[k - 1] >> 32));
      if (nt < T) {
        T = nt;
        if (lane == 0 && bound) atomicMin(bound, __float_as_uint(T));
      }
    }
  }
}

// Candidate index of `unit` among the LB-ordered candidate leaves: the
// largest c with unit_prefix[c] <= unit, searched from the previous c.
__device__ __forceinline__ int unit_candidate(const uint32_t* unit_prefix, int ncand, int c, uint32_t unit) {
  int lo = c, hi = ncand - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (unit_prefix[mid] <= unit) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// The same search by a whole warp (every lane calls it; all get the answer):
// 32 probes per round narrow [lo, ncand - 1] 32-fold.  unit_prefix[lo] <=
// unit must hold on entry.
__device__ __forceinline__ int unit_candidate_warp(const uint32_t* unit_prefix, int ncand, int lo, uint32_t unit,
                                                   int lane) {
  int hi = ncand - 1;
  while (true) {
    const int step = hi - lo >= 32 ? (hi - lo + 32) / 32 : 1;  // probes lo, lo + step, ... cover [lo, hi]
    const int p = lo + lane * step;
    const uint32_t le = __ballot_sync(0xffffffffu, p <= hi && unit_prefix[p] <= unit);
    const int j = le ? 31 - __clz(le) : 0;  // probes at or below `unit` form a prefix of the lanes
    if (step == 1) return lo + j;
    lo += j * step;
    hi = min(hi, lo + step - 1);
  }
}


}  // namespace hg
