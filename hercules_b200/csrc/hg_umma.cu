// hg_umma.cu -- the batched filter's q.x products on the 5th-generation tensor
// cores: tcgen05.mma (BF16 x BF16 -> FP32 in tensor memory), operands staged
// by TMA with the 128-byte swizzle, fused epilogues read back with tcgen05.ld.
//
// One persistent CTA per SM, 12 warps:
//   warp 0      TMA producer (one elected lane): row tiles (A, 128 rows x 64 K
//               per stage) and the query tile (B, 256 queries x L, resident
//               in shared memory for L <= 256, else streamed with A);
//   warp 1      MMA issuer (one lane): per 128-row tile, L/16 MMAs of
//               M=128, N=256, K=16 into one of two TMEM accumulators;
//   warp 2      allocates / frees the 512 TMEM columns;
//   warps 4-11  epilogue: warp w reads TMEM lanes 32 (w % 4) .. +31 (the
//               tile's rows) and columns 128 ((w - 4) / 4) .. +127 (queries).
// Work items are (128-row tiles, query tile) pairs, pulled by the producer
// from a device queue (an atomic counter; a static round robin without one)
// and handed to the MMA and epilogue warps through a two-entry ring:
// mode 1 walks row chunks x query tiles (a chunk's query tiles run side by
// side so the chunk is read from HBM once); mode 0 walks an item list
// (approximate leaves x the queries routed there) for the bound pass; mode 3
// walks an item list (leaves x the queries that LB_EAPCA keeps for them) with
// mode 1's screening epilogue; mode 2 writes the raw dot products
// (diagnostics).  Every mbarrier wait gives up after kWaitNs (or the
// launch's wait_ns) of global time: the CTA then raises *err, drains its copies and MMAs, frees
// TMEM and returns.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "hg_batch.h"
#include "hg_device.cuh"

namespace hg {
namespace {

constexpr int kUM = 128;       // rows per tile (MMA M)
constexpr int kUN = 256;       // queries per tile (MMA N)
constexpr int kUK = 64;        // K elements per stage: one 128-byte swizzle row
constexpr int kAStages = 5;      // A stages (4 when the query tile is streamed with A)
constexpr int kThreads = 384;  // 12 warps
constexpr int kEpiThreads = 256;
constexpr uint32_t kABytes = kUM * kUK * 2;  // 16 KB per A stage
constexpr uint32_t kQBytes = kUN * kUK * 2;  // 32 KB per query K block
constexpr int kResidentKB = 4;               // L <= 256: the query tile stays resident
constexpr uint64_t kWaitNs = 2000000000ull;  // 2 s per wait
constexpr int kErrTimeout = 1;
constexpr uint32_t kPairBlock = 1024;        // survivor pairs reserved per warp at a time

// The screening modes fold each query's threshold into the accumulator with
// one more K = 16 MMA per tile: A_ext (128 rows x 16, every element 1) times
// B_ext (the item's queries x 16: -t_hi, -t_lo, then zeros), both K-major in
// the 32-byte swizzle layout (rows of 32 bytes, 8-row groups 256 bytes apart)
constexpr uint32_t kExtRow = 32;                               // bytes per row of a K = 16 BF16 slab
constexpr uint32_t kNoItem = 0xffffffffu;                      // ring entry: no more items

// Shared memory map (offsets from a 1024-byte aligned base): the query tile
// (4 K blocks; 256 queries, or 64 in the bound pass with L <= 256, which then
// keeps eleven row stages instead of five), the row stages (128 rows x 64 K),
// A_ext (128 x 32 B), B_ext (256 x 32 B), the mbarriers (full / empty per
// stage, query tile full / empty, TMEM full / empty x2, done, item ring
// full / empty x2, B_ext full / empty), the TMEM base address, the abort
// flag, the tile's query indices and norms, the epilogue warps' flags and the
// item ring.
template <bool kBound>
struct FilterLayout {
  static constexpr uint32_t kQBlk = kBound ? (uint32_t)kBatchBoundQueries * kUK * 2 : kQBytes;  // per K block
  static constexpr int kStages = kBound ? 11 : kAStages;
  static constexpr uint32_t kQ = 0;
  static constexpr uint32_t kA = kQ + kResidentKB * kQBlk;
  static constexpr uint32_t kAext = kA + kStages * kABytes;
  static constexpr uint32_t kBext = kAext + kUM * kExtRow;
  static constexpr uint32_t kBar = kBext + kUN * kExtRow;
  static constexpr uint32_t kBars = 2 * kStages + 2 + 4 + 1 + 4 + 2;
  static constexpr uint32_t kTmem = kBar + kBars * 8;
  static constexpr uint32_t kAbort = kTmem + 4;
  static constexpr uint32_t kQidx = (kAbort + 4 + 15) & ~15u;
  static constexpr uint32_t kQn2 = kQidx + kUN * 4;
  static constexpr uint32_t kOkw = kQn2 + kUN * 4;
  static constexpr uint32_t kItem = kOkw + 32;
  static constexpr size_t kDyn = kItem + 8 + 1024;
};
static_assert(FilterLayout<true>::kDyn <= 232448 && FilterLayout<false>::kDyn <= 232448, "filter shared memory");

// --- PTX wrappers -------------------------------------------------------------

__device__ __forceinline__ uint32_t s2u(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

// Bounded wait for the phase of `parity`; false when this CTA aborted or
// the wait ran past wait_ns (then the CTA aborts and *err is raised).
__device__ __noinline__ bool mbar_wait_slow(uint32_t bar, uint32_t parity, volatile int* abort_flag, int* err,
                                            uint64_t wait_ns) {
  const uint64_t t0 = global_ns();
  for (uint32_t i = 1;; ++i) {
    if (mbar_try(bar, parity)) return true;
    if ((i & 63) == 0) {
      if (*abort_flag) return false;
      if (global_ns() - t0 > wait_ns) {
        *abort_flag = 1;
        atomicExch(err, kErrTimeout);
        return false;
      }
    }
  }
}

// the first test inline, the polling loop out of line
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, volatile int* abort_flag, int* err,
                                         uint64_t wait_ns) {
  return mbar_try(bar, parity) || mbar_wait_slow(bar, parity, abort_flag, err, wait_ns);
}

// Wait for a phase that is known to complete on its own (copies and MMAs
// already issued), bounded, ignoring the abort flag.
__device__ __noinline__ void drain_wait(uint32_t bar, uint32_t parity, uint64_t wait_ns) {
  const uint64_t t0 = global_ns();
  while (!mbar_try(bar, parity) && global_ns() - t0 < wait_ns) {
  }
}

__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int x, int y, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
          dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
      : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}
// D[tmem] (+)= A[smem] x B[smem]^T, both K-major
__device__ __forceinline__ void tc_mma(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(d),
      "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
      : "memory");
}
__device__ __forceinline__ void tc_ld32(uint32_t taddr, uint32_t (&r)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
}
__device__ __forceinline__ void tc_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void named_sync(uint32_t id, uint32_t n) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(n) : "memory");
}

// Shared-memory matrix descriptor of a K-major operand in the 128-byte
// swizzle layout: rows of 128 bytes, 8-row groups 1024 bytes apart
// (stride byte offset 64 x 16 B), leading byte offset unused (1),
// descriptor version 1, layout type 2 (128-byte swizzle).
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
  return (uint64_t)((saddr & 0x3FFFFu) >> 4) | ((uint64_t)1 << 16) | ((uint64_t)64 << 32) | ((uint64_t)1 << 46) |
         ((uint64_t)2 << 61);
}

// The same for a K = 16 slab in the 32-byte swizzle layout: rows of 32
// bytes, 8-row groups 256 bytes apart (stride byte offset 16 x 16 B),
// layout type 6.
__device__ __forceinline__ uint64_t sw32_desc(uint32_t saddr) {
  return (uint64_t)((saddr & 0x3FFFFu) >> 4) | ((uint64_t)1 << 16) | ((uint64_t)16 << 32) | ((uint64_t)1 << 46) |
         ((uint64_t)6 << 61);
}

// BF16 bits of a float, round to nearest even (finite or infinite inputs)
__device__ __forceinline__ uint32_t bf16_bits(float f) {
  return (uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(f));
}

// Instruction descriptor: FP32 accumulator, BF16 A and B, both K-major,
// N (bits 17-22: N / 8; a multiple of 16 up to 256), M = 128 (bits 24-28: M / 16).
__host__ __device__ constexpr uint32_t idesc_for(int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(kUM >> 4) << 24);
}
// MMA width of an item: its query count rounded up to 16, at most the tile
// (the bound pass groups at most kBatchBoundQueries queries per approximate
// leaf; a leaf's last query tile in the pruned filter is partly filled)
__device__ __forceinline__ int item_n(uint32_t qcnt, int qtile) {
  const int n = (int)((qcnt + 15u) & ~15u);
  return n < 16 ? 16 : (n > qtile ? qtile : n);
}

// max(a, b, c) in one instruction (three-input max.f32 of sm_100)
__device__ __forceinline__ float fmax3(float a, float b, float c) {
  float r;
  asm("max.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
  return r;
}

// Survivor mask of 32 accumulators against h (bit j: j < nv and v[j] >= h):
// the maxima of four 8-column groups first (three-input max), then the
// compares only in the groups whose maximum reaches h
__device__ __forceinline__ uint32_t screen32(const float* v, float h, int nv) {
  float g[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const float* w = v + 8 * q;
    g[q] = fmaxf(fmax3(fmax3(w[0], w[1], w[2]), w[3], w[4]), fmax3(w[5], w[6], w[7]));
  }
  uint32_t mask = 0;
  if (fmax3(g[0], g[1], fmaxf(g[2], g[3])) >= h) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      if (g[q] >= h) {
#pragma unroll
        for (int j = 8 * q; j < 8 * q + 8; ++j) mask |= (j < nv && v[j] >= h) ? (1u << j) : 0u;
      }
    }
  }
  return mask;
}

__device__ __forceinline__ uint32_t ordered_key(float f) {
  const uint32_t b = __float_as_uint(f);
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}

struct Item {
  uint64_t rb, re;  // tile t covers rows rb + 128 t .., valid in [vb, re)
  uint64_t vb;
  uint32_t qoff, qcnt;
  uint32_t t_lo, t_hi;
  uint32_t sub;
};

__device__ __forceinline__ Item item_of(const BatchGemm& a, uint32_t w, uint32_t QT, uint64_t ntiles, int qtile,
                                        int nq) {
  Item it;
  if (a.mode == 0 || a.mode == 3) {
    const BatchItem b = a.items[w];
    it.rb = b.row_begin;
    it.re = b.row_end;
    it.vb = b.row_begin + b.row_skip;
    it.qoff = b.q_off;
    it.qcnt = b.q_cnt;
    it.t_lo = b.tile_lo;
    it.t_hi = b.tile_hi;
    it.sub = b.sub;
  } else {
    const uint32_t chunk = w / QT, qt = w % QT;
    it.rb = 0;
    it.re = a.nrows;
    it.vb = 0;
    it.qoff = qt * (uint32_t)qtile;
    it.qcnt = (uint32_t)min(nq - (int)it.qoff, qtile);
    it.t_lo = chunk * a.tiles_per_item;
    const uint64_t th = (uint64_t)it.t_lo + a.tiles_per_item;
    it.t_hi = (uint32_t)(th < ntiles ? th : ntiles);
    it.sub = 1;
  }
  return it;
}

}  // namespace

// kScreen: modes 1 and 3 (else 0 and 2); kResident: L <= 256, the query tile
// stays in shared memory (else it is streamed with the row tiles).  The
// launcher picks the instance, so the per-stage loops carry no mode tests.
template <bool kScreen, bool kResident, bool kBound>
__global__ void __launch_bounds__(kThreads, 1)
    k_umma_filter(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmQ, BatchGemm a) {
  using LY = FilterLayout<kBound>;
  extern __shared__ unsigned char umma_raw[];
  unsigned char* sm = umma_raw + ((1024 - (s2u(umma_raw) & 1023)) & 1023);
  const uint32_t base = s2u(sm);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t bar0 = base + LY::kBar;
  auto full_bar = [&](int s) { return bar0 + 8u * s; };
  auto empty_bar = [&](int s) { return bar0 + 8u * (LY::kStages + s); };
  const uint32_t qfull_bar = bar0 + 8u * (2 * LY::kStages);
  const uint32_t qempty_bar = qfull_bar + 8;
  auto tfull_bar = [&](int b) { return qempty_bar + 8u + 8u * b; };
  auto tempty_bar = [&](int b) { return qempty_bar + 24u + 8u * b; };
  const uint32_t done_bar = qempty_bar + 40u;
  auto ifull_bar = [&](int sl) { return done_bar + 8u + 8u * sl; };
  auto iempty_bar = [&](int sl) { return done_bar + 24u + 8u * sl; };
  const uint32_t bfull_bar = done_bar + 40u;   // B_ext written for the item (epilogue -> MMA)
  const uint32_t bempty_bar = done_bar + 48u;  // the item's MMAs have read B_ext (MMA -> epilogue)
  volatile uint32_t* s_item = reinterpret_cast<volatile uint32_t*>(sm + LY::kItem);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(sm + LY::kAbort);
  uint32_t* s_qidx = reinterpret_cast<uint32_t*>(sm + LY::kQidx);
  float* s_qn2 = reinterpret_cast<float*>(sm + LY::kQn2);
  volatile int* s_okw = reinterpret_cast<volatile int*>(sm + LY::kOkw);

  const uint64_t wns = a.wait_ns ? a.wait_ns : kWaitNs;  // every bounded wait gives up after this
  const int nkb = (a.L + kUK - 1) / kUK;
  constexpr bool resident = kResident;
  // A streamed query tile (L > 256) is shared by two row tiles: each stage
  // holds one query K block and the same K block of two row tiles, whose
  // products go to the two TMEM accumulators (the epilogue then takes both at
  // once); three such stages of 64 KB fit.  A resident tile serves one row
  // tile per accumulator, double-buffered.
  constexpr uint32_t kGroup = resident ? 1u : 2u;                 // row tiles per MMA group
  constexpr uint32_t nst = resident ? (uint32_t)LY::kStages : 3u;
  constexpr uint32_t aBase = resident ? LY::kA : 3u * kQBytes;  // row stages (streamed: after the 3 query slots)
  static_assert(resident || aBase + nst * kGroup * kABytes <= LY::kAext, "streamed stages");
  // query count (read on the device for rounds planned there) and queries
  // per tile (MMA N): 64 in the bound pass, else the launch's choice or, for
  // 0, the narrowest of 64 / 128 / 256 that holds the queries
  const int nq = a.nq_dev ? (int)min((uint32_t)a.nq, *a.nq_dev) : a.nq;
  const bool listed = a.mode == 0 || a.mode == 3;  // items from a.items
  constexpr bool screen = kScreen;  // threshold epilogue, survivor pairs
  const int qtile = a.mode == 0 ? kBatchBoundQueries
                                : (a.qtile ? a.qtile : (nq <= 64 ? 64 : (nq <= 128 ? 128 : kUN)));
  const uint32_t QT = (uint32_t)((nq + qtile - 1) / qtile);
  const uint64_t ntiles = (a.nrows + kUM - 1) / kUM;
  const uint32_t nchunks = (uint32_t)((ntiles + a.tiles_per_item - 1) / a.tiles_per_item);
  const uint32_t total = listed ? (a.nitems_dev ? min(a.nitems, *a.nitems_dev) : a.nitems) : nchunks * QT;

  if (tid == 0) {
    for (int s = 0; s < LY::kStages; ++s) {
      mbar_init(full_bar(s), 1);
      mbar_init(empty_bar(s), 1);
    }
    mbar_init(qfull_bar, 1);
    mbar_init(qempty_bar, 1);
    for (int b = 0; b < 2; ++b) {
      mbar_init(tfull_bar(b), 1);
      mbar_init(tempty_bar(b), kEpiThreads / 32);
    }
    mbar_init(done_bar, 1);
    mbar_init(bfull_bar, 1);
    mbar_init(bempty_bar, 1);
    for (int sl = 0; sl < 2; ++sl) {
      mbar_init(ifull_bar(sl), 1);
      mbar_init(iempty_bar(sl), 1 + kEpiThreads / 32);  // the MMA lane and every epilogue warp
    }
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (screen) {
    // A_ext: every element 1 (BF16 0x3F80); B_ext: zero until an item's
    // thresholds are written.  Generic-proxy writes, made visible to the
    // tensor cores (async proxy) before the barrier below.
    uint32_t* ae = reinterpret_cast<uint32_t*>(sm + LY::kAext);
    uint32_t* be = reinterpret_cast<uint32_t*>(sm + LY::kBext);
    for (int i = tid; i < (int)(kUM * kExtRow / 4); i += kThreads) ae[i] = 0x3F803F80u;
    for (int i = tid; i < (int)(kUN * kExtRow / 4); i += kThreads) be[i] = 0u;
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  if (warp == 2) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;" ::"r"(base + LY::kTmem)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *reinterpret_cast<volatile uint32_t*>(sm + LY::kTmem);

  if (warp == 0) {
    // ---------------- TMA producer
    if (lane == 0) {
      uint32_t g = 0, it_n = 0, q_issued = 0;
      uint32_t s_cur = 0, ph = 0;  // stage g % nst and the parity of g / nst
      bool ok = true;
      for (;; ++it_n) {
        // the next item into the ring (its entry free once every consumer
        // has read it), or kNoItem when the queue is empty
        const int sl = (int)(it_n & 1);
        ok = mbar_wait(iempty_bar(sl), ((it_n >> 1) & 1) ^ 1, abort_flag, a.err, wns);
        if (!ok) break;
        const uint32_t w = a.queue ? atomicAdd(a.queue, 1u) : blockIdx.x + it_n * gridDim.x;
        s_item[sl] = w < total ? w : kNoItem;
        mbar_arrive(ifull_bar(sl));
        if (w >= total) break;
        const Item it = item_of(a, w, QT, ntiles, qtile, nq);
        if (resident) {
          ok = mbar_wait(qempty_bar, (it_n & 1) ^ 1, abort_flag, a.err, wns);
          if (!ok) break;
          mbar_expect_tx(qfull_bar, (uint32_t)nkb * LY::kQBlk);
          for (int kb = 0; kb < nkb; ++kb)
            tma_load_2d(base + LY::kQ + kb * LY::kQBlk, &tmQ, kb * kUK, (int)it.qoff, qfull_bar);
          ++q_issued;
        }
        const uint32_t ngroups = it.t_hi > it.t_lo ? (it.t_hi - it.t_lo + kGroup - 1) / kGroup : 0u;
        for (uint32_t jg = 0; ok && jg < ngroups; ++jg) {
          const uint32_t t0 = it.t_lo + jg * kGroup;
          for (int kb = 0; kb < nkb; ++kb, ++g) {
            const int s = (int)s_cur;
            const uint32_t par = ph;
            if (++s_cur == nst) {
              s_cur = 0;
              ph ^= 1u;
            }
            ok = mbar_wait(empty_bar(s), par ^ 1, abort_flag, a.err, wns);
            if (!ok) break;
            // diagnostics: the first stage's copy withheld, so its barrier
            // phase never completes and the MMA warp's bounded wait runs out
            if (a.withhold_first_copy && g == 0) continue;
            mbar_expect_tx(full_bar(s), kGroup * kABytes + (resident ? 0u : kQBytes));
#pragma unroll
            for (uint32_t gi = 0; gi < kGroup; ++gi)
              tma_load_2d(base + aBase + (s * kGroup + gi) * kABytes, &tmA, kb * kUK,
                          (int)(it.rb + (uint64_t)(t0 + gi) * kUM), full_bar(s));
            if (!resident) tma_load_2d(base + LY::kQ + s * kQBytes, &tmQ, kb * kUK, (int)it.qoff, full_bar(s));
          }
        }
        if (!ok) break;
      }
      if (!ok || a.withhold_first_copy) {
        // drain the copies still in flight before the CTA leaves (bounded:
        // a withheld copy's phase never completes)
        const uint32_t first = g > nst ? g - nst : 0;
        for (uint32_t gg = first; gg < g; ++gg) drain_wait(full_bar((int)(gg % nst)), (gg / nst) & 1, wns);
        if (resident && q_issued > 0) drain_wait(qfull_bar, (q_issued - 1) & 1, wns);
      }
    }
  } else if (warp == 1) {
    // ---------------- MMA issuer
    if (lane == 0) {
      uint32_t g = 0, tcount = 0, it_n = 0;
      uint32_t s_cur = 0, ph = 0;  // stage g % nst and the parity of g / nst
      const uint64_t dae = sw32_desc(base + LY::kAext), dbe = sw32_desc(base + LY::kBext);
      bool ok = true;
      for (; ok; ++it_n) {
        const int sl = (int)(it_n & 1);
        ok = mbar_wait(ifull_bar(sl), (it_n >> 1) & 1, abort_flag, a.err, wns);
        if (!ok) break;
        const uint32_t w = s_item[sl];
        mbar_arrive(iempty_bar(sl));
        if (w == kNoItem) break;
        const Item it = item_of(a, w, QT, ntiles, qtile, nq);
        if (resident) {
          ok = mbar_wait(qfull_bar, it_n & 1, abort_flag, a.err, wns);
          if (!ok) break;
          tc_fence_after();
        }
        if (screen) {
          // the item's thresholds in B_ext (written by the epilogue warps)
          ok = mbar_wait(bfull_bar, it_n & 1, abort_flag, a.err, wns);
          if (!ok) break;
          tc_fence_after();
        }
        const uint32_t idesc = idesc_for(item_n(it.qcnt, qtile));
        const uint32_t ngroups = it.t_hi > it.t_lo ? (it.t_hi - it.t_lo + kGroup - 1) / kGroup : 0u;
        for (uint32_t jg = 0; ok && jg < ngroups; ++jg, ++tcount) {
          const int b = kGroup == 1 ? (int)(tcount & 1) : 0;
          const uint32_t tph = kGroup == 1 ? ((tcount >> 1) & 1) : (tcount & 1);
          ok = mbar_wait(tempty_bar(b), tph ^ 1, abort_flag, a.err, wns);
          if (!ok) break;
          tc_fence_after();
          const uint32_t d = tmem + (uint32_t)b * kUN;  // + gi * kUN for the group's row tile gi
          // screening: the accumulator starts as -(t_hi + t_lo) of its column
          if (screen) {
#pragma unroll
            for (uint32_t gi = 0; gi < kGroup; ++gi) tc_mma(d + gi * kUN, dae, dbe, idesc, 0u);
          }
          for (int kb = 0; kb < nkb; ++kb, ++g) {
            const int s = (int)s_cur;
            const uint32_t par = ph;
            if (++s_cur == nst) {
              s_cur = 0;
              ph ^= 1u;
            }
            ok = mbar_wait(full_bar(s), par, abort_flag, a.err, wns);
            if (!ok) break;
            tc_fence_after();
            // K step k16 is 32 bytes on: 2 in the descriptors' address field
            const uint64_t dq = sw128_desc(base + LY::kQ + (resident ? (uint32_t)kb * LY::kQBlk : (uint32_t)s * kQBytes));
#pragma unroll
            for (uint32_t gi = 0; gi < kGroup; ++gi) {
              const uint64_t da = sw128_desc(base + aBase + (s * kGroup + gi) * kABytes);
#pragma unroll
              for (int k16 = 0; k16 < kUK / 16; ++k16)
                tc_mma(d + gi * kUN, da + 2 * k16, dq + 2 * k16, idesc, (screen || kb || k16) ? 1u : 0u);
            }
            tc_commit(empty_bar(s));
          }
          if (ok) tc_commit(tfull_bar(b));
        }
        if (ok && resident) tc_commit(qempty_bar);
        if (ok && screen) tc_commit(bempty_bar);  // B_ext free once the item's MMAs are done
      }
      // every MMA issued has completed before TMEM is freed
      tc_commit(done_bar);
      drain_wait(done_bar, 0, wns);
    }
  } else if (warp >= 4) {
    // ---------------- epilogue
    const int etid = tid - 128;
    const int ew = warp - 4;
    const int quarter = warp & 3;
    const int half = ew >> 2;
    const float inf = __int_as_float(0x7f800000);
    uint32_t tcount = 0;
    uint32_t pcur = 0, pend = 0;  // the warp's reserved block of the pair list
    bool ok = true;
    // the certified bounds this thread's columns used (a.errstat)
    float e_sum = 0.0f, e_rel = 0.0f, e_max = 0.0f;
    uint32_t e_cnt = 0, e_rcnt = 0;
    for (uint32_t it_n = 0;; ++it_n) {
      // the next item from the ring (lane 0 waits, bounded)
      const int sl = (int)(it_n & 1);
      uint32_t w = kNoItem;
      int got = 1;
      if (lane == 0) {
        got = mbar_wait(ifull_bar(sl), (it_n >> 1) & 1, abort_flag, a.err, wns) ? 1 : 0;
        if (got) {
          w = s_item[sl];
          mbar_arrive(iempty_bar(sl));
        }
      }
      got = __shfl_sync(HG_FULL, got, 0);
      w = __shfl_sync(HG_FULL, w, 0);
      ok = ok && got;
      // item boundary: every epilogue warp is done with the previous item
      // and all of them learn whether any gave up; all of them read the
      // same entry, so they leave together at the end of the queue
      if (lane == 0) s_okw[ew] = ok ? 1 : 0;
      named_sync(1, kEpiThreads);
      bool all_ok = true;
#pragma unroll
      for (int i = 0; i < kEpiThreads / 32; ++i) all_ok = all_ok && s_okw[i] != 0;
      if (!all_ok || w == kNoItem) break;
      const Item it = item_of(a, w, QT, ntiles, qtile, nq);
      // column etid of the query tile
      uint32_t q = 0xffffffffu;
      float4 qm = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
      float qb = -1.0f;
      if ((uint32_t)etid < it.qcnt) {
        q = a.qperm[it.qoff + etid];
        qm = a.qmeta[q];
        if (screen) {
          const float b = a.bound[q];
          qb = b < inf ? b : -1.0f;
        }
      }
      s_qidx[etid] = q;
      s_qn2[etid] = qm.x;
      float tv = inf;
      if (screen) {
        // norm maxima over the item's rows (its 128-row tiles), then the
        // column's threshold: keep (row, q) when acc - t_q >= |x|^2 / 2 with
        // t_q = (|q|^2 - B - err) / 2
        float4 tm = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        for (uint32_t t = it.t_lo + lane; t < it.t_hi; t += 32) {
          const float4 v = a.tile_meta[(it.rb + (uint64_t)t * kUM) / kUM];
          tm.x = fmaxf(tm.x, v.x);
          tm.y = fmaxf(tm.y, v.y);
          tm.z = fmaxf(tm.z, v.z);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
          tm.x = fmaxf(tm.x, __shfl_xor_sync(HG_FULL, tm.x, o));
          tm.y = fmaxf(tm.y, __shfl_xor_sync(HG_FULL, tm.y, o));
          tm.z = fmaxf(tm.z, __shfl_xor_sync(HG_FULL, tm.z, o));
        }
        tv = inf;  // no bound (or no query): acc - inf = -inf never survives
        if (qb >= 0.0f) {
          const float err = 2.000002f * (qm.y * tm.z + qm.z * tm.y + qm.z * tm.z + a.c_acc * qm.y * tm.y) +
                            a.c_sq * (qm.x + tm.x + qb) + 1e-5f;
          tv = 0.5f * (qm.x - qb - err);
          if (a.errstat) {
            e_sum += err;
            e_max = fmaxf(e_max, err);
            ++e_cnt;
            if (qb > 0.0f) {
              e_rel += err / qb;
              ++e_rcnt;
            }
          }
        }
        // the tensor cores subtract tv as the BF16 pair t_hi + t_lo inside
        // the accumulation: lower it by the split's rounding (2^-16 |tv|)
        // and by the accumulation's rounding of the larger partial sums
        // (c_acc |tv|), with room to spare (2^-14 (|tv| + |q~| |x~|)), so
        // the test keeps at least every pair the exact test keeps
        if (tv < inf) tv -= a.c_acc * fabsf(tv) + 6.103515625e-05f * (fabsf(tv) + qm.y * tm.y);
      }
      if (screen) {
        // B_ext may be rewritten once the previous item's MMAs have read it
        if (ew == 0 && it_n > 0) {
          int okb = 1;
          if (lane == 0) okb = mbar_wait(bempty_bar, (it_n - 1) & 1, abort_flag, a.err, wns) ? 1 : 0;
          okb = __shfl_sync(HG_FULL, okb, 0);
          ok = ok && okb;
        }
        named_sync(1, kEpiThreads);
        // row etid of B_ext: -t_hi, -t_lo in K positions 0 and 1 (the rest
        // stays zero); the 32-byte swizzle puts a row's logical 16-byte
        // chunk 0 at chunk (row >> 2) & 1 (address bit 4 ^= bit 7)
        float th = tv, tl = 0.0f;
        if (tv < inf) {
          th = __bfloat162float(__float2bfloat16_rn(tv));
          tl = tv - th;  // exact: th is within a factor 2 of tv
        }
        const uint32_t row = (uint32_t)etid;
        *reinterpret_cast<uint32_t*>(sm + LY::kBext + row * kExtRow + (((row >> 2) & 1u) << 4)) =
            bf16_bits(-th) | (bf16_bits(-tl) << 16);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      }
      named_sync(1, kEpiThreads);
      if (screen && etid == 0) mbar_arrive(bfull_bar);
      // the two warp groups split the item's columns (32-column granules)
      const int half_cols = min(qtile / 2, (int)((it.qcnt + 63u) / 64u) * 32);
      const int c_lo = half * half_cols;
      const int c_hi = min(c_lo + half_cols, (int)it.qcnt);
      // the bound pass (64-query tiles: one 32-column chunk per warp): half
      // the query norms of the warp's columns in registers; its keys order
      // d~ / 2 = (|x|^2 + |q|^2) / 2 - q~.x~
      static_assert(kBatchBoundQueries == 64, "one chunk per epilogue warp in the bound pass");
      float gq[32];
      if (!screen && a.mode == 0) {
#pragma unroll
        for (int j = 0; j < 32; ++j) gq[j] = 0.5f * s_qn2[(c_lo + j) & (kUN - 1)];
      }
      // the rows' |x|^2, loaded one group of row tiles ahead
      float xn_next[kGroup];
      auto prefetch = [&](uint32_t jg) {
#pragma unroll
        for (uint32_t gi = 0; gi < kGroup; ++gi) {
          const uint32_t t = it.t_lo + jg * kGroup + gi;
          const uint64_t rw = it.rb + (uint64_t)t * kUM + quarter * 32 + lane;
          xn_next[gi] = (t < it.t_hi && rw >= it.vb && rw < it.re && rw < a.nrows) ? a.xmeta[rw].x : 0.0f;
        }
      };
      const uint32_t ngroups = it.t_hi > it.t_lo ? (it.t_hi - it.t_lo + kGroup - 1) / kGroup : 0u;
      prefetch(0);
      for (uint32_t jg = 0; ok && jg < ngroups; ++jg, ++tcount) {
        const int b = kGroup == 1 ? (int)(tcount & 1) : 0;
        const uint32_t tph = kGroup == 1 ? ((tcount >> 1) & 1) : (tcount & 1);
        float xn2s[kGroup];
#pragma unroll
        for (uint32_t gi = 0; gi < kGroup; ++gi) xn2s[gi] = xn_next[gi];
        if (jg + 1 < ngroups) prefetch(jg + 1);
        // each warp waits for the accumulator itself (lane 0, result shared)
        int go = 0;
        if (lane == 0) go = mbar_wait(tfull_bar(b), tph, abort_flag, a.err, wns) ? 1 : 0;
        go = __shfl_sync(HG_FULL, go, 0);
        if (!go) {
          ok = false;
          break;
        }
        tc_fence_after();
        // mode 1: survivor masks of the warp's (up to) four 32-column chunks
        // per row tile; the buckets are written after the accumulator is
        // handed back
        uint32_t masks[kGroup][4];
        uint64_t rows_g[kGroup];
#pragma unroll
        for (uint32_t gi = 0; gi < kGroup; ++gi) {
        const uint32_t t = it.t_lo + jg * kGroup + gi;
        const uint64_t row = it.rb + (uint64_t)t * kUM + quarter * 32 + lane;
        const bool row_ok = t < it.t_hi && row >= it.vb && row < it.re && row < a.nrows;
        rows_g[gi] = row;
        const float xn2 = xn2s[gi];
        const float h_row = row_ok ? 0.5f * xn2 : inf;
        const uint32_t tbase = tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(b + (int)gi) * kUN;
        masks[gi][0] = masks[gi][1] = masks[gi][2] = masks[gi][3] = 0u;
        if (screen) {
#pragma unroll
          for (int i2 = 0; i2 < 2; ++i2) {
            const int c0 = c_lo + 64 * i2;
            if (c0 >= c_hi) break;  // uniform over the warp
            uint32_t r[2][32];
            tc_ld32(tbase + (uint32_t)c0, r[0]);
            tc_ld32(tbase + (uint32_t)(c0 + 32), r[1]);
            tc_wait_ld();
#pragma unroll
            for (int hh = 0; hh < 2; ++hh) {
              const int cb = c0 + 32 * hh;
              if (cb >= c_hi) break;  // uniform over the warp
              // the accumulators already hold acc_j - t_j: screen by their
              // maximum; columns past the item's queries never survive
              masks[gi][2 * i2 + hh] = screen32(reinterpret_cast<const float*>(r[hh]), h_row, c_hi - cb);
            }
          }
        } else {
          for (int c0 = c_lo; c0 < c_hi; c0 += 32) {
            uint32_t r[32];
            tc_ld32(tbase + (uint32_t)c0, r);
            tc_wait_ld();
            if (a.mode == 0) {
              const int span = kUM / (int)it.sub;  // rows per slot: 8 .. 128
              const float h2 = 0.5f * xn2;
              // 32-bit keys: the order-preserving bits of d~ with the low 7
              // replaced by the row's index in its 128-row tile (a relative
              // 2^-16 of d~; the exact ranking of the candidates decides)
              const uint32_t rit = (uint32_t)(quarter * 32 + lane);
              const uint64_t tile_row0 = it.rb + (uint64_t)t * kUM;
              auto slot_key = [&](uint32_t k32) {
                return ((unsigned long long)(k32 & ~0x7Fu) << 32) | (uint32_t)(tile_row0 + (k32 & 0x7Fu));
              };
              if (span >= 32 && c_hi - c0 <= 16) {
                // at most 16 columns (the usual bound-pass group): rows l and
                // l + 16 combined first, then a 16-column butterfly
                // transpose-min in each half, so lane l (< 16) ends with
                // column c0 + l reduced over the 32 rows
                uint32_t v[16];
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                  const float dd = (h2 + gq[j]) - __uint_as_float(r[j]);
                  v[j] = row_ok ? ((ordered_key(dd) & ~0x7Fu) | rit) : 0xffffffffu;
                }
#pragma unroll
                for (int j = 0; j < 16; ++j) v[j] = min(v[j], __shfl_xor_sync(HG_FULL, v[j], 16));
#pragma unroll
                for (int o = 8; o >= 1; o >>= 1) {
                  const bool upper = (lane & o) != 0;
#pragma unroll
                  for (int i = 0; i < o; ++i) {
                    const uint32_t send = upper ? v[i] : v[i + o];
                    const uint32_t keep = upper ? v[i + o] : v[i];
                    v[i] = min(keep, __shfl_xor_sync(HG_FULL, send, o));
                  }
                }
                const uint32_t slot = t * it.sub + (uint32_t)(quarter * 32 / span);
                if (lane < 16 && c0 + lane < c_hi && v[0] != 0xffffffffu && slot < a.bm_cap)
                  atomicMin(&a.bm[(uint64_t)s_qidx[c0 + lane] * a.bm_cap + slot], slot_key(v[0]));
              } else if (span >= 32) {
                // the warp's 32 rows lie in one slot: butterfly transpose-min,
                // lane l ends with column c0 + l reduced over the 32 rows
                uint32_t v[32];
#pragma unroll
                for (int j = 0; j < 32; ++j) {
                  const float dd = (h2 + gq[j]) - __uint_as_float(r[j]);
                  v[j] = row_ok ? ((ordered_key(dd) & ~0x7Fu) | rit) : 0xffffffffu;
                }
#pragma unroll
                for (int o = 16; o >= 1; o >>= 1) {
                  const bool upper = (lane & o) != 0;
#pragma unroll
                  for (int i = 0; i < o; ++i) {
                    const uint32_t send = upper ? v[i] : v[i + o];
                    const uint32_t keep = upper ? v[i + o] : v[i];
                    v[i] = min(keep, __shfl_xor_sync(HG_FULL, send, o));
                  }
                }
                const uint32_t slot = t * it.sub + (uint32_t)(quarter * 32 / span);
                if (c0 + lane < c_hi && v[0] != 0xffffffffu && slot < a.bm_cap)
                  atomicMin(&a.bm[(uint64_t)s_qidx[c0 + lane] * a.bm_cap + slot], slot_key(v[0]));
              } else {
                const int grp = span;
#pragma unroll
                for (int j = 0; j < 32; ++j) {
                  if (c0 + j >= c_hi) break;  // uniform over the warp
                  uint32_t key = 0xffffffffu;
                  if (row_ok) {
                    const float dd = (h2 + gq[j]) - __uint_as_float(r[j]);
                    key = (ordered_key(dd) & ~0x7Fu) | rit;
                  }
                  for (int o = 1; o < grp; o <<= 1) key = min(key, __shfl_xor_sync(HG_FULL, key, o));
                  const uint32_t slot = t * it.sub + (uint32_t)((quarter * 32 + lane) / span);
                  if ((lane & (grp - 1)) == 0 && key != 0xffffffffu && slot < a.bm_cap)
                    atomicMin(&a.bm[(uint64_t)s_qidx[c0 + j] * a.bm_cap + slot], slot_key(key));
                }
              }
            } else if (row_ok) {
#pragma unroll
              for (int j = 0; j < 32; ++j)
                if (c0 + j < c_hi) a.dots[(uint64_t)(it.qoff + c0 + j) * a.dots_ld + row] = __uint_as_float(r[j]);
            }
          }
        }
        }  // row tiles of the group
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(tempty_bar(b));
        // survivor pairs into the warp's reserved block of the pair list:
        // plain stores, one atomic per kPairBlock pairs
#pragma unroll
        for (uint32_t gi = 0; gi < kGroup; ++gi) {
        const uint64_t row = rows_g[gi];
#pragma unroll
        for (int ci = 0; ci < 4; ++ci) {
          uint32_t mask = masks[gi][ci];
          while (__any_sync(HG_FULL, mask != 0)) {
            const bool has = mask != 0;
            unsigned long long e = 0;
            if (has) {
              const int j = __ffs(mask) - 1;
              mask &= mask - 1;
              e = ((unsigned long long)s_qidx[c_lo + 32 * ci + j] << 32) | (uint32_t)row;
            }
            const uint32_t bal = __ballot_sync(HG_FULL, has);
            const uint32_t n = (uint32_t)__popc(bal);
            if (pcur + n > pend) {
              // close the block (sentinels in its tail) and reserve the next
              for (uint32_t i = pcur + lane; i < pend; i += 32) a.pairs[i] = ~0ull;
              uint32_t nb = 0;
              if (lane == 0) nb = atomicAdd(a.pairs_cnt, (uint32_t)kPairBlock);
              nb = __shfl_sync(HG_FULL, nb, 0);
              pcur = nb;
              pend = nb + kPairBlock < a.pairs_cap ? nb + kPairBlock : (nb < a.pairs_cap ? a.pairs_cap : nb);
            }
            const uint32_t slot = pcur + (uint32_t)__popc(bal & ((1u << lane) - 1));
            if (has && slot < pend) a.pairs[slot] = e;
            pcur += n;
          }
        }
        }  // row tiles of the group
      }
    }
    for (uint32_t i = pcur + lane; i < pend; i += 32) a.pairs[i] = ~0ull;  // close the last block
    if (a.errstat) {
      double ds = e_sum, dr = e_rel;
      uint32_t c = e_cnt, rc = e_rcnt;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        ds += __shfl_xor_sync(HG_FULL, ds, o);
        dr += __shfl_xor_sync(HG_FULL, dr, o);
        c += __shfl_xor_sync(HG_FULL, c, o);
        rc += __shfl_xor_sync(HG_FULL, rc, o);
        e_max = fmaxf(e_max, __shfl_xor_sync(HG_FULL, e_max, o));
      }
      if (lane == 0 && c) {
        atomicAdd(&a.errstat[0], ds);
        atomicAdd(&a.errstat[1], dr);
        atomicAdd(&a.errstat[2], (double)c);
        atomicAdd(&a.errstat[3], (double)rc);
        // err >= 0: the order of the bit patterns is the order of the values
        atomicMax(reinterpret_cast<unsigned long long*>(&a.errstat[4]),
                  (unsigned long long)__double_as_longlong((double)e_max));
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 2) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;" ::"r"(tmem) : "memory");
  }
}

// ---------------------------------------------------------------------------
// The screening passes (modes 1 and 3) on CTA pairs: tcgen05.mma with
// cta_group::2, M = 256 rows (128 in each CTA of a 2-CTA cluster) x N
// queries (N / 2 of the query tile in each CTA).  Each CTA keeps only half
// of the query tile resident (64 KB instead of 128 KB), so nine 16 KB row
// stages fit beside it instead of five, and each SM's tensor core reads half
// of the query tile from shared memory per MMA.  Same roles as
// k_umma_filter; the even CTA of the pair (the leader) fetches the work
// items and hands them to its peer, waits for both CTAs' copies (each CTA's
// TMA signals the leader's mbarrier), issues the MMAs, and its commits
// arrive on the barriers of both CTAs (multicast).  Each CTA's epilogue
// reads its own 128 TMEM lanes (its rows) and hands the accumulator back to
// the leader.  Every wait is bounded; a CTA that gives up raises the abort
// flag of both CTAs.  Rows are walked in 256-row pair tiles: the item's
// 128-row tiles t_lo + 2j (even CTA) and t_lo + 2j + 1 (odd CTA).
// ---------------------------------------------------------------------------
namespace {

constexpr int kPStages = 9;                              // row stages of 16 KB
constexpr uint32_t kPQBytes = (kUN / 2) * kUK * 2;       // 16 KB: half a query K block
constexpr uint32_t kPSmQ = 0;                            // 4 x 16 KB
constexpr uint32_t kPSmA = kPSmQ + kResidentKB * kPQBytes;
constexpr uint32_t kPSmAext = kPSmA + kPStages * kABytes;   // 128 x 32 B of ones
constexpr uint32_t kPSmBext = kPSmAext + kUM * kExtRow;     // this CTA's N / 2 thresholds
constexpr uint32_t kPSmBar = kPSmBext + (kUN / 2) * kExtRow;
constexpr uint32_t kPNumBars = 2 * kPStages + 2 + 4 + 1 + 4 + 2;
constexpr uint32_t kPSmTmem = kPSmBar + kPNumBars * 8;
constexpr uint32_t kPSmAbort = kPSmTmem + 4;
constexpr uint32_t kPSmQidx = (kPSmAbort + 4 + 15) & ~15u;
constexpr uint32_t kPSmOkw = kPSmQidx + kUN * 4;
constexpr uint32_t kPSmItem = kPSmOkw + 32;
constexpr uint32_t kPSmBytes = kPSmItem + 8;
constexpr size_t kPDynSmem = kPSmBytes + 1024;
constexpr uint32_t kPEpiArrivals = 2 * kEpiThreads / 32;  // epilogue warps of both CTAs
static_assert(kPDynSmem <= 232448, "pair kernel shared memory");

__device__ __forceinline__ uint32_t cluster_rank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}
// shared::cluster address of the same offset in CTA `rank` of the cluster
__device__ __forceinline__ uint32_t mapa(uint32_t addr, uint32_t rank) {
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(addr), "r"(rank));
  return r;
}
__device__ __forceinline__ void st_cluster(uint32_t caddr, uint32_t v) {
  asm volatile("st.shared::cluster.u32 [%0], %1;" ::"r"(caddr), "r"(v) : "memory");
}
// arrive on a barrier of either CTA (shared::cluster address), release at cluster scope
__device__ __forceinline__ void mbar_arrive_cl(uint32_t caddr) {
  asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(caddr) : "memory");
}
__device__ __forceinline__ bool mbar_try_cl(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait (acquire at cluster scope); on timeout both CTAs' abort flags
// are raised and *err is set.
__device__ __noinline__ bool mbar_wait_cl_slow(uint32_t bar, uint32_t parity, volatile int* abort_flag,
                                               uint32_t peer_abort, int* err, uint64_t wait_ns) {
  const uint64_t t0 = global_ns();
  for (uint32_t i = 1;; ++i) {
    if (mbar_try_cl(bar, parity)) return true;
    if ((i & 63) == 0) {
      if (*abort_flag) return false;
      if (global_ns() - t0 > wait_ns) {
        *abort_flag = 1;
        st_cluster(peer_abort, 1u);
        atomicExch(err, kErrTimeout);
        return false;
      }
    }
  }
}
__device__ __forceinline__ bool mbar_wait_cl(uint32_t bar, uint32_t parity, volatile int* abort_flag,
                                             uint32_t peer_abort, int* err, uint64_t wait_ns) {
  return mbar_try_cl(bar, parity) || mbar_wait_cl_slow(bar, parity, abort_flag, peer_abort, err, wait_ns);
}
__device__ __noinline__ void drain_wait_cl(uint32_t bar, uint32_t parity, uint64_t wait_ns) {
  const uint64_t t0 = global_ns();
  while (!mbar_try_cl(bar, parity) && global_ns() - t0 < wait_ns) {
  }
}
// a CTA-pair TMA load into this CTA's shared memory, completing on the
// mbarrier at `mbar` (shared::cluster address, the leader's)
__device__ __forceinline__ void tma_load_2d_pair(uint32_t dst, const CUtensorMap* map, int x, int y, uint32_t mbar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
      "[%4];" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(mbar)
      : "memory");
}
__device__ __forceinline__ void tc_mma_pair(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::2.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(d),
      "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
      : "memory");
}
// arrive on the barrier at this offset in both CTAs once the MMAs issued so far complete
__device__ __forceinline__ void tc_commit_pair_both(uint32_t bar) {
  asm volatile(
      "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64 [%0], %1;" ::"r"(bar),
      "h"((uint16_t)3)
      : "memory");
}
__device__ __forceinline__ void tc_commit_pair_own(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void cluster_sync_all() {
  asm volatile("barrier.cluster.arrive.release;\n\tbarrier.cluster.wait.acquire;" ::: "memory");
}
__host__ __device__ constexpr uint32_t idesc_pair(int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(2 * kUM >> 4) << 24);
}

}  // namespace

__global__ void __launch_bounds__(kThreads, 1)
    k_umma_pair(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmQ, BatchGemm a) {
  extern __shared__ unsigned char umma_raw[];
  unsigned char* sm = umma_raw + ((1024 - (s2u(umma_raw) & 1023)) & 1023);
  const uint32_t base = s2u(sm);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t rank = cluster_rank(), peer = rank ^ 1u;
  const bool leader = rank == 0;
  const uint32_t bar0 = base + kPSmBar;
  auto full_bar = [&](int s) { return bar0 + 8u * s; };
  auto empty_bar = [&](int s) { return bar0 + 8u * (kPStages + s); };
  const uint32_t qfull_bar = bar0 + 8u * (2 * kPStages);
  const uint32_t qempty_bar = qfull_bar + 8;
  auto tfull_bar = [&](int b) { return qempty_bar + 8u + 8u * b; };
  auto tempty_bar = [&](int b) { return qempty_bar + 24u + 8u * b; };
  const uint32_t done_bar = qempty_bar + 40u;
  auto ifull_bar = [&](int sl) { return done_bar + 8u + 8u * sl; };
  auto iempty_bar = [&](int sl) { return done_bar + 24u + 8u * sl; };
  const uint32_t bfull_bar = done_bar + 40u;   // both halves of B_ext written (leader's)
  const uint32_t bempty_bar = done_bar + 48u;  // the item's MMAs have read B_ext (both CTAs)
  volatile uint32_t* s_item = reinterpret_cast<volatile uint32_t*>(sm + kPSmItem);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(sm + kPSmAbort);
  const uint32_t peer_abort = mapa(base + kPSmAbort, peer);
  uint32_t* s_qidx = reinterpret_cast<uint32_t*>(sm + kPSmQidx);
  volatile int* s_okw = reinterpret_cast<volatile int*>(sm + kPSmOkw);

  const uint64_t wns = a.wait_ns ? a.wait_ns : kWaitNs;
  const int nkb = (a.L + kUK - 1) / kUK;  // <= kResidentKB (checked by the launcher)
  const int nq = a.nq_dev ? (int)min((uint32_t)a.nq, *a.nq_dev) : a.nq;
  const bool listed = a.mode == 3;
  const int qtile = a.qtile ? a.qtile : (nq <= 64 ? 64 : (nq <= 128 ? 128 : kUN));
  const uint32_t QT = (uint32_t)((nq + qtile - 1) / qtile);
  const uint64_t ntiles = (a.nrows + kUM - 1) / kUM;
  const uint32_t nchunks = (uint32_t)((ntiles + a.tiles_per_item - 1) / a.tiles_per_item);
  const uint32_t total = listed ? (a.nitems_dev ? min(a.nitems, *a.nitems_dev) : a.nitems) : nchunks * QT;
  auto wait = [&](uint32_t bar, uint32_t parity) {
    return mbar_wait_cl(bar, parity, abort_flag, peer_abort, a.err, wns);
  };

  if (tid == 0) {
    for (int s = 0; s < kPStages; ++s) {
      mbar_init(full_bar(s), 1);
      mbar_init(empty_bar(s), 1);
    }
    mbar_init(qfull_bar, 1);
    mbar_init(qempty_bar, 1);
    for (int b = 0; b < 2; ++b) {
      mbar_init(tfull_bar(b), 1);
      mbar_init(tempty_bar(b), kPEpiArrivals);
    }
    mbar_init(done_bar, 1);
    mbar_init(bfull_bar, 2);  // the epilogue of each CTA
    mbar_init(bempty_bar, 1);
    for (int sl = 0; sl < 2; ++sl) {
      mbar_init(ifull_bar(sl), 1);
      // the leader's MMA lane and, of both CTAs, the epilogue warps; the
      // peer's producer lane
      mbar_init(iempty_bar(sl), 1 + kPEpiArrivals + 1);
    }
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  {
    uint32_t* ae = reinterpret_cast<uint32_t*>(sm + kPSmAext);
    uint32_t* be = reinterpret_cast<uint32_t*>(sm + kPSmBext);
    for (int i = tid; i < (int)(kUM * kExtRow / 4); i += kThreads) ae[i] = 0x3F803F80u;
    for (int i = tid; i < (int)((kUN / 2) * kExtRow / 4); i += kThreads) be[i] = 0u;
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  }
  if (warp == 2) {
    asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], 512;" ::"r"(base + kPSmTmem)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  // both CTAs' barriers are initialised before any remote arrival or copy
  cluster_sync_all();
  tc_fence_after();
  const uint32_t tmem = *reinterpret_cast<volatile uint32_t*>(sm + kPSmTmem);

  // the item's 128-row tiles [t_lo, t_hi) are walked as pair tiles of 256 rows
  auto pair_tiles = [](const Item& it) { return it.t_hi > it.t_lo ? (it.t_hi - it.t_lo + 1) / 2 : 0u; };

  if (warp == 0) {
    // ---------------- TMA producer of this CTA's half
    if (lane == 0) {
      uint32_t g = 0, q_issued = 0;
      uint32_t s_cur = 0, ph = 0;  // stage g % kPStages and the parity of g / kPStages
      bool ok = true;
      const uint32_t lq = mapa(qfull_bar, 0);
      for (uint32_t it_n = 0;; ++it_n) {
        const int sl = (int)(it_n & 1);
        uint32_t w;
        if (leader) {
          ok = wait(iempty_bar(sl), ((it_n >> 1) & 1) ^ 1);
          if (!ok) break;
          const uint32_t v = a.queue ? atomicAdd(a.queue, 1u) : (blockIdx.x >> 1) + it_n * (gridDim.x >> 1);
          w = v < total ? v : kNoItem;
          s_item[sl] = w;
          st_cluster(mapa(base + kPSmItem + 4u * sl, 1), w);
          mbar_arrive(ifull_bar(sl));
          mbar_arrive_cl(mapa(ifull_bar(sl), 1));
        } else {
          ok = wait(ifull_bar(sl), (it_n >> 1) & 1);
          if (!ok) break;
          w = s_item[sl];
          mbar_arrive_cl(mapa(iempty_bar(sl), 0));
        }
        if (w == kNoItem) break;
        const Item it = item_of(a, w, QT, ntiles, qtile, nq);
        const int n = item_n(it.qcnt, qtile);
        ok = wait(qempty_bar, (it_n & 1) ^ 1);
        if (!ok) break;
        if (leader) mbar_expect_tx(qfull_bar, 2u * (uint32_t)nkb * kPQBytes);
        for (int kb = 0; kb < nkb; ++kb)
          tma_load_2d_pair(base + kPSmQ + kb * kPQBytes, &tmQ, kb * kUK, (int)(it.qoff + rank * (uint32_t)(n / 2)), lq);
        ++q_issued;
        const uint32_t np = pair_tiles(it);
        for (uint32_t j = 0; ok && j < np; ++j) {
          const int row0 = (int)(it.rb + (uint64_t)(it.t_lo + 2 * j + rank) * kUM);
          for (int kb = 0; kb < nkb; ++kb, ++g) {
            const int s = (int)s_cur;
            const uint32_t par = ph;
            if (++s_cur == kPStages) {
              s_cur = 0;
              ph ^= 1u;
            }
            ok = wait(empty_bar(s), par ^ 1);
            if (!ok) break;
            if (a.withhold_first_copy && g == 0 && !leader) continue;
            if (leader) mbar_expect_tx(full_bar(s), 2u * kABytes);
            tma_load_2d_pair(base + kPSmA + s * kABytes, &tmA, kb * kUK, row0, mapa(full_bar(s), 0));
          }
        }
        if (!ok) break;
      }
      if (leader && (!ok || a.withhold_first_copy)) {
        // the copies of both CTAs complete on the leader's barriers: wait
        // (bounded) for the stages issued before the CTAs leave
        const uint32_t first = g > kPStages ? g - kPStages : 0;
        for (uint32_t gg = first; gg < g; ++gg) drain_wait_cl(full_bar((int)(gg % kPStages)), (gg / kPStages) & 1, wns);
        if (q_issued > 0) drain_wait_cl(qfull_bar, (q_issued - 1) & 1, wns);
      }
    }
  } else if (warp == 1) {
    // ---------------- MMA issuer (the leader's lane 0)
    if (leader && lane == 0) {
      uint32_t g = 0, tcount = 0;
      uint32_t s_cur = 0, ph = 0;
      const uint64_t dae = sw32_desc(base + kPSmAext), dbe = sw32_desc(base + kPSmBext);
      bool ok = true;
      for (uint32_t it_n = 0; ok; ++it_n) {
        const int sl = (int)(it_n & 1);
        ok = wait(ifull_bar(sl), (it_n >> 1) & 1);
        if (!ok) break;
        const uint32_t w = s_item[sl];
        mbar_arrive(iempty_bar(sl));
        if (w == kNoItem) break;
        const Item it = item_of(a, w, QT, ntiles, qtile, nq);
        ok = wait(qfull_bar, it_n & 1);
        if (!ok) break;
        tc_fence_after();
        ok = wait(bfull_bar, it_n & 1);
        if (!ok) break;
        tc_fence_after();
        const uint32_t idesc = idesc_pair(item_n(it.qcnt, qtile));
        const uint32_t np = pair_tiles(it);
        for (uint32_t j = 0; ok && j < np; ++j, ++tcount) {
          const int b = (int)(tcount & 1);
          ok = wait(tempty_bar(b), ((tcount >> 1) & 1) ^ 1);
          if (!ok) break;
          tc_fence_after();
          const uint32_t d = tmem + (uint32_t)b * kUN;
          // the accumulator starts as -(t_hi + t_lo) of its column
          tc_mma_pair(d, dae, dbe, idesc, 0u);
          for (int kb = 0; kb < nkb; ++kb, ++g) {
            const int s = (int)s_cur;
            const uint32_t par = ph;
            if (++s_cur == kPStages) {
              s_cur = 0;
              ph ^= 1u;
            }
            ok = wait(full_bar(s), par);
            if (!ok) break;
            tc_fence_after();
            const uint64_t da = sw128_desc(base + kPSmA + s * kABytes);
            const uint64_t dq = sw128_desc(base + kPSmQ + kb * kPQBytes);
#pragma unroll
            for (int k16 = 0; k16 < kUK / 16; ++k16) tc_mma_pair(d, da + 2 * k16, dq + 2 * k16, idesc, 1u);
            tc_commit_pair_both(empty_bar(s));
          }
          if (ok) tc_commit_pair_both(tfull_bar(b));
        }
        if (ok) {
          tc_commit_pair_both(qempty_bar);
          tc_commit_pair_both(bempty_bar);
        }
      }
      // every MMA issued has completed before either CTA frees its TMEM
      tc_commit_pair_own(done_bar);
      drain_wait_cl(done_bar, 0, wns);
    }
  } else if (warp >= 4) {
    // ---------------- epilogue of this CTA's 128 rows
    const int etid = tid - 128;
    const int ew = warp - 4;
    const int quarter = warp & 3;
    const int half = ew >> 2;
    const float inf = __int_as_float(0x7f800000);
    const uint32_t l_bfull = mapa(bfull_bar, 0);
    uint32_t tcount = 0;
    uint32_t pcur = 0, pend = 0;
    bool ok = true;
    float e_sum = 0.0f, e_rel = 0.0f, e_max = 0.0f;
    uint32_t e_cnt = 0, e_rcnt = 0;
    for (uint32_t it_n = 0;; ++it_n) {
      const int sl = (int)(it_n & 1);
      uint32_t w = kNoItem;
      int got = 1;
      if (lane == 0) {
        got = wait(ifull_bar(sl), (it_n >> 1) & 1) ? 1 : 0;
        if (got) {
          w = s_item[sl];
          if (leader) mbar_arrive(iempty_bar(sl));
          else mbar_arrive_cl(mapa(iempty_bar(sl), 0));
        }
      }
      got = __shfl_sync(HG_FULL, got, 0);
      w = __shfl_sync(HG_FULL, w, 0);
      ok = ok && got;
      if (lane == 0) s_okw[ew] = ok ? 1 : 0;
      named_sync(1, kEpiThreads);
      bool all_ok = true;
#pragma unroll
      for (int i = 0; i < kEpiThreads / 32; ++i) all_ok = all_ok && s_okw[i] != 0;
      if (!all_ok || w == kNoItem) break;
      const Item it = item_of(a, w, QT, ntiles, qtile, nq);
      const int n = item_n(it.qcnt, qtile);
      // column etid of the item's query tile
      uint32_t q = 0xffffffffu;
      float4 qm = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
      float qb = -1.0f;
      if ((uint32_t)etid < it.qcnt) {
        q = a.qperm[it.qoff + etid];
        qm = a.qmeta[q];
        const float b = a.bound[q];
        qb = b < inf ? b : -1.0f;
      }
      s_qidx[etid] = q;
      // this CTA holds columns [rank n / 2, rank n / 2 + n / 2) of B_ext
      const int col0 = (int)rank * (n / 2);
      const bool mine = etid >= col0 && etid < col0 + n / 2;
      float4 tm = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
      for (uint32_t t = it.t_lo + lane; t < it.t_hi; t += 32) {
        const float4 v = a.tile_meta[(it.rb + (uint64_t)t * kUM) / kUM];
        tm.x = fmaxf(tm.x, v.x);
        tm.y = fmaxf(tm.y, v.y);
        tm.z = fmaxf(tm.z, v.z);
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        tm.x = fmaxf(tm.x, __shfl_xor_sync(HG_FULL, tm.x, o));
        tm.y = fmaxf(tm.y, __shfl_xor_sync(HG_FULL, tm.y, o));
        tm.z = fmaxf(tm.z, __shfl_xor_sync(HG_FULL, tm.z, o));
      }
      float tv = inf;
      if (qb >= 0.0f) {
        const float err = 2.000002f * (qm.y * tm.z + qm.z * tm.y + qm.z * tm.z + a.c_acc * qm.y * tm.y) +
                          a.c_sq * (qm.x + tm.x + qb) + 1e-5f;
        tv = 0.5f * (qm.x - qb - err);
        if (a.errstat && mine) {
          e_sum += err;
          e_max = fmaxf(e_max, err);
          ++e_cnt;
          if (qb > 0.0f) {
            e_rel += err / qb;
            ++e_rcnt;
          }
        }
      }
      // the split's and the accumulation's rounding, with room to spare (as
      // in k_umma_filter)
      if (tv < inf) tv -= a.c_acc * fabsf(tv) + 6.103515625e-05f * (fabsf(tv) + qm.y * tm.y);
      // B_ext may be rewritten once the previous item's MMAs have read it
      if (ew == 0 && it_n > 0) {
        int okb = 1;
        if (lane == 0) okb = wait(bempty_bar, (it_n - 1) & 1) ? 1 : 0;
        okb = __shfl_sync(HG_FULL, okb, 0);
        ok = ok && okb;
      }
      named_sync(1, kEpiThreads);
      if (mine) {
        float th = tv, tl = 0.0f;
        if (tv < inf) {
          th = __bfloat162float(__float2bfloat16_rn(tv));
          tl = tv - th;
        }
        const uint32_t row = (uint32_t)(etid - col0);
        *reinterpret_cast<uint32_t*>(sm + kPSmBext + row * kExtRow + (((row >> 2) & 1u) << 4)) =
            bf16_bits(-th) | (bf16_bits(-tl) << 16);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      }
      named_sync(1, kEpiThreads);
      if (etid == 0) mbar_arrive_cl(l_bfull);
      const int half_cols = min(qtile / 2, (int)((it.qcnt + 63u) / 64u) * 32);
      const int c_lo = half * half_cols;
      const int c_hi = min(c_lo + half_cols, (int)it.qcnt);
      const uint32_t np = pair_tiles(it);
      auto row_of = [&](uint32_t j) {
        return it.rb + (uint64_t)(it.t_lo + 2 * j + rank) * kUM + quarter * 32 + lane;
      };
      auto valid = [&](uint32_t j, uint64_t rw) {
        return it.t_lo + 2 * j + rank < it.t_hi && rw >= it.vb && rw < it.re && rw < a.nrows;
      };
      float xn_next = 0.0f;
      auto prefetch = [&](uint32_t j) {
        if (j >= np) return;
        const uint64_t rw = row_of(j);
        xn_next = valid(j, rw) ? a.xmeta[rw].x : 0.0f;
      };
      prefetch(0);
      for (uint32_t j = 0; ok && j < np; ++j, ++tcount) {
        const int b = (int)(tcount & 1);
        const uint64_t row = row_of(j);
        const bool row_ok = valid(j, row);
        const float xn2 = xn_next;
        prefetch(j + 1);
        const float h_row = row_ok ? 0.5f * xn2 : inf;
        int go = 0;
        if (lane == 0) go = wait(tfull_bar(b), (tcount >> 1) & 1) ? 1 : 0;
        go = __shfl_sync(HG_FULL, go, 0);
        if (!go) {
          ok = false;
          break;
        }
        tc_fence_after();
        const uint32_t tbase = tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)b * kUN;
        uint32_t masks[4] = {0u, 0u, 0u, 0u};
#pragma unroll
        for (int i2 = 0; i2 < 2; ++i2) {
          const int c0 = c_lo + 64 * i2;
          if (c0 >= c_hi) break;
          uint32_t r[2][32];
          tc_ld32(tbase + (uint32_t)c0, r[0]);
          tc_ld32(tbase + (uint32_t)(c0 + 32), r[1]);
          tc_wait_ld();
#pragma unroll
          for (int hh = 0; hh < 2; ++hh) {
            const int cb = c0 + 32 * hh;
            if (cb >= c_hi) break;
            masks[2 * i2 + hh] = screen32(reinterpret_cast<const float*>(r[hh]), h_row, c_hi - cb);
          }
        }
        tc_fence_before();
        __syncwarp();
        if (lane == 0) {
          if (leader) mbar_arrive(tempty_bar(b));
          else mbar_arrive_cl(mapa(tempty_bar(b), 0));
        }
#pragma unroll
        for (int ci = 0; ci < 4; ++ci) {
          uint32_t mask = masks[ci];
          while (__any_sync(HG_FULL, mask != 0)) {
            const bool has = mask != 0;
            unsigned long long e = 0;
            if (has) {
              const int jj = __ffs(mask) - 1;
              mask &= mask - 1;
              e = ((unsigned long long)s_qidx[c_lo + 32 * ci + jj] << 32) | (uint32_t)row;
            }
            const uint32_t bal = __ballot_sync(HG_FULL, has);
            const uint32_t cnt = (uint32_t)__popc(bal);
            if (pcur + cnt > pend) {
              for (uint32_t i = pcur + lane; i < pend; i += 32) a.pairs[i] = ~0ull;
              uint32_t nb = 0;
              if (lane == 0) nb = atomicAdd(a.pairs_cnt, (uint32_t)kPairBlock);
              nb = __shfl_sync(HG_FULL, nb, 0);
              pcur = nb;
              pend = nb + kPairBlock < a.pairs_cap ? nb + kPairBlock : (nb < a.pairs_cap ? a.pairs_cap : nb);
            }
            const uint32_t slot = pcur + (uint32_t)__popc(bal & ((1u << lane) - 1));
            if (has && slot < pend) a.pairs[slot] = e;
            pcur += cnt;
          }
        }
      }
    }
    for (uint32_t i = pcur + lane; i < pend; i += 32) a.pairs[i] = ~0ull;
    if (a.errstat) {
      double ds = e_sum, dr = e_rel;
      uint32_t c = e_cnt, rc = e_rcnt;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        ds += __shfl_xor_sync(HG_FULL, ds, o);
        dr += __shfl_xor_sync(HG_FULL, dr, o);
        c += __shfl_xor_sync(HG_FULL, c, o);
        rc += __shfl_xor_sync(HG_FULL, rc, o);
        e_max = fmaxf(e_max, __shfl_xor_sync(HG_FULL, e_max, o));
      }
      if (lane == 0 && c) {
        atomicAdd(&a.errstat[0], ds);
        atomicAdd(&a.errstat[1], dr);
        atomicAdd(&a.errstat[2], (double)c);
        atomicAdd(&a.errstat[3], (double)rc);
        atomicMax(reinterpret_cast<unsigned long long*>(&a.errstat[4]),
                  (unsigned long long)__double_as_longlong((double)e_max));
      }
    }
  }
  // no CTA of the pair leaves (or frees TMEM) while the other may still
  // signal its barriers or the MMAs may still write its TMEM
  tc_fence_before();
  cluster_sync_all();
  if (warp == 2) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, 512;" ::"r"(tmem) : "memory");
  }
}

size_t umma_pair_smem() { return kPDynSmem; }

cudaError_t launch_umma_pair(const CUtensorMap& rows_map, const CUtensorMap& q_half_map, const BatchGemm& g,
                             int blocks, cudaStream_t s) {
  if (g.mode != 1 && g.mode != 3) return cudaErrorInvalidValue;
  if ((g.L + kUK - 1) / kUK > kResidentKB) return cudaErrorInvalidValue;
  if (g.qtile != 0 && g.qtile != 64 && g.qtile != 128 && g.qtile != 256) return cudaErrorInvalidValue;
  static SmemLimit attr;
  const cudaError_t ea = attr.ensure((const void*)k_umma_pair, (int)kPDynSmem);
  if (ea != cudaSuccess) return ea;
  int grid = blocks & ~1;
  if (!(g.mode == 3 ? g.nitems_dev : g.nq_dev)) {
    const uint64_t ntiles = (g.nrows + kUM - 1) / kUM;
    const int qtile = g.qtile ? g.qtile : (g.nq <= 64 ? 64 : (g.nq <= 128 ? 128 : kUN));
    const uint32_t QT = (uint32_t)((g.nq + qtile - 1) / qtile);
    const uint64_t total = g.mode == 3 ? g.nitems : ((ntiles + g.tiles_per_item - 1) / g.tiles_per_item) * (uint64_t)QT;
    if (total == 0) return cudaSuccess;
    if (2 * total < (uint64_t)grid) grid = (int)(2 * total);
  }
  if (grid < 2) return cudaErrorInvalidValue;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)grid, 1, 1);
  cfg.blockDim = dim3(kThreads, 1, 1);
  cfg.dynamicSmemBytes = kPDynSmem;
  cfg.stream = s;
  cudaLaunchAttribute attr2[1];
  attr2[0].id = cudaLaunchAttributeClusterDimension;
  attr2[0].val.clusterDim.x = 2;
  attr2[0].val.clusterDim.y = 1;
  attr2[0].val.clusterDim.z = 1;
  cfg.attrs = attr2;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, k_umma_pair, rows_map, q_half_map, g);
}

size_t umma_filter_smem() { return FilterLayout<false>::kDyn; }

template <bool kScreen, bool kResident, bool kBound>
static cudaError_t launch_filter_instance(const CUtensorMap& rows_map, const CUtensorMap& q_map, const BatchGemm& g,
                                          int grid, cudaStream_t s) {
  constexpr int smem = (int)FilterLayout<kBound>::kDyn;
  static SmemLimit attr;
  const cudaError_t ea = attr.ensure((const void*)k_umma_filter<kScreen, kResident, kBound>, smem);
  if (ea != cudaSuccess) return ea;
  k_umma_filter<kScreen, kResident, kBound><<<grid, kThreads, smem, s>>>(rows_map, q_map, g);
  return cudaGetLastError();
}

cudaError_t launch_umma_filter(const CUtensorMap& rows_map, const CUtensorMap& q_map, const BatchGemm& g, int blocks,
                               cudaStream_t s) {
  const uint64_t ntiles = (g.nrows + kUM - 1) / kUM;
  if (g.mode != 0 && g.qtile != 0 && g.qtile != 64 && g.qtile != 128 && g.qtile != 256) return cudaErrorInvalidValue;
  // counts read on the device: every CTA starts and leaves when out of items
  int grid = blocks;
  const bool listed = g.mode == 0 || g.mode == 3;
  if (!(listed ? g.nitems_dev : g.nq_dev)) {
    const int qtile = g.mode == 0 ? kBatchBoundQueries : (g.qtile ? g.qtile : (g.nq <= 64 ? 64 : (g.nq <= 128 ? 128 : kUN)));
    const uint32_t QT = (uint32_t)((g.nq + qtile - 1) / qtile);
    const uint64_t total =
        listed ? g.nitems : ((ntiles + g.tiles_per_item - 1) / g.tiles_per_item) * (uint64_t)QT;
    if (total == 0) return cudaSuccess;
    grid = (int)(total < (uint64_t)blocks ? total : (uint64_t)blocks);
  }
  const bool screen = g.mode == 1 || g.mode == 3;
  const bool resident = (g.L + kUK - 1) / kUK <= kResidentKB;
  if (screen) {
    return resident ? launch_filter_instance<true, true, false>(rows_map, q_map, g, grid, s)
                    : launch_filter_instance<true, false, false>(rows_map, q_map, g, grid, s);
  }
  // the bound pass with a resident query tile: q_map has 64-query boxes
  if (g.mode == 0 && resident) return launch_filter_instance<false, true, true>(rows_map, q_map, g, grid, s);
  return resident ? launch_filter_instance<false, true, false>(rows_map, q_map, g, grid, s)
                  : launch_filter_instance<false, false, false>(rows_map, q_map, g, grid, s);
}

}  // namespace hg
