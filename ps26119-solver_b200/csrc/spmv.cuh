// spmv.cuh — CSR row-slab SpMV with fused epilogues: the per-iteration hot path.
//
// One thread block owns a slab of kSlabRows consecutive rows. The slab's row pointers and
// its contiguous nonzero range (col, val) are staged into shared memory with coalesced loads
// (tiles of kSlabTile nonzeros), then each thread accumulates ITS row sequentially in CSR
// order in fp64, exactly as the reference's Csr::multiply<double> (src/la/csr.h:30-43):
//     s = 0; for k in row: s += double(val[k]) * double(x[col[k]]);   out = T(s)
// The gathers of x are issued in batches of 4 independent loads before the ordered adds.
// The epilogue functor receives (row, s) and performs the rest of the fused update in
// registers, so the SpMV output never round-trips through HBM.
//
// Roofline: HBM-bound. Per nonzero: val (s_v bytes) + col (4 bytes) streamed once, plus
// 4 bytes of row pointer per row and the epilogue's vectors; x gathers hit L2 when x fits.
#pragma once

#include <algorithm>
#include <cstddef>
#include <cstdint>
#include <type_traits>
#include <vector>

#include "common.cuh"

namespace b200 {

// Build-time tuning knobs (defaults are the tuned values): CTAs per SM the register budget is
// sized for, whether the engine's own CSR arrays are staged by TMA bulk copies, and the
// shared-memory carveout preference (percent, or -1 to leave the driver default).
#ifndef B200_SLAB_MIN_BLOCKS
#define B200_SLAB_MIN_BLOCKS 4
#endif
#ifndef B200_STAGE_TMA
#define B200_STAGE_TMA 1
#endif
#ifndef B200_SLAB_CARVEOUT
#define B200_SLAB_CARVEOUT -1
#endif
// 1: the staged CSR tiles (read once per iteration) are loaded with an L2 evict-first policy, so
// they do not push the gathered vector out of L2.
#ifndef B200_TMA_EVICT_FIRST
#define B200_TMA_EVICT_FIRST 1
#endif
// 1: the iteration kernels read each slab's nonzero range [k0, k1) from a small precomputed
// table kept in L2 (evict-last), instead of from the row pointers: the first load of a block
// is then an L2 hit, not a DRAM round trip, and the tile copy starts sooner.
#ifndef B200_SLAB_TABLE
#define B200_SLAB_TABLE 0
#endif
// 1: the iteration epilogues load their streamed operands evict-first and store the vector the
// next kernel gathers (x̄, y) evict-last, so that it is still in L2 when the gathers come.
#ifndef B200_EPI_HINTS
#define B200_EPI_HINTS 1
#endif

// 1: the iteration kernels stage their epilogue operands and row pointers by TMA as well
// (k_slab_fed); 0: they use k_slab.
#ifndef B200_SLAB_FED
#define B200_SLAB_FED 1
#endif

#ifndef B200_SLAB_ROWS
#define B200_SLAB_ROWS 256
#endif
#ifndef B200_GATHER_BATCH
#define B200_GATHER_BATCH 4
#endif

constexpr int kSlabRows = B200_SLAB_ROWS;  // rows per slab = threads per block
constexpr int kSlabTile = 2048;  // nonzeros staged per tile
constexpr int kTilePad = 8;      // room for the 16-byte widening of a bulk copy

template <class T>
struct SlabSmem {
  alignas(16) int col[kSlabTile + kTilePad];
  alignas(16) T val[kSlabTile + kTilePad];
  alignas(8) unsigned long long bar;
};

// Bulk-copy waits that ran out (never expected to move). Each launch counts into the counter it is
// given (a solve passes its own, so a timeout is reported by the solve it happened in); launches
// given none count into this process-wide one.
static __device__ unsigned int g_stage_timeouts;
__device__ __forceinline__ void count_stage_timeout(unsigned* err) { atomicAdd(err ? err : &g_stage_timeouts, 1u); }

// Programmatic dependent launch (sm_90+): a kernel launched with the programmatic-serialisation
// attribute may start while the kernel before it in the stream is still running; it must not
// touch that kernel's outputs (or anything a kernel still running may read or write) before
// pdl_wait(), which returns once every earlier kernel has completed and its writes are visible.
// pdl_allow_next() lets the next such kernel be scheduled once every block of this one has issued
// it. In a kernel launched without the attribute both are no-ops.
__device__ __forceinline__ void pdl_allow_next() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

__device__ __forceinline__ unsigned smem_u32(const void* p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(unsigned long long* bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
// One TMA bulk copy global -> this CTA's shared memory (no multicast); both addresses and the
// size are multiples of 16 bytes.
__device__ __forceinline__ void tma_load_1d(void* dst, const void* src, unsigned bytes, unsigned long long* bar) {
#if B200_TMA_EVICT_FIRST
  unsigned long long policy;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(policy));
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar)), "l"(policy)
      : "memory");
#else
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
#endif
}
// A bulk prefetch of [src, src + bytes) into L2 (no shared memory, no completion to wait for);
// src 16-byte aligned, bytes a multiple of 16.
__device__ __forceinline__ void prefetch_l2(const void* src, unsigned bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Waits for phase `parity` of the barrier, at most ~2^22 try_wait rounds.
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long* bar, unsigned parity) {
  for (int it = 0; it < (1 << 22); ++it)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

// L2-policy loads and stores (createpolicy + .L2::cache_hint).
__device__ __forceinline__ unsigned long long l2_policy_last() {
  unsigned long long p;
  asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ unsigned long long l2_policy_first() {
  unsigned long long p;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ int2 ld_keep(const int2* p) {
  int2 v;
  asm volatile("ld.global.L2::cache_hint.v2.s32 {%0, %1}, [%2], %3;" : "=r"(v.x), "=r"(v.y) : "l"(p), "l"(l2_policy_last()));
  return v;
}
template <class T>
__device__ __forceinline__ T ld_stream(const T* p) {
#if B200_EPI_HINTS
  if constexpr (sizeof(T) == 8) {
    double v;
    asm volatile("ld.global.L2::cache_hint.f64 %0, [%1], %2;" : "=d"(v) : "l"(p), "l"(l2_policy_first()));
    return static_cast<T>(v);
  } else {
    float v;
    asm volatile("ld.global.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(p), "l"(l2_policy_first()));
    return static_cast<T>(v);
  }
#else
  return *p;
#endif
}
template <class T>
__device__ __forceinline__ void st_keep(T* p, T v) {
#if B200_EPI_HINTS
  if constexpr (sizeof(T) == 8)
    asm volatile("st.global.L2::cache_hint.f64 [%0], %1, %2;" ::"l"(p), "d"(static_cast<double>(v)), "l"(l2_policy_last())
                 : "memory");
  else
    asm volatile("st.global.L2::cache_hint.f32 [%0], %1, %2;" ::"l"(p), "f"(static_cast<float>(v)), "l"(l2_policy_last())
                 : "memory");
#else
  *p = v;
#endif
}

// The gathered operand x[col] of the row products. B200_GATHER_NA=1 loads it with
// L1::no_allocate (the gathers have almost no L1 reuse).
#ifndef B200_GATHER_NA
#define B200_GATHER_NA 1
#endif
template <class T>
__device__ __forceinline__ double gather(const T* __restrict__ x, int i) {
#if B200_GATHER_NA
  if constexpr (sizeof(T) == 8) {
    double v;
    asm volatile("ld.global.nc.L1::no_allocate.f64 %0, [%1];" : "=d"(v) : "l"(x + i));
    return v;
  } else {
    float v;
    asm volatile("ld.global.nc.L1::no_allocate.f32 %0, [%1];" : "=f"(v) : "l"(x + i));
    return static_cast<double>(v);
  }
#else
  return static_cast<double>(x[i]);
#endif
}

// Epilogues may prefetch their operands: `Pre load(int row)` is issued at kernel entry, before
// the nonzeros are staged, so its latency overlaps the SpMV; `operator()(row, s, pre)` then
// finishes the update. Epilogues that take maxima expose `Acc` (fields written by the
// epilogue) and `flush(acc)`, called by every thread after the epilogue so that maxima are
// combined per warp before one atomic (see warp_max_atomic).
struct NoPre {};
struct NoAcc {};
template <class E>
__device__ __forceinline__ auto epi_load(const E& e, int i, int) -> decltype(e.load(i)) {
  return e.load(i);
}
template <class E>
__device__ __forceinline__ NoPre epi_load(const E&, int, long) {
  return NoPre{};
}
template <class E>
__device__ __forceinline__ auto epi_acc(const E&, int) -> typename E::Acc {
  return typename E::Acc{};
}
template <class E>
__device__ __forceinline__ NoAcc epi_acc(const E&, long) {
  return NoAcc{};
}
template <class E, class P, class A>
__device__ __forceinline__ void epi_apply(const E& e, int i, double s, const P& p, A& acc) {
  if constexpr (!std::is_same<A, NoAcc>::value) e(i, s, acc);
  else if constexpr (std::is_same<P, NoPre>::value) e(i, s);
  else e(i, s, p);
}
template <class E, class A>
__device__ __forceinline__ void epi_flush(const E& e, const A& acc) {
  if constexpr (!std::is_same<A, NoAcc>::value) e.flush(acc);
}

// gather() without the conversion to double.
template <class T>
__device__ __forceinline__ T gather_t(const T* __restrict__ x, int i) {
#if B200_GATHER_NA
  if constexpr (sizeof(T) == 8) {
    double v;
    asm volatile("ld.global.nc.L1::no_allocate.f64 %0, [%1];" : "=d"(v) : "l"(x + i));
    return v;
  } else {
    float v;
    asm volatile("ld.global.nc.L1::no_allocate.f32 %0, [%1];" : "=f"(v) : "l"(x + i));
    return v;
  }
#else
  return x[i];
#endif
}

constexpr int kGatherBatch = B200_GATHER_BATCH;  // independent x-gathers issued per round trip

// Row-sequential fp64 accumulation of `rows` CSR rows; calls the epilogue with (row, s).
// kTma: the tiles of col/val are staged by TMA bulk copies (the arrays must be this library's
// own allocations, whose 64-byte tail padding covers the 16-byte widening); otherwise by a
// batched register copy (caller-owned arrays). epi.active() lets graph-replayed launches exit.
template <class T, class Epi, bool kTma>
__global__ void __launch_bounds__(kSlabRows, B200_SLAB_MIN_BLOCKS) k_slab(int rows, const int* __restrict__ rp,
                                                        const int* __restrict__ col,
                                                        const T* __restrict__ val,
                                                        const T* __restrict__ x, Epi epi,
                                                        const int2* __restrict__ slab, unsigned* err) {
  __shared__ SlabSmem<T> sm;
  if (!epi.active()) return;
  const int r0 = blockIdx.x * kSlabRows;
  const int nr = min(kSlabRows, rows - r0);
  const bool mine = threadIdx.x < nr;
  const int row = r0 + static_cast<int>(threadIdx.x);
  // independent loads first: the slab's nonzero range, this thread's row bounds, the epilogue
  int k0, k1;
  if (slab) {
    const int2 kr = ld_keep(slab + blockIdx.x);
    k0 = kr.x, k1 = kr.y;
  } else {
    k0 = __ldg(rp + r0), k1 = __ldg(rp + r0 + nr);
  }
  const int beg = mine ? __ldg(rp + row) : 0, end = mine ? __ldg(rp + row + 1) : 0;
  const auto pre = epi_load(epi, mine ? row : r0, 0);
  auto acc = epi_acc(epi, 0);
  if constexpr (kTma) {
    if (threadIdx.x == 0) mbar_init(&sm.bar);
    __syncthreads();
  }
  constexpr int kValAlign = 16 / static_cast<int>(sizeof(T));  // elements per 16 bytes
  unsigned phase = 0;
  double s = 0.0;
  bool staged = true;
  for (int t0 = k0; t0 < k1; t0 += kSlabTile) {
    const int t1 = min(t0 + kSlabTile, k1);
    int c0 = t0, v0 = t0;  // first element held in sm.col / sm.val
    if (t0 != k0) __syncthreads();  // previous tile fully consumed
    if constexpr (kTma) {
      c0 = t0 & ~3;
      v0 = t0 & ~(kValAlign - 1);
      const int c1 = (t1 + 3) & ~3, v1 = (t1 + kValAlign - 1) & ~(kValAlign - 1);
      if (threadIdx.x == 0) {
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        const unsigned cb = static_cast<unsigned>(c1 - c0) * 4u, vb = static_cast<unsigned>(v1 - v0) * sizeof(T);
        mbar_expect_tx(&sm.bar, cb + vb);
        tma_load_1d(sm.col, col + c0, cb, &sm.bar);
        tma_load_1d(sm.val, val + v0, vb, &sm.bar);
      }
      // thread 0 waits; the others sleep in the barrier instead of spinning on the barrier word
      const int ok = threadIdx.x == 0 ? (mbar_wait_bounded(&sm.bar, phase) ? 1 : 0) : 1;
      phase ^= 1u;
      if (!__syncthreads_and(ok)) {  // never expected: record, drain, give up on the tile
        if (threadIdx.x == 0) {
          count_stage_timeout(err);
          mbar_wait_bounded(&sm.bar, phase ^ 1u);
        }
        staged = false;
        break;
      }
    } else {
      constexpr int kB = 4;
      for (int base = t0 + static_cast<int>(threadIdx.x); base < t1; base += kB * kSlabRows) {
        int cc[kB];
        T vv[kB];
#pragma unroll
        for (int q = 0; q < kB; ++q) {
          const int k = base + q * kSlabRows;
          if (k < t1) cc[q] = __ldg(col + k), vv[q] = __ldg(val + k);
        }
#pragma unroll
        for (int q = 0; q < kB; ++q) {
          const int k = base + q * kSlabRows;
          if (k < t1) sm.col[k - t0] = cc[q], sm.val[k - t0] = vv[q];
        }
      }
      __syncthreads();
    }
    const int a = max(beg, t0), b = min(end, t1);
    for (int k = a; k < b; k += kGatherBatch) {
      double p[kGatherBatch];
#pragma unroll
      for (int q = 0; q < kGatherBatch; ++q)
        p[q] = (k + q < b) ? static_cast<double>(sm.val[k + q - v0]) * static_cast<double>(x[sm.col[k + q - c0]])
                           : 0.0;
#pragma unroll
      for (int q = 0; q < kGatherBatch; ++q)
        if (k + q < b) s += p[q];  // in CSR order
    }
  }
  if (!staged) s = __longlong_as_double(0x7ff8000000000000LL);  // NaN: the check reports a numerical error
  if (mine) epi_apply(epi, row, s, pre, acc);
  epi_flush(epi, acc);
}

// ---------------------------------------------------------------------- fully staged form
// k_slab_fed: the row products and epilogue of k_slab, with every streamed operand of the slab
// brought in by TMA bulk copies issued at block entry: the slab's row pointers and the
// epilogue's per-row operand vectors (Epi::vec(k), rows r0 … r0+nr), and the col/val tile.
// Threads hold no operand registers while the gathers are in flight (lower register use), and
// the start of a slab waits on one DRAM round trip (the copies, all issued together) instead of
// a chain of them. The slab's nonzero range comes from the L2-resident slab table. Sums are
// k_slab's sequential CSR-order sums.
//
// Launched back to back with programmatic dependent launch (the iteration kernels of an epoch),
// a block may start while the previous kernel's last blocks still run. Everything that no kernel
// of the epoch writes — the matrix, the row pointers, the slab table and the epilogue vectors
// outside Epi::kLiveVecs (bit k: vec(k) is written by the iteration kernels) — is requested
// before pdl_wait(); the live vectors and the gathered x are touched only after it, and so is
// every store. Without the launch attribute pdl_wait() returns at once.
//
// The tile capacity `cap` is chosen per matrix (the largest slab, rounded up; see
// fed_tile_capacity) and the shared memory is sized to it: the gathers' outstanding L1 misses
// need L1 capacity, which shared memory takes away. A slab with more than `cap` nonzeros is
// summed in several tiles. Only thread 0 waits on the barriers; the other threads sleep in
// __syncthreads instead of spinning on the shared-memory barrier word.
// Requirements (checked on the host): rp, col, val and every Epi::vec(k) are this library's
// 16-byte-aligned, tail-padded allocations.
struct FedLayout {
  unsigned rp, vec, col, val, bytes;  // byte offsets into the dynamic shared memory, and its size
};
// bar[3] (24 bytes) and the slab's nonzero range (8 bytes) come first.
__host__ __device__ constexpr FedLayout fed_layout(int vecs, int elem, int cap) {
  const unsigned rp = 32u;
  const unsigned vec = rp + static_cast<unsigned>(kSlabRows + kTilePad) * 4u;
  const unsigned col = vec + static_cast<unsigned>(vecs * kSlabRows * elem);
  const unsigned val = col + static_cast<unsigned>(cap + kTilePad) * 4u;
  const unsigned bytes = val + static_cast<unsigned>((cap + kTilePad) * elem);
  return FedLayout{rp, vec, col, val, bytes};
}
// Tile capacity for a matrix whose largest slab has `max_slab_nnz` nonzeros: a multiple of 16,
// at least 16, at most kSlabTile.
inline int fed_tile_capacity(long long max_slab_nnz) {
  const long long c = (std::max(16LL, max_slab_nnz) + 15) / 16 * 16;
  return static_cast<int>(std::min<long long>(c, kSlabTile));
}

#ifndef B200_FED_MIN_BLOCKS
#define B200_FED_MIN_BLOCKS 5
#endif

// The fp64 product of staged nonzero k, written over the staged tile once its col and val are
// read: in the val slot for fp64 values; for fp32 values its high word in the col slot and its low
// word in the val slot (k's 8 bytes of tile), so the tile needs no extra room.
template <class T>
__device__ __forceinline__ void put_product(int* s_col, T* s_val, int ic, int iv, double p) {
  if constexpr (sizeof(T) == 8) {
    s_val[iv] = p;
  } else {
    s_col[ic] = __double2hiint(p);
    reinterpret_cast<int*>(s_val)[iv] = __double2loint(p);
  }
}
template <class T>
__device__ __forceinline__ double get_product(const int* s_col, const T* s_val, int ic, int iv) {
  if constexpr (sizeof(T) == 8) return static_cast<double>(s_val[iv]);
  else return __hiloint2double(s_col[ic], reinterpret_cast<const int*>(s_val)[iv]);
}

// The body of k_slab_fed for slab `blk` (the block's slab: blockIdx.x in k_slab_fed, a slab of
// one LP's matrix in the grouped kernel of several LPs).
template <class T, class Epi, int GB>
__device__ __forceinline__ void slab_fed_body(int blk, int rows, const int* __restrict__ rp, const int* __restrict__ col,
                                              const T* __restrict__ val, const T* __restrict__ x, const Epi& epi,
                                              const int2* __restrict__ slab, int cap, unsigned* err,
                                              int ahead = 0) {
  constexpr int V = Epi::kVecs;
  constexpr unsigned kLive = Epi::kLiveVecs;
  constexpr int kNumLive = __builtin_popcount(kLive);
  constexpr int kValAlign = 16 / static_cast<int>(sizeof(T));
  extern __shared__ __align__(16) unsigned char fed_smem[];
  pdl_allow_next();
  if (!epi.active()) return;
  const FedLayout L = fed_layout(V, static_cast<int>(sizeof(T)), cap);
  // [0] row pointers + constant vectors, [1] tile, [2] live vectors (after pdl_wait)
  unsigned long long* bar = reinterpret_cast<unsigned long long*>(fed_smem);
  int2* krange = reinterpret_cast<int2*>(fed_smem + 24);
  int* s_rp = reinterpret_cast<int*>(fed_smem + L.rp);
  T* s_vec = reinterpret_cast<T*>(fed_smem + L.vec);
  int* s_col = reinterpret_cast<int*>(fed_smem + L.col);
  T* s_val = reinterpret_cast<T*>(fed_smem + L.val);
  const int tid = static_cast<int>(threadIdx.x);
  const int r0 = blk * kSlabRows;
  const int nr = min(kSlabRows, rows - r0);
  const unsigned vb = (static_cast<unsigned>(nr) * sizeof(T) + 15u) & ~15u;
  auto issue_tile = [&](int t0, int t1) {  // thread 0
    const int c0 = t0 & ~3, v0 = t0 & ~(kValAlign - 1);
    const int c1 = (t1 + 3) & ~3, v1 = (t1 + kValAlign - 1) & ~(kValAlign - 1);
    const unsigned cb = static_cast<unsigned>(c1 - c0) * 4u, tb = static_cast<unsigned>(v1 - v0) * sizeof(T);
    mbar_expect_tx(&bar[1], cb + tb);
    tma_load_1d(s_col, col + c0, cb, &bar[1]);
    tma_load_1d(s_val, val + v0, tb, &bar[1]);
  };
  bool tile_pending = false;  // thread 0: a tile copy not yet waited for
  if (tid == 0) {
    mbar_init(&bar[0]);
    mbar_init(&bar[1]);
    mbar_init(&bar[2]);
    const unsigned rb = (static_cast<unsigned>(nr + 1) * 4u + 15u) & ~15u;
    mbar_expect_tx(&bar[0], rb + static_cast<unsigned>(V - kNumLive) * vb);
    tma_load_1d(s_rp, rp + r0, rb, &bar[0]);
#pragma unroll
    for (int k = 0; k < V; ++k)
      if (!((kLive >> k) & 1u)) tma_load_1d(s_vec + k * kSlabRows, epi.vec(k) + r0, vb, &bar[0]);
    const int2 kr = slab ? ld_keep(slab + blk) : make_int2(__ldg(rp + r0), __ldg(rp + r0 + nr));
    *krange = kr;
    if (kr.x < kr.y) {
      issue_tile(kr.x, min(kr.x + cap, kr.y));
      tile_pending = true;
    }
    // Wave-ahead prefetch: bring the operands of slab blk + ahead (the block that takes this
    // block's place about one wave of resident blocks later) from DRAM into L2 now, with the same
    // 16-byte widened ranges its own copies will request; its copies then complete from L2. A
    // prefetch only warms the cache: the values that block reads are the ones in memory then.
    const int pb = blk + ahead;
    if (ahead > 0 && pb < (rows + kSlabRows - 1) / kSlabRows) {
      const int pr0 = pb * kSlabRows, pnr = min(kSlabRows, rows - pr0);
      prefetch_l2(rp + pr0, (static_cast<unsigned>(pnr + 1) * 4u + 15u) & ~15u);
      const unsigned pvb = (static_cast<unsigned>(pnr) * sizeof(T) + 15u) & ~15u;
#pragma unroll
      for (int k = 0; k < V; ++k) prefetch_l2(epi.vec(k) + pr0, pvb);
      const int2 pk = slab ? ld_keep(slab + pb) : make_int2(__ldg(rp + pr0), __ldg(rp + pr0 + pnr));
      if (pk.x < pk.y) {
        const int t1 = min(pk.x + cap, pk.y);
        const int c0 = pk.x & ~3, v0 = pk.x & ~(kValAlign - 1);
        const int c1 = (t1 + 3) & ~3, v1 = (t1 + kValAlign - 1) & ~(kValAlign - 1);
        prefetch_l2(col + c0, static_cast<unsigned>(c1 - c0) * 4u);
        prefetch_l2(val + v0, static_cast<unsigned>(v1 - v0) * sizeof(T));
      }
    }
  }
  pdl_wait();  // from here on the previous kernels' outputs are complete and visible
  int ok = 1;
  if (tid == 0) {
    if (kNumLive > 0) {
      mbar_expect_tx(&bar[2], static_cast<unsigned>(kNumLive) * vb);
#pragma unroll
      for (int k = 0; k < V; ++k)
        if ((kLive >> k) & 1u) tma_load_1d(s_vec + k * kSlabRows, epi.vec(k) + r0, vb, &bar[2]);
    }
    ok = mbar_wait_bounded(&bar[0], 0) ? 1 : 0;
    if (kNumLive > 0) ok = (mbar_wait_bounded(&bar[2], 0) && ok) ? 1 : 0;
  }
  bool staged = __syncthreads_and(ok) != 0;
  const int2 kr = *krange;
  const bool mine = tid < nr;
  int beg = 0, end = 0;
  if (staged && mine) beg = s_rp[tid], end = s_rp[tid + 1];
  auto acc = epi_acc(epi, 0);
  unsigned phase = 0;
  double s = 0.0;
  for (int t0 = kr.x; staged && t0 < kr.y; t0 += cap) {
    const int t1 = min(t0 + cap, kr.y);
    if (t0 != kr.x) {  // later tiles of a long slab: reuse the buffer once the previous tile is summed
      __syncthreads();
      if (tid == 0) {
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        issue_tile(t0, t1);
        tile_pending = true;
      }
    }
    if (tid == 0) {
      ok = mbar_wait_bounded(&bar[1], phase) ? 1 : 0;
      if (ok) phase ^= 1u, tile_pending = false;
    }
    if (!__syncthreads_and(ok)) {
      staged = false;
      break;
    }
    const int c0 = t0 & ~3, v0 = t0 & ~(kValAlign - 1);
    const int a = max(beg, t0), b = min(end, t1);
    if constexpr (GB == 0) {
      // Spread: the tile's products are formed by the whole block, nonzero t0 + tid + j·kSlabRows
      // by thread tid, every gather of a thread issued before the first is used, and written back
      // over the tile; then each thread adds its row's products in CSR order. A thread issues
      // about nnz/rows gathers whatever its row's length, all in one round trip.
      constexpr int kSpread = (kSlabTile + kSlabRows - 1) / kSlabRows;  // cap <= kSlabTile
      const int base = t0 + tid;
      int cl[kSpread];
#pragma unroll
      for (int q = 0; q < kSpread; ++q) cl[q] = (base + q * kSlabRows < t1) ? s_col[base + q * kSlabRows - c0] : 0;
      T g[kSpread];  // x[col] in T: the fp64 product below is the same (float -> double is exact)
#pragma unroll
      for (int q = 0; q < kSpread; ++q) g[q] = (base + q * kSlabRows < t1) ? gather_t(x, cl[q]) : T(0);
#pragma unroll
      for (int q = 0; q < kSpread; ++q) {
        const int k = base + q * kSlabRows;
        if (k < t1)
          put_product<T>(s_col, s_val, k - c0, k - v0,
                         static_cast<double>(s_val[k - v0]) * static_cast<double>(g[q]));
      }
      __syncthreads();
      for (int k = a; k < b; ++k) s += get_product<T>(s_col, s_val, k - c0, k - v0);  // in CSR order
    } else {
      for (int k = a; k < b; k += GB) {  // GB gathers in flight, then their products added in CSR order
        double p[GB];
#pragma unroll
        for (int q = 0; q < GB; ++q)
          p[q] = (k + q < b) ? static_cast<double>(s_val[k + q - v0]) * gather(x, s_col[k + q - c0]) : 0.0;
#pragma unroll
        for (int q = 0; q < GB; ++q)
          if (k + q < b) s += p[q];  // in CSR order
      }
    }
  }
  if (!staged) {  // never expected: record, wait (bounded) for copies still in flight, report NaN
    if (tid == 0) {
      count_stage_timeout(err);
      mbar_wait_bounded(&bar[0], 0);
      if (kNumLive > 0) mbar_wait_bounded(&bar[2], 0);
      if (tile_pending) mbar_wait_bounded(&bar[1], phase);
    }
    s = __longlong_as_double(0x7ff8000000000000LL);
  }
  if (mine) {
    const auto pre = staged ? epi.pre_at(s_vec, tid) : epi.load(r0 + tid);
    epi_apply(epi, r0 + tid, s, pre, acc);
  }
  epi_flush(epi, acc);
}

template <class T, class Epi, int GB = kGatherBatch>
__global__ void __launch_bounds__(kSlabRows, B200_FED_MIN_BLOCKS) k_slab_fed(int rows, const int* __restrict__ rp,
                                                           const int* __restrict__ col,
                                                           const T* __restrict__ val,
                                                           const T* __restrict__ x, Epi epi,
                                                           const int2* __restrict__ slab, int cap, unsigned* err,
                                                           int ahead) {
  slab_fed_body<T, Epi, GB>(static_cast<int>(blockIdx.x), rows, rp, col, val, x, epi, slab, cap, err, ahead);
}

// ---------------------------------------------------------------------- several LPs in one launch
// One LP's part of a grouped launch: its matrix, gathered vector, epilogue, and the first block of
// the grid that works on it (its slabs are blocks first … first + ⌈rows/kSlabRows⌉ − 1).
template <class T, class Epi>
struct GroupPart {
  int rows, cap, first;
  const int *rp, *col;
  const T *val, *x;
  const int2* slab;
  unsigned* err;
  Epi epi;
};
// The iteration kernel of several LPs at once (the request loop's continuous batching): each block
// finds its LP by a binary search over the parts' first blocks, then runs k_slab_fed's body on that
// LP's slab with the epilogue at step `step` — the same arithmetic as the LP's own launch, so an
// LP's iterates do not depend on which others share the launch. Shared memory is sized for the
// largest tile capacity among the parts.
template <class T, class Epi, int GB = kGatherBatch>
__global__ void __launch_bounds__(kSlabRows, B200_FED_MIN_BLOCKS) k_group_fed(const GroupPart<T, Epi>* __restrict__ parts,
                                                                             int nparts, int step) {
  const int b = static_cast<int>(blockIdx.x);
  int lo = 0, hi = nparts - 1;  // the last part whose first block is <= b
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (parts[mid].first <= b) lo = mid;
    else hi = mid - 1;
  }
  const GroupPart<T, Epi>& g = parts[lo];
  Epi epi = g.epi;
  epi.step = step;
  slab_fed_body<T, Epi, GB>(b - g.first, g.rows, g.rp, g.col, g.val, g.x, epi, g.slab, g.cap, g.err);
}

// Once per instantiation, outside any stream capture: prefer shared memory so that 8 CTAs of
// 24.6 KB fit on an SM.
template <class T, class Epi, bool kTma>
inline void slab_prepare() {
  static const bool done = [] {
    if (B200_SLAB_CARVEOUT >= 0)
      (void)cudaFuncSetAttribute(k_slab<T, Epi, kTma>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 B200_SLAB_CARVEOUT);
    (void)cudaGetLastError();
    return true;
  }();
  (void)done;
}

template <class T, class Epi, bool kTma = false>
inline void launch_slab(int rows, const int* rp, const int* col, const T* val, const T* x, const Epi& epi,
                        cudaStream_t st, const int2* slab = nullptr, unsigned* err = nullptr) {
  if (rows <= 0) return;
  slab_prepare<T, Epi, kTma>();
  const int grid = (rows + kSlabRows - 1) / kSlabRows;
  k_slab<T, Epi, kTma><<<grid, kSlabRows, 0, st>>>(rows, rp, col, val, x, epi, slab, err);
  B200_LAUNCH_CHECK();
}

// The TMA-staged form, for CSR arrays allocated by this library (tail-padded DevBufs). `slab`:
// an optional table of each slab's nonzero range (see slab_table). `err`: the bulk-copy timeout
// counter (nullptr: the process-wide one).
template <class T, class Epi>
inline void launch_slab_tma(int rows, const int* rp, const int* col, const T* val, const T* x, const Epi& epi,
                            cudaStream_t st, const int2* slab = nullptr, unsigned* err = nullptr) {
  launch_slab<T, Epi, B200_STAGE_TMA != 0>(rows, rp, col, val, x, epi, st, B200_SLAB_TABLE ? slab : nullptr, err);
}

// The fully staged form (k_slab_fed) for the iteration epilogues, whose operand vectors are
// library allocations; `rp` must be one too, `slab` the slab table of rp and `cap` the tile
// capacity from fed_tile_capacity. Falls back to launch_slab_tma when an operand is not 16-byte
// aligned or the shared memory would exceed the 48 KB that needs no opt-in. `pdl`: launch with
// programmatic dependent launch (B200_PDL builds), so the kernel's blocks may start while the
// previous kernel of the stream finishes: only where Epi::kLiveVecs names every operand vector a
// kernel still in flight may write. The fallback never uses it.
#ifndef B200_PDL
#define B200_PDL 1
#endif

// Launch variants of k_slab_fed, chosen per matrix by the autotuner (tune.hpp): `gather` = GB
// (2, 4 or 8 gathers in flight per thread, each thread walking its own row; 0: the spread form,
// where the block forms the tile's products together, an equal share per thread, before each
// thread adds its row's), `ctas` = resident CTAs per SM (0: as many as the registers and shared
// memory allow; k: dynamic shared memory padded so that no more than k fit), `ahead` = the
// wave-ahead L2 prefetch distance in waves of resident blocks (0: none). Every variant computes
// the same products and adds them in the same order: the results do not depend on the choice.
struct SlabVariant {
  int gather, ctas, ahead;
};
constexpr SlabVariant kSlabVariants[] = {{4, 0, 0}, {2, 0, 0}, {8, 0, 0}, {4, 5, 0}, {4, 4, 0}, {0, 0, 0}, {4, 0, 1}};
constexpr int kNumSlabVariants = static_cast<int>(sizeof(kSlabVariants) / sizeof(kSlabVariants[0]));

// Streaming multiprocessors of the current device (read once; 148 on a B200).
inline int device_sm_count() {
  static const int sms = [] {
    int dev = 0, v = 0;
    (void)cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0) v = 148;
    (void)cudaGetLastError();
    return v;
  }();
  return sms;
}

// Dynamic shared memory of a k_slab_fed launch that needs `bytes` under variant `v`.
inline unsigned fed_smem_bytes(unsigned bytes, const SlabVariant& v) {
  if (v.ctas <= 0) return bytes;
  static const int per_sm = [] {
    int dev = 0, v = 0;
    (void)cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev) != cudaSuccess) v = 233472;
    (void)cudaGetLastError();
    return v;
  }();
  static const int reserved = [] {
    int dev = 0, v = 0;
    (void)cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&v, cudaDevAttrReservedSharedMemoryPerBlock, dev) != cudaSuccess) v = 1024;
    (void)cudaGetLastError();
    return v;
  }();
  // v.ctas + 1 blocks of this size (plus their reserved bytes) exceed the SM's shared memory
  const long long pad = static_cast<long long>(per_sm) / (v.ctas + 1) - reserved + 16;
  return static_cast<unsigned>(std::max<long long>(bytes, (pad + 15) / 16 * 16));
}

template <class T, class Epi, int GB>
inline void launch_fed_gb(int grid, unsigned smem, cudaStream_t st, bool pdl, int rows, const int* rp, const int* col,
                          const T* val, const T* x, const Epi& epi, const int2* slab, int cap, unsigned* err,
                          int ahead) {
  if (smem > 48u * 1024u) {  // once per instantiation, outside any capture: allow the padded size
    static const bool opt = [] {
      (void)cudaFuncSetAttribute(k_slab_fed<T, Epi, GB>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
      (void)cudaGetLastError();
      return true;
    }();
    (void)opt;
  }
  if (B200_PDL && pdl) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(static_cast<unsigned>(grid));
    cfg.blockDim = dim3(kSlabRows);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    B200_CHECK(cudaLaunchKernelEx(&cfg, k_slab_fed<T, Epi, GB>, rows, rp, col, val, x, epi, slab, cap, err, ahead));
    return;
  }
  k_slab_fed<T, Epi, GB><<<grid, kSlabRows, smem, st>>>(rows, rp, col, val, x, epi, slab, cap, err, ahead);
  B200_LAUNCH_CHECK();
}

// The fully staged form (k_slab_fed) for the iteration epilogues, whose operand vectors are
// library allocations; `rp` must be one too, `slab` the slab table of rp and `cap` the tile
// capacity from fed_tile_capacity. Falls back to launch_slab_tma when an operand is not 16-byte
// aligned or the kernel's own shared memory would exceed 48 KB. `pdl`: launch with programmatic
// dependent launch (B200_PDL builds), so the kernel's blocks may start while the previous kernel
// of the stream finishes: only where Epi::kLiveVecs names every operand vector a kernel still in
// flight may write. The fallback never uses it. `variant`: an index into kSlabVariants.
template <class T, class Epi>
inline void launch_slab_fed(int rows, const int* rp, const int* col, const T* val, const T* x, const Epi& epi,
                            cudaStream_t st, const int2* slab, int cap, unsigned* err = nullptr, bool pdl = false,
                            int variant = 0) {
  if (rows <= 0) return;
  const FedLayout L = fed_layout(Epi::kVecs, static_cast<int>(sizeof(T)), cap);
  bool ok = B200_SLAB_FED && B200_STAGE_TMA && cap >= 16 && cap % 16 == 0 && L.bytes <= 48u * 1024u &&
            (reinterpret_cast<std::uintptr_t>(rp) & 15u) == 0;
  for (int k = 0; k < Epi::kVecs; ++k) ok = ok && (reinterpret_cast<std::uintptr_t>(epi.vec(k)) & 15u) == 0;
  if (!ok) return launch_slab_tma<T>(rows, rp, col, val, x, epi, st, slab, err);
  const SlabVariant v = kSlabVariants[(variant >= 0 && variant < kNumSlabVariants) ? variant : 0];
  const int grid = (rows + kSlabRows - 1) / kSlabRows;
  const unsigned smem = fed_smem_bytes(L.bytes, v);
  // one wave: the blocks resident at once (SMs x blocks per SM, the padded count or the usual 5)
  const int ahead = v.ahead * device_sm_count() * (v.ctas > 0 ? v.ctas : B200_FED_MIN_BLOCKS);
  switch (v.gather) {
    case 2: return launch_fed_gb<T, Epi, 2>(grid, smem, st, pdl, rows, rp, col, val, x, epi, slab, cap, err, ahead);
    case 8: return launch_fed_gb<T, Epi, 8>(grid, smem, st, pdl, rows, rp, col, val, x, epi, slab, cap, err, ahead);
    case 0: return launch_fed_gb<T, Epi, 0>(grid, smem, st, pdl, rows, rp, col, val, x, epi, slab, cap, err, ahead);
    default: return launch_fed_gb<T, Epi, 4>(grid, smem, st, pdl, rows, rp, col, val, x, epi, slab, cap, err, ahead);
  }
}

// The nonzero range [rp[b·kSlabRows], rp[min((b+1)·kSlabRows, rows)]) of every slab b.
static __global__ void k_slab_table(int rows, const int* rp, int2* out) {
  const int nb = (rows + kSlabRows - 1) / kSlabRows;
  B200_FOR(b, nb) {
    const int r0 = static_cast<int>(b) * kSlabRows, r1 = min(r0 + kSlabRows, rows);
    out[b] = make_int2(rp[r0], rp[r1]);
  }
}
inline int slab_count(int rows) { return rows <= 0 ? 0 : (rows + kSlabRows - 1) / kSlabRows; }

// The largest slab's nonzero count, from a slab table (synchronises `st`; setup only).
inline long long slab_max_nnz(const int2* table, int nb, cudaStream_t st) {
  if (nb <= 0) return 0;
  std::vector<int2> h(static_cast<std::size_t>(nb));
  B200_CHECK(cudaMemcpyAsync(h.data(), table, h.size() * sizeof(int2), cudaMemcpyDeviceToHost, st));
  B200_CHECK(cudaStreamSynchronize(st));
  long long mx = 0;
  for (const int2& r : h) mx = std::max<long long>(mx, static_cast<long long>(r.y) - r.x);
  return mx;
}

// Number of bulk-copy waits that ran out since the library was loaded (host side).
inline unsigned stage_timeouts() {
  unsigned v = 0;
  cudaMemcpyFromSymbol(&v, g_stage_timeouts, sizeof v);
  return v;
}

// Element-wise form of an epilogue: epi(i, double(v[i])) — the unfused backend ops use the
// same functors as the fused kernels, so both paths share one arithmetic definition.
template <class T, class Epi>
static __global__ void k_elementwise(std::int64_t n, const T* __restrict__ v, Epi epi) {
  if (!epi.active()) return;
  B200_FOR(i, n) epi(static_cast<int>(i), static_cast<double>(v[i]));
}

// ---------------------------------------------------------------------- step parameters
// Written by the host before each epoch (pinned -> device copy); read by every kernel of the
// captured epoch graph, so the graph never needs re-instantiation.
struct StepParams {
  double tau, sigma;       // η/ω, ηω (host-computed in fp64, as r2hpdhg.cpp:67)
  double rho;              // reflection coefficient ρ
  long long inner0;        // Halpern counter k at the start of the epoch
  int K;                   // iterations per epoch
  int done;                // 1: the solve has ended; every kernel returns at once
  int skip_r0;             // 1: the epoch continues a Halpern cycle (no r⁰ residual)
};

// Device address of the r⁰ skip flag inside a device-resident StepParams.
inline const int* skip_r0_flag(const StepParams* d_params) {
  return reinterpret_cast<const int*>(reinterpret_cast<const char*>(d_params) + offsetof(StepParams, skip_r0));
}

// Halpern weight of step `step` in the epoch: w = (k+1)/(k+2), k = inner0 + step
// (r2hpdhg.cpp:69, computed in fp64 then cast to T).
__device__ __forceinline__ double halpern_weight(const StepParams* P, int step) {
  const long long k = P->inner0 + step;
  return static_cast<double>(k + 1) / static_cast<double>(k + 2);
}

// ---------------------------------------------------------------------- epilogues
struct AlwaysActive {
  __device__ bool active() const { return true; }
};

template <class T>
struct EpiStore : AlwaysActive {  // out = T(s)
  T* out;
  __device__ void operator()(int i, double s) const { out[i] = static_cast<T>(s); }
};

// r2h_primal fused after aty = Ãᵀy (cpu_backend.cpp:140-157):
//   x̂ = clamp(x − τ(c − aty), l, u); x̄ = 2x̂ − x; x ← w(2ρx̂ + (1−2ρ)x) + (1−w)x0
// Either from a StepParams (fused engine path) or from explicit scalars (backend ops).
template <class T>
struct EpiPrimal {
  T *x, *xh, *xb;
  const T *x0, *c, *l, *u;
  const StepParams* P;  // non-null: engine path
  int step;
  double tau, w, rho;   // backend-op path
  struct Pre {
    T x, x0, c, l, u;
  };
  __device__ bool active() const { return P == nullptr || !P->done; }
  __device__ Pre load(int j) const {
    return Pre{ld_stream(x + j), ld_stream(x0 + j), ld_stream(c + j), ld_stream(l + j), ld_stream(u + j)};
  }
  // The streamed operands as arrays (k_slab_fed stages their slab ranges in shared memory);
  // x is written by the primal kernel of the previous step (live), the others only between epochs.
  static constexpr int kVecs = 5;
  static constexpr unsigned kLiveVecs = 0x1u;
  __host__ __device__ const T* vec(int k) const { return k == 0 ? x : k == 1 ? x0 : k == 2 ? c : k == 3 ? l : u; }
  __device__ Pre pre_at(const T* sv, int t) const {
    return Pre{sv[t], sv[kSlabRows + t], sv[2 * kSlabRows + t], sv[3 * kSlabRows + t], sv[4 * kSlabRows + t]};
  }
  __device__ void operator()(int j, double s) const { (*this)(j, s, load(j)); }
  __device__ void operator()(int j, double s, const Pre& p) const {
    double tau_d = tau, w_d = w, rho_d = rho;
    if (P) tau_d = P->tau, w_d = halpern_weight(P, step), rho_d = P->rho;
    const T aty = static_cast<T>(s);
    const T t = static_cast<T>(tau_d), tw = static_cast<T>(w_d);
    const T a = static_cast<T>(2 * rho_d), b = static_cast<T>(1 - 2 * rho_d);
    const T xj = p.x;
    const T h = ref_clamp<T>(xj - t * (p.c - aty), p.l, p.u);
    // x̂ is read only by the residual and the check that follow an epoch's first step (when it
    // starts a Halpern cycle) and its last step; on the other steps it is not stored.
    const bool store_hat = !P || step == P->K - 1 || P->inner0 + step == 0;
    if (store_hat) xh[j] = h;
    st_keep(xb + j, static_cast<T>(static_cast<T>(2) * h - xj));  // gathered by the dual kernel next
    x[j] = tw * (a * h + b * xj) + (static_cast<T>(1) - tw) * p.x0;
  }
};

// r2h_dual fused after ax = Ãx̄ (cpu_backend.cpp:159-178):
//   v = ax − y/σ; ŷ = y − σax + σ clamp(v, rl, ru); ȳ = 2ŷ − y (residual steps only);
//   y ← w(2ρŷ + (1−2ρ)y) + (1−w)y0
template <class T>
struct EpiDual {
  T *y, *yh, *yb;
  const T *y0, *rl, *ru;
  const StepParams* P;
  int step;
  double sigma, w, rho;
  int write_yb;  // backend-op path
  struct Pre {
    T y, y0, rl, ru;
  };
  __device__ bool active() const { return P == nullptr || !P->done; }
  __device__ Pre load(int i) const { return Pre{ld_stream(y + i), ld_stream(y0 + i), ld_stream(rl + i), ld_stream(ru + i)}; }
  static constexpr int kVecs = 4;
  static constexpr unsigned kLiveVecs = 0x1u;  // y (the dual kernel of the previous step writes it)
  __host__ __device__ const T* vec(int k) const { return k == 0 ? y : k == 1 ? y0 : k == 2 ? rl : ru; }
  __device__ Pre pre_at(const T* sv, int t) const {
    return Pre{sv[t], sv[kSlabRows + t], sv[2 * kSlabRows + t], sv[3 * kSlabRows + t]};
  }
  __device__ void operator()(int i, double s) const { (*this)(i, s, load(i)); }
  __device__ void operator()(int i, double s, const Pre& p) const {
    double sig_d = sigma, w_d = w, rho_d = rho;
    bool wb = write_yb != 0;
    if (P) {
      sig_d = P->sigma, w_d = halpern_weight(P, step), rho_d = P->rho;
      wb = (step == P->K - 1) || (P->inner0 + step == 0);
    }
    const T ax = static_cast<T>(s);
    const T sg = static_cast<T>(sig_d), tw = static_cast<T>(w_d);
    const T a = static_cast<T>(2 * rho_d), b = static_cast<T>(1 - 2 * rho_d);
    const T yi = p.y;
    const T v = ax - yi / sg;
    const T h = yi - sg * ax + sg * ref_clamp<T>(v, p.rl, p.ru);
    if (wb) {  // ŷ, ȳ are read only after the steps that feed a residual (as x̂ above)
      yh[i] = h;
      yb[i] = static_cast<T>(2) * h - yi;
    } else if (!P) {
      yh[i] = h;
    }
    st_keep(y + i, static_cast<T>(tw * (a * h + b * yi) + (static_cast<T>(1) - tw) * p.y0));  // gathered next
  }
};

// PDLP steps (pdlp.cpp:54-67), in the backend ops' arithmetic, fused after the SpMVs. The running
// averages use w_a = 1/inner with inner = inner0 + step + 1 (the iterate count since the last
// restart, after this step):
//   primal, after aty = Ãᵀy:  x⁺ = clamp(x − τ(c − aty), l, u);  x̄ = −1·x + 2·x⁺ (copy + axpby);
//                             xa ← w_a·x⁺ + (1 − w_a)·xa
//   dual, after ax = Ãx̄:     y⁺ = y − σ·ax + σ·clamp(ax − y/σ, rl, ru);  ya ← w_a·y⁺ + (1 − w_a)·ya
template <class T>
struct EpiPdlpPrimal {
  const T *x, *c, *l, *u;
  T *xn, *xb, *xa;
  const StepParams* P;
  int step;
  struct Pre {
    T x, c, l, u, xa;
  };
  __device__ bool active() const { return !P->done; }
  __device__ Pre load(int j) const { return Pre{x[j], c[j], l[j], u[j], xa[j]}; }
  static constexpr int kVecs = 5;
  static constexpr unsigned kLiveVecs = 0x11u;  // x and the running average xa
  __host__ __device__ const T* vec(int k) const { return k == 0 ? x : k == 1 ? c : k == 2 ? l : k == 3 ? u : xa; }
  __device__ Pre pre_at(const T* sv, int t) const {
    return Pre{sv[t], sv[kSlabRows + t], sv[2 * kSlabRows + t], sv[3 * kSlabRows + t], sv[4 * kSlabRows + t]};
  }
  __device__ void operator()(int j, double s) const { (*this)(j, s, load(j)); }
  __device__ void operator()(int j, double s, const Pre& p) const {
    const T t = static_cast<T>(P->tau);
    const T aty = static_cast<T>(s);
    const T h = ref_clamp<T>(p.x - t * (p.c - aty), p.l, p.u);
    xn[j] = h;
    xb[j] = static_cast<T>(-1.0) * p.x + static_cast<T>(2.0) * h;
    const double wa = 1.0 / static_cast<double>(P->inner0 + step + 1);
    xa[j] = static_cast<T>(wa) * h + static_cast<T>(1.0 - wa) * p.xa;
  }
};
template <class T>
struct EpiPdlpDual {
  const T *y, *rl, *ru;
  T *yn, *ya;
  const StepParams* P;
  int step;
  struct Pre {
    T y, rl, ru, ya;
  };
  __device__ bool active() const { return !P->done; }
  __device__ Pre load(int i) const { return Pre{y[i], rl[i], ru[i], ya[i]}; }
  static constexpr int kVecs = 4;
  static constexpr unsigned kLiveVecs = 0x9u;  // y and the running average ya
  __host__ __device__ const T* vec(int k) const { return k == 0 ? y : k == 1 ? rl : k == 2 ? ru : ya; }
  __device__ Pre pre_at(const T* sv, int t) const {
    return Pre{sv[t], sv[kSlabRows + t], sv[2 * kSlabRows + t], sv[3 * kSlabRows + t]};
  }
  __device__ void operator()(int i, double s) const { (*this)(i, s, load(i)); }
  __device__ void operator()(int i, double s, const Pre& p) const {
    const T sg = static_cast<T>(P->sigma);
    const T ax = static_cast<T>(s);
    const T v = ax - p.y / sg;
    const T h = p.y - sg * ax + sg * ref_clamp<T>(v, p.rl, p.ru);
    yn[i] = h;
    const double wa = 1.0 / static_cast<double>(P->inner0 + step + 1);
    ya[i] = static_cast<T>(wa) * h + static_cast<T>(1.0 - wa) * p.ya;
  }
};

// primal_step / dual_step of the backend (cpu_backend.cpp:113-138).
template <class T>
struct EpiPrimalStep : AlwaysActive {
  const T *x, *c, *l, *u;
  T* xh;
  double tau;
  __device__ void operator()(int j, double s) const {
    const T t = static_cast<T>(tau);
    const T aty = static_cast<T>(s);
    xh[j] = ref_clamp<T>(x[j] - t * (c[j] - aty), l[j], u[j]);
  }
};
template <class T>
struct EpiDualStep : AlwaysActive {
  const T *y, *rl, *ru;
  T* yh;
  double sigma;
  __device__ void operator()(int i, double s) const {
    const T sg = static_cast<T>(sigma);
    const T ax = static_cast<T>(s);
    const T v = ax - y[i] / sg;
    yh[i] = y[i] - sg * ax + sg * ref_clamp<T>(v, rl[i], ru[i]);
  }
};

}  // namespace b200
