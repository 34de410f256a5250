// reduce.cuh — deterministic fp64 sums over term arrays, in two selectable orders.
//
// Every reduction of the engine first materialises its per-element terms (double), then a
// SumPlan reduces them. Two orders:
//   exact: the reference CPU's own order. kSeq = one sequential chain (the reference's plain
//          host loops, e.g. kkt_general, cpu_backend.cpp:226-284); kChunk64 = 64 contiguous
//          chunks summed sequentially, then the 64 partials in order (la::parallel_sum,
//          parallel.h:169-188, used by Backend::dot / diff_norm2). Each chain's result is the
//          sequential chain's bit for bit, computed in parallel (k_xstat / k_xagg / k_xchain
//          below): the order is exactly i = lo, lo+1, … as far as rounding can tell.
//   fast:  a fixed two-level tree (kTreeBlocks blocks per sum, block tree, then one block
//          combines the partials) — deterministic run to run, but a different rounding.
// Maxima never go through a SumPlan: they are taken with integer atomics on non-negative
// doubles, which is order-independent and exact.
#pragma once

#include <climits>
#include <vector>

#include "common.cuh"

namespace b200 {

enum class SumOrder { kSeq, kChunk64 };

struct TreeSeg {
  const double* t;
  long long lo, hi;
  double init;
  double* out;
};

constexpr int kTreeBlocks = 96;
constexpr int kChunks = 64;  // la::kReduceChunks

__device__ __forceinline__ double block_sum_fixed(double v, double* sh) {
  for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(kFull, v, off);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) sh[wid] = v;
  __syncthreads();
  if (wid == 0) {
    v = lane < static_cast<int>(blockDim.x >> 5) ? sh[lane] : 0.0;
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(kFull, v, off);
  }
  return v;  // valid in thread 0
}

// ------------------------------------------------------------------ exact chains, in parallel
// A chain s = init; s = fl(s + t[i]) for i = lo, lo+1, … is inherently sequential, and walking
// 2.5 million terms with one warp costs milliseconds. It is evaluated here in parallel, with the
// sequential chain's result bit for bit, from one property of round-to-nearest: while every
// partial sum stays inside one binade [2^e, 2^(e+1)) (ulp u = 2^(e−52)), each partial sum is a
// multiple of u, so fl(s + t) = s + u·rint(t/u) exactly — unless t/u is a tie (x.5), or the exact
// sum leaves the binade. Inside such a run the chain is an INTEGER sum of k = rint(t/u), which is
// associative. So:
//   k_xstat   per tile of kXTile terms: an approximate fp64 sum and the approximate range of the
//             tile's running sums (any order; only used to guess each tile's binade);
//   k_xagg    per tile: the guessed binade's u from the approximate start (the approximate sums
//             of the chain's earlier tiles), then K = Σ k and the minimum / maximum of the
//             integer running sums, in int64 (exact); ties and |t/u| ≥ 2^51 mark the tile;
//   k_xchain  one warp per chain walks its tiles in order with the EXACT s: a tile is committed
//             as s ← (s/u + K)·u when s lies in the guessed binade and s/u plus every running
//             integer sum stays within [2^52 + 1, 2^53 − 1] (so each exact partial sum lies inside
//             the binade, at least u/2 from its ends); any other tile is walked in windows of
//             256 terms with the same test per term, committing the valid prefix and adding the
//             first failing term with one plain fp64 addition (so ties, binade changes, zeros,
//             subnormals, infinities and NaN get exactly the sequential chain's arithmetic).
// The approximations only choose between two exact paths; the result never depends on them.
constexpr int kXTile = 2048;    // terms per tile (8 per thread of a 256-thread block)
constexpr int kXPer = 8;        // terms per thread (tiles) and per lane (windows)
constexpr int kXThreads = kXTile / kXPer;

struct XChain {
  const double* t;
  long long lo, hi;  // terms t[lo, hi)
  double init;
  double* out;
  int tile0, ntiles;  // this chain's tiles in the tile arrays (ntiles = 0: windows only)
};
struct XTileStat {
  double sum, pmin, pmax;  // approximate: Σ t, min / max of the running sums from the tile start
  int bad;                 // a non-finite term
  int pad;
};
struct XTileAgg {
  double u;               // the binade's ulp the integers are counted in (0: no guess)
  long long K, pmin, pmax;  // Σ k and the min / max of the running integer sums (positions 1…len)
  int ok;                 // no tie, every |t/u| < 2^51
  int pad;
};

constexpr long long kX52 = 1LL << 52, kX53 = 1LL << 53;

// e = floor(log2 |v|) for a normal v whose ulp 2^(e−52) and 2^(52−e) are both normal doubles;
// otherwise returns false.
__device__ __forceinline__ bool x_binade(double v, int& e) {
  const long long bits = __double_as_longlong(v);
  const int ef = static_cast<int>((bits >> 52) & 0x7ff);
  if (ef == 0 || ef == 0x7ff) return false;  // zero, subnormal, inf, NaN
  e = ef - 1023;
  return e >= -970 && e <= 1023;
}
__device__ __forceinline__ double x_pow2(int p) {  // 2^p, p in [−1022, 1023]
  return __longlong_as_double(static_cast<long long>(p + 1023) << 52);
}
// k = rint(t/u) with inv_u = 1/u (powers of two: t·inv_u is exact unless it under/overflows);
// returns false for a tie, |t/u| ≥ 2^51, or a non-finite t.
__device__ __forceinline__ bool x_count(double t, double inv_u, long long& k) {
  const double q = t * inv_u;
  if (!(fabs(q) < 2251799813685248.0)) return false;  // 2^51; also NaN / inf
  const double f = floor(q);
  if (q - f == 0.5) return false;  // a tie: rounding depends on the partial sum's last bit
  k = static_cast<long long>(rint(q));
  return true;
}
// |S| inside [2^52 + 1, 2^53 − 1] with the sign of S0.
__device__ __forceinline__ bool x_inside(long long S0, long long S) {
  return S0 > 0 ? (S >= kX52 + 1 && S <= kX53 - 1) : (S <= -(kX52 + 1) && S >= -(kX53 - 1));
}

template <class T, class Op>
__device__ __forceinline__ T x_block_reduce(T v, Op op, T* sh) {  // result valid in every thread
  for (int off = 16; off > 0; off >>= 1) v = op(v, __shfl_xor_sync(kFull, v, off));
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  __syncthreads();
  if (lane == 0) sh[wid] = v;
  __syncthreads();
  v = sh[0];
  for (int w = 1; w < nw; ++w) v = op(v, sh[w]);
  return v;
}
// Exclusive prefix of per-thread values over the block (thread order), and the block total.
template <class T>
__device__ __forceinline__ T x_block_excl(T v, T& total, T* sh) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  T inc = v;
  for (int off = 1; off < 32; off <<= 1) {
    const T o = __shfl_up_sync(kFull, inc, off);
    if (lane >= off) inc += o;
  }
  __syncthreads();
  if (lane == 31) sh[wid] = inc;
  __syncthreads();
  T before = T(0);
  total = T(0);
  for (int w = 0; w < nw; ++w) {
    if (w < wid) before += sh[w];
    total += sh[w];
  }
  return before + inc - v;
}

__device__ __forceinline__ void x_tile_range(const XChain& c, int tile, long long& a, long long& b) {
  a = c.lo + static_cast<long long>(tile - c.tile0) * kXTile;
  b = a + kXTile < c.hi ? a + kXTile : c.hi;
}

static __global__ void __launch_bounds__(kXThreads) k_xstat(const XChain* ch, const int* tile_chain,
                                                            XTileStat* st, const int* skip) {
  __shared__ double shd[32];
  __shared__ int shi[32];
  if (skip && *skip) return;
  const int tile = blockIdx.x;
  const XChain c = ch[tile_chain[tile]];
  long long a, b;
  x_tile_range(c, tile, a, b);
  const long long i0 = a + static_cast<long long>(threadIdx.x) * kXPer;
  double run = 0.0, mn = INFINITY, mx = -INFINITY;
  int bad = 0;
#pragma unroll
  for (int q = 0; q < kXPer; ++q)
    if (i0 + q < b) {
      const double v = c.t[i0 + q];
      bad |= !isfinite(v);
      run += v;
      mn = fmin(mn, run), mx = fmax(mx, run);
    }
  double total;
  const double before = x_block_excl(run, total, shd);
  mn += before, mx += before;
  mn = x_block_reduce(mn, [](double x, double y) { return fmin(x, y); }, shd);
  mx = x_block_reduce(mx, [](double x, double y) { return fmax(x, y); }, shd);
  bad = x_block_reduce(bad, [](int x, int y) { return x | y; }, shi);
  if (threadIdx.x == 0) st[tile] = XTileStat{total, mn, mx, bad, 0};
}

static __global__ void __launch_bounds__(kXThreads) k_xagg(const XChain* ch, const int* tile_chain,
                                                           const XTileStat* st, XTileAgg* ag, const int* skip) {
  __shared__ double shd[32];
  __shared__ long long shl[32];
  __shared__ int shi[32];
  if (skip && *skip) return;
  const int tile = blockIdx.x;
  const XChain c = ch[tile_chain[tile]];
  long long a, b;
  x_tile_range(c, tile, a, b);
  // the approximate running sum at the tile's start
  double pre = 0.0;
  for (int k = c.tile0 + static_cast<int>(threadIdx.x); k < tile; k += blockDim.x) pre += st[k].sum;
  pre = x_block_reduce(pre, [](double x, double y) { return x + y; }, shd);
  const double s0 = c.init + pre, lo_v = s0 + st[tile].pmin, hi_v = s0 + st[tile].pmax;
  int e0, e1, e2;
  const bool guess = x_binade(s0, e0) && x_binade(lo_v, e1) && x_binade(hi_v, e2) && e0 == e1 && e0 == e2 &&
                     (s0 > 0) == (lo_v > 0) && (s0 > 0) == (hi_v > 0);
  if (!guess) {
    if (threadIdx.x == 0) ag[tile] = XTileAgg{0.0, 0, 0, 0, 0, 0};
    return;
  }
  const double inv_u = x_pow2(52 - e0);
  const long long i0 = a + static_cast<long long>(threadIdx.x) * kXPer;
  long long run = 0, mn = LLONG_MAX, mx = LLONG_MIN;
  int ok = 1;
#pragma unroll
  for (int q = 0; q < kXPer; ++q)
    if (i0 + q < b) {
      long long k = 0;
      ok &= x_count(c.t[i0 + q], inv_u, k) ? 1 : 0;
      run += k;
      mn = run < mn ? run : mn;
      mx = run > mx ? run : mx;
    }
  long long total;
  const long long before = x_block_excl(run, total, shl);
  if (mn != LLONG_MAX) mn += before, mx += before;
  mn = x_block_reduce(mn, [](long long x, long long y) { return x < y ? x : y; }, shl);
  mx = x_block_reduce(mx, [](long long x, long long y) { return x > y ? x : y; }, shl);
  ok = x_block_reduce(ok, [](int x, int y) { return x & y; }, shi);
  if (threadIdx.x == 0) ag[tile] = XTileAgg{x_pow2(e0 - 52), total, mn, mx, ok, 0};
}

// The chain over t[a, b) from the exact partial sum s, by windows of 32·kXPer terms (all 32 lanes
// call it with the same s and return the same s).
__device__ __forceinline__ double x_window_walk(const double* __restrict__ t, long long a, long long b, double s) {
  const int lane = threadIdx.x & 31;
  long long pos = a;
  while (pos < b) {
    int e;
    if (!x_binade(s, e)) {  // zero, subnormal, inf or NaN: a plain sequential run of up to 32 terms
      const long long rem = b - pos;
      const int cnt = rem < 32 ? static_cast<int>(rem) : 32;
      const double v = lane < cnt ? t[pos + lane] : 0.0;
      for (int j = 0; j < cnt; ++j) s += __shfl_sync(kFull, v, j);
      pos += cnt;
      continue;
    }
    const double u = x_pow2(e - 52), inv_u = x_pow2(52 - e);
    const long long S0 = static_cast<long long>(s * inv_u);
    const long long i0 = pos + static_cast<long long>(lane) * kXPer;
    double v[kXPer];
    long long pk[kXPer];  // this lane's inclusive running integer sums
    int first = kXPer;    // this lane's first invalid position (kXPer: none)
    long long run = 0;
#pragma unroll
    for (int q = 0; q < kXPer; ++q) {
      v[q] = i0 + q < b ? t[i0 + q] : 0.0;
      long long k = 0;
      const bool ok = i0 + q < b && x_count(v[q], inv_u, k);
      run += k;
      pk[q] = run;
      if (!ok && first == kXPer && i0 + q < b) first = q;
    }
    long long inc = run;  // warp inclusive scan of the lane totals
    for (int off = 1; off < 32; off <<= 1) {
      const long long o = __shfl_up_sync(kFull, inc, off);
      if (lane >= off) inc += o;
    }
    const long long before = inc - run;
#pragma unroll
    for (int q = 0; q < kXPer; ++q)
      if (q < first && i0 + q < b && !x_inside(S0, S0 + before + pk[q])) first = q;
    const bool has_end = i0 < b;  // this lane holds at least one term
    const unsigned fail = __ballot_sync(kFull, has_end && first < kXPer && i0 + first < b);
    if (fail == 0) {
      const long long total = __shfl_sync(kFull, inc, 31);
      s = static_cast<double>(S0 + total) * u;
      pos = pos + 32LL * kXPer < b ? pos + 32LL * kXPer : b;
      continue;
    }
    const int fl = __ffs(fail) - 1;
    const int fq = __shfl_sync(kFull, first, fl);
    long long committed = before;  // the running sum just before this lane's first invalid term
#pragma unroll
    for (int q = 0; q < kXPer; ++q)
      if (q + 1 == first) committed = before + pk[q];
    committed = __shfl_sync(kFull, committed, fl);
    double vf = 0.0;
#pragma unroll
    for (int q = 0; q < kXPer; ++q)
      if (q == fq) vf = v[q];
    vf = __shfl_sync(kFull, vf, fl);
    s = static_cast<double>(S0 + committed) * u;  // the valid prefix (nothing when it is empty)
    s += vf;                                      // the failing term, as the sequential chain adds it
    const long long f = static_cast<long long>(fl) * kXPer + fq;
    pos += f + 1;
    if (f < kXPer) {  // little progress: a plain run of up to 32 terms before the next window
      const long long rem = b - pos;
      const int cnt = rem <= 0 ? 0 : (rem < 32 ? static_cast<int>(rem) : 32);
      const double w = lane < cnt ? t[pos + lane] : 0.0;
      for (int j = 0; j < cnt; ++j) s += __shfl_sync(kFull, w, j);
      pos += cnt;
    }
  }
  return s;
}

// One warp per chain: tiles in order (committed whole when valid for the exact s), the rest
// walked in windows.
static __global__ void k_xchain(const XChain* ch, int nch, const XTileAgg* ag, const int* skip) {
  if (skip && *skip) return;
  const int warp = static_cast<int>((blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (warp >= nch) return;
  const XChain c = ch[warp];
  double s = c.init;
  if (c.ntiles == 0) {
    s = x_window_walk(c.t, c.lo, c.hi, s);
  } else {
    for (int g = 0; g < c.ntiles; g += 32) {
      XTileAgg mine{0.0, 0, 0, 0, 0, 0};
      if (g + lane < c.ntiles) mine = ag[c.tile0 + g + lane];
      const int cnt = c.ntiles - g < 32 ? c.ntiles - g : 32;
      for (int j = 0; j < cnt; ++j) {
        const double u = __shfl_sync(kFull, mine.u, j);
        const long long K = __shfl_sync(kFull, mine.K, j), pmin = __shfl_sync(kFull, mine.pmin, j);
        const long long pmax = __shfl_sync(kFull, mine.pmax, j);
        const int ok = __shfl_sync(kFull, mine.ok, j);
        bool commit = false;
        int e;
        if (ok && u != 0.0 && x_binade(s, e) && x_pow2(e - 52) == u) {
          const long long S0 = static_cast<long long>(s * x_pow2(52 - e));
          commit = x_inside(S0, S0 + pmin) && x_inside(S0, S0 + pmax);
          if (commit) s = static_cast<double>(S0 + K) * u;
        }
        if (!commit) {
          long long a, b;
          x_tile_range(c, c.tile0 + g + j, a, b);
          s = x_window_walk(c.t, a, b, s);
        }
      }
    }
  }
  if (lane == 0) *c.out = s;
}

static __global__ void k_tree1(const TreeSeg* segs, int nseg, double* partials, const int* skip) {
  __shared__ double sh[32];
  if (skip && *skip) return;
  const int s = blockIdx.x / kTreeBlocks, b = blockIdx.x % kTreeBlocks;
  if (s >= nseg) return;
  const TreeSeg g = segs[s];
  const long long len = g.hi - g.lo;
  const long long a = g.lo + len * b / kTreeBlocks, e = g.lo + len * (b + 1) / kTreeBlocks;
  double acc = 0.0;
  for (long long i = a + threadIdx.x; i < e; i += blockDim.x) acc += g.t[i];
  acc = block_sum_fixed(acc, sh);
  if (threadIdx.x == 0) partials[static_cast<long long>(s) * kTreeBlocks + b] = acc;
}

static __global__ void k_tree2(const TreeSeg* segs, int nseg, const double* partials, const int* skip) {
  __shared__ double sh[32];
  if (skip && *skip) return;
  const int s = blockIdx.x;
  if (s >= nseg) return;
  double acc = 0.0;
  for (int i = threadIdx.x; i < kTreeBlocks; i += blockDim.x) acc += partials[static_cast<long long>(s) * kTreeBlocks + i];
  acc = block_sum_fixed(acc, sh);
  if (threadIdx.x == 0) *segs[s].out = segs[s].init + acc;
}

// A fixed set of sums over fixed term arrays. Built once (descriptors live on the device),
// launched any number of times, also inside stream capture.
class SumPlan {
 public:
  void add(const double* terms, long long lo, long long hi, double init, SumOrder order, double* out) {
    jobs_.push_back({terms, lo, hi, init, order, out});
  }
  // skip: optional device int; when non-zero at run time every kernel of the plan returns.
  // st: the stream the plan is launched on; the segment descriptors are copied to the device on
  // it, so they are in place before the plan's first launch on that stream.
  void build(bool exact, const int* skip, cudaStream_t st) {
    exact_ = exact;
    skip_ = skip;
    if (exact) {
      std::vector<XChain> phase1, phase2;
      std::vector<int> tile_chain;
      long long nchunk_jobs = 0;
      for (const Job& j : jobs_)
        if (j.order == SumOrder::kChunk64) ++nchunk_jobs;
      partials_.alloc(static_cast<std::size_t>(nchunk_jobs > 0 ? nchunk_jobs * kChunks : 1));
      auto chain = [&](const double* t, long long lo, long long hi, double init, double* out) {
        XChain c{t, lo, hi, init, out, static_cast<int>(tile_chain.size()), 0};
        const long long n = hi - lo;
        if (n >= 2LL * kXTile) {  // long chains go by tiles; short ones by windows only
          c.ntiles = static_cast<int>((n + kXTile - 1) / kXTile);
          for (int k = 0; k < c.ntiles; ++k) tile_chain.push_back(static_cast<int>(phase1.size()));
        }
        phase1.push_back(c);
      };
      long long slot = 0;
      for (const Job& j : jobs_) {
        const long long n = j.hi - j.lo;
        if (j.order == SumOrder::kSeq) {
          chain(j.t, j.lo, j.hi, j.init, j.out);
        } else {
          const long long chunks = n < kChunks ? (n < 1 ? 1 : n) : kChunks;
          double* part = partials_.get() + slot * kChunks;
          for (long long c = 0; c < chunks; ++c)
            chain(j.t, j.lo + n * c / chunks, j.lo + n * (c + 1) / chunks, 0.0, part + c);
          // parallel_sum: s = 0; s += part[c] in order — then the caller's init (0 for dots)
          phase2.push_back({part, 0, chunks, j.init, j.out, 0, 0});
          ++slot;
        }
      }
      ntiles_ = static_cast<int>(tile_chain.size());
      upload(phase1, seg1_, st);
      upload(phase2, seg2_, st);
      upload(tile_chain, tile_chain_, st);
      tile_stat_.alloc(static_cast<std::size_t>(ntiles_ > 0 ? ntiles_ : 1) * sizeof(XTileStat));
      tile_agg_.alloc(static_cast<std::size_t>(ntiles_ > 0 ? ntiles_ : 1) * sizeof(XTileAgg));
      n1_ = static_cast<int>(phase1.size());
      n2_ = static_cast<int>(phase2.size());
    } else {
      std::vector<TreeSeg> tree;
      for (const Job& j : jobs_) tree.push_back({j.t, j.lo, j.hi, j.init, j.out});
      upload(tree, tseg_, st);
      nt_ = static_cast<int>(tree.size());
      partials_.alloc(static_cast<std::size_t>(nt_ > 0 ? nt_ : 1) * kTreeBlocks);
    }
  }
  void launch(cudaStream_t st) const {
    if (exact_) {
      const XChain* c1 = reinterpret_cast<const XChain*>(seg1_.get());
      const int* tc = reinterpret_cast<const int*>(tile_chain_.get());
      XTileStat* ts = reinterpret_cast<XTileStat*>(tile_stat_.get());
      XTileAgg* ta = reinterpret_cast<XTileAgg*>(tile_agg_.get());
      if (ntiles_ > 0) {
        k_xstat<<<ntiles_, kXThreads, 0, st>>>(c1, tc, ts, skip_);
        k_xagg<<<ntiles_, kXThreads, 0, st>>>(c1, tc, ts, ta, skip_);
        B200_LAUNCH_CHECK();
      }
      if (n1_ > 0) {
        k_xchain<<<(n1_ + 3) / 4, 128, 0, st>>>(c1, n1_, ta, skip_);
        B200_LAUNCH_CHECK();
      }
      if (n2_ > 0) {
        k_xchain<<<(n2_ + 3) / 4, 128, 0, st>>>(reinterpret_cast<const XChain*>(seg2_.get()), n2_, ta, skip_);
        B200_LAUNCH_CHECK();
      }
    } else if (nt_ > 0) {
      k_tree1<<<nt_ * kTreeBlocks, kBlock, 0, st>>>(reinterpret_cast<const TreeSeg*>(tseg_.get()), nt_,
                                                    partials_.get(), skip_);
      B200_LAUNCH_CHECK();
      k_tree2<<<nt_, kBlock, 0, st>>>(reinterpret_cast<const TreeSeg*>(tseg_.get()), nt_, partials_.get(), skip_);
      B200_LAUNCH_CHECK();
    }
  }
  int kernel_count() const { return exact_ ? 2 * (ntiles_ > 0) + (n1_ > 0) + (n2_ > 0) : (nt_ > 0 ? 2 : 0); }
  bool empty() const { return jobs_.empty(); }

 private:
  struct Job {
    const double* t;
    long long lo, hi;
    double init;
    SumOrder order;
    double* out;
  };
  // Stream-ordered copy from pageable memory: cudaMemcpyAsync stages the source before it
  // returns, and the device copy lands before any later work on `st`. (A plain cudaMemcpy on the
  // legacy stream may return before the copy lands and is not ordered with a non-blocking `st`.)
  template <class S>
  static void upload(const std::vector<S>& v, DevBuf<unsigned char>& dst, cudaStream_t st) {
    dst.alloc(v.size() * sizeof(S) + 1);
    if (!v.empty())
      B200_CHECK(cudaMemcpyAsync(dst.get(), v.data(), v.size() * sizeof(S), cudaMemcpyHostToDevice, st));
  }
  std::vector<Job> jobs_;
  bool exact_ = false;
  const int* skip_ = nullptr;
  DevBuf<unsigned char> seg1_, seg2_, tseg_, tile_chain_;
  mutable DevBuf<unsigned char> tile_stat_, tile_agg_;
  mutable DevBuf<double> partials_;
  int n1_ = 0, n2_ = 0, nt_ = 0, ntiles_ = 0;
};

}  // namespace b200
