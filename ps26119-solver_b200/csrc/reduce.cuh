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
// sequential chain's result bit for bit, from one property of round-to-nearest-even: while every
// partial sum stays inside one binade [2^e, 2^(e+1)) (ulp u = 2^(e−52)), each partial sum is an
// integer multiple S·u, and fl(S·u + t) = (S + k)·u with k = rint(t/u) — or, when t/u = f + ½ is a
// tie, k = f or f + 1, whichever makes S + k even. So inside such a run the chain is an integer
// walk whose only dependence on the past is the parity of S: a run of terms is summarised by its
// effect for each of the two parities (XRun), and effects compose associatively. So:
//   k_xstat   per tile of kXTile terms: an approximate fp64 sum and the approximate range of the
//             tile's running sums (any order; only used to guess each tile's binade);
//   k_xagg    per tile: the guessed binade's u from the approximate start (the approximate sums
//             of the chain's earlier tiles), then the tile's XRun (exact int64: change of S, its
//             lowest and highest running value, parity after, per parity before); a term with
//             |t/u| ≥ 2^51 (or non-finite) marks the tile;
//   k_xgroup  per group of kXGroup consecutive tiles of a long chain: the composition of the
//             tiles' XRuns when all of them count in one grid with no split and no bad term;
//   k_xchain  one warp per chain walks its groups, then its tiles, in order with the EXACT s: a
//             run of whole groups is committed like one tile (below) as far as every running S
//             provably stays inside the binade; the first group that is not is walked tile by
//             tile. A tile is committed
//             as s ← (S0 + K[S0 mod 2])·u when s = S0·u lies in the guessed binade and every
//             running S stays within [2^52 + 1, 2^53 − 1] (then each exact partial sum lies inside
//             the binade, at least u/2 from its ends, and rounds to that grid); any other tile is
//             walked in windows of 256 terms with the same exact test per term (a warp scan of
//             the lanes' XRuns), committing the valid prefix and adding the first failing term
//             with one plain fp64 addition (so binade changes, zeros, subnormals, infinities and
//             NaN get exactly the sequential chain's arithmetic).
// The approximations only choose between two exact paths; the result never depends on them.
constexpr int kXTile = 2048;    // terms per tile (8 per thread of a 256-thread block)
constexpr int kXPer = 8;        // terms per thread (tiles) and per lane (windows)
constexpr int kXThreads = kXTile / kXPer;

struct XChain {
  const double* t;
  long long lo, hi;  // terms t[lo, hi)
  double init;
  double* out;
  int tile0, ntiles;    // this chain's tiles in the tile arrays (ntiles = 0: windows only)
  int group0, ngroups;  // its groups of kXGroup tiles in the group array (ngroups = 0: none)
};
constexpr int kXGroup = 32;  // tiles per group (one warp lane per tile)
constexpr int kXChainWarps = 4;  // warps per block of k_xchain / k_xgroup
struct XTileStat {
  double sum, pmin, pmax;  // approximate: Σ t, min / max of the running sums from the tile start
  int bad;                 // a non-finite term
  int pad;
};
// The effect of a run of terms on S (the partial sum in units of u), for S even (index 0) and
// odd (1) at the run's start: K the change of S, mn / mx the lowest / highest running change
// over positions 1…len (LLONG_MAX / LLONG_MIN for an empty run), out the parity after; bad: a
// term the integer form cannot take (|t/u| ≥ 2^51 or non-finite).
struct XRun {
  long long K[2], mn[2], mx[2];
  int out[2];
  int bad;
};
// A tile's summary: its terms before `split` counted in the grid u (the binade of the tile's
// approximate start), the term at `split` (where the approximate running sum leaves that binade;
// split = −1: it never does) added as a plain fp64 addition, the terms after it counted in the
// grid u1 of the binade the running sum moved to. u = 0: no usable guess (bad is set).
struct XTileAgg {
  double u, u1;
  XRun pre, suf;
  int split;
  int pad;
};
// A group of kXGroup consecutive tiles of one chain that all count in the same grid u with no
// split and no bad term: the composition of their runs. u = 0: the group cannot be taken whole.
struct XGroupAgg {
  double u;
  XRun run;
};

constexpr long long kX52 = 1LL << 52, kX53 = 1LL << 53;

__device__ __forceinline__ XRun x_identity() {
  XRun r;
  r.K[0] = r.K[1] = 0;
  r.mn[0] = r.mn[1] = LLONG_MAX;
  r.mx[0] = r.mx[1] = LLONG_MIN;
  r.out[0] = 0, r.out[1] = 1;
  r.bad = 0;
  return r;
}
// a then b (selects instead of indexing with a.out[p], so everything stays in registers)
__device__ __forceinline__ XRun x_compose(const XRun& a, const XRun& b) {
  XRun r;
  r.bad = a.bad | b.bad;
#pragma unroll
  for (int p = 0; p < 2; ++p) {
    const bool q = a.out[p] != 0;
    const long long bK = q ? b.K[1] : b.K[0], bmn = q ? b.mn[1] : b.mn[0], bmx = q ? b.mx[1] : b.mx[0];
    r.K[p] = a.K[p] + bK;
    r.mn[p] = bmn == LLONG_MAX ? a.mn[p] : min(a.mn[p], a.K[p] + bmn);
    r.mx[p] = bmx == LLONG_MIN ? a.mx[p] : max(a.mx[p], a.K[p] + bmx);
    r.out[p] = q ? b.out[1] : b.out[0];
  }
  return r;
}
__device__ __forceinline__ XRun x_shfl_down(const XRun& v, int off) {
  XRun r;
#pragma unroll
  for (int p = 0; p < 2; ++p) {
    r.K[p] = __shfl_down_sync(kFull, v.K[p], off);
    r.mn[p] = __shfl_down_sync(kFull, v.mn[p], off);
    r.mx[p] = __shfl_down_sync(kFull, v.mx[p], off);
  }
  const int packed = __shfl_down_sync(kFull, v.out[0] | (v.out[1] << 1) | (v.bad << 2), off);
  r.out[0] = packed & 1, r.out[1] = (packed >> 1) & 1, r.bad = packed >> 2;
  return r;
}
__device__ __forceinline__ XRun x_shfl_up(const XRun& v, int off) {
  XRun r;
#pragma unroll
  for (int p = 0; p < 2; ++p) {
    r.K[p] = __shfl_up_sync(kFull, v.K[p], off);
    r.mn[p] = __shfl_up_sync(kFull, v.mn[p], off);
    r.mx[p] = __shfl_up_sync(kFull, v.mx[p], off);
  }
  const int packed = __shfl_up_sync(kFull, v.out[0] | (v.out[1] << 1) | (v.bad << 2), off);
  r.out[0] = packed & 1, r.out[1] = (packed >> 1) & 1, r.bad = packed >> 2;
  return r;
}

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
// A term in units of u (inv_u = 1/u, powers of two: t·inv_u is exact unless it under/overflows):
// false for |t/u| ≥ 2^51 or a non-finite t; else kf = rint(t/u), or floor(t/u) for a tie.
__device__ __forceinline__ bool x_term(double t, double inv_u, long long& kf, bool& tie) {
  const double q = t * inv_u;
  if (!(fabs(q) < 2251799813685248.0)) return false;  // 2^51; also NaN / inf
  const double f = floor(q);
  tie = q - f == 0.5;
  kf = static_cast<long long>(tie ? f : rint(q));
  return true;
}
// The step of S with parity `par` for a term (kf, tie): returns k; par becomes S + k's parity.
__device__ __forceinline__ long long x_step(long long kf, bool tie, int& par) {
  long long k = kf;
  if (tie) {
    k += (par + kf) & 1;  // to the even neighbour
    par = 0;
  } else {
    par = static_cast<int>((par + k) & 1);
  }
  return k;
}
// The XRun of up to kXPer terms v[0, cnt).
__device__ __forceinline__ XRun x_run_of(const double* v, int cnt, double inv_u) {
  XRun r = x_identity();
  long long kf[kXPer];
  bool tie[kXPer];
#pragma unroll
  for (int q = 0; q < kXPer; ++q)
    if (q < cnt && !x_term(v[q], inv_u, kf[q], tie[q])) r.bad = 1, kf[q] = 0, tie[q] = false;
#pragma unroll
  for (int p = 0; p < 2; ++p) {
    int par = p;
    long long K = 0;
#pragma unroll
    for (int q = 0; q < kXPer; ++q)
      if (q < cnt) {
        K += x_step(kf[q], tie[q], par);
        r.mn[p] = min(r.mn[p], K);
        r.mx[p] = max(r.mx[p], K);
      }
    r.K[p] = K;
    r.out[p] = par;
  }
  return r;
}
// The XRun of the terms v[q] whose bit q is set in `mask` (the others left out).
__device__ __forceinline__ XRun x_run_masked(const double* v, unsigned mask, double inv_u) {
  XRun r = x_identity();
  long long kf[kXPer];
  bool tie[kXPer];
#pragma unroll
  for (int q = 0; q < kXPer; ++q) {
    kf[q] = 0, tie[q] = false;
    if (((mask >> q) & 1u) && !x_term(v[q], inv_u, kf[q], tie[q])) r.bad = 1, kf[q] = 0, tie[q] = false;
  }
#pragma unroll
  for (int p = 0; p < 2; ++p) {
    int par = p;
    long long K = 0;
#pragma unroll
    for (int q = 0; q < kXPer; ++q)
      if ((mask >> q) & 1u) {
        K += x_step(kf[q], tie[q], par);
        r.mn[p] = min(r.mn[p], K);
        r.mx[p] = max(r.mx[p], K);
      }
    r.K[p] = K;
    r.out[p] = par;
  }
  return r;
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

// Ordered reduction of the block's per-thread runs (thread order); the result in thread 0.
__device__ __forceinline__ XRun x_block_ordered(XRun r, XRun* sh) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int off = 1; off < 32; off <<= 1) {
    const XRun o = x_shfl_down(r, off);
    if ((lane & (2 * off - 1)) == 0 && lane + off < 32) r = x_compose(r, o);
  }
  __syncthreads();
  if (lane == 0) sh[wid] = r;
  __syncthreads();
  if (threadIdx.x == 0)
    for (int w = 1; w < kXThreads / 32; ++w) r = x_compose(r, sh[w]);
  return r;
}

static __global__ void __launch_bounds__(kXThreads) k_xagg(const XChain* ch, const int* tile_chain,
                                                           const XTileStat* st, XTileAgg* ag, const int* skip) {
  __shared__ double shd[32];
  __shared__ int shi[32];
  __shared__ XRun shr[kXThreads / 32];
  __shared__ double sh_at_split;
  if (skip && *skip) return;
  const int tile = blockIdx.x;
  const XChain c = ch[tile_chain[tile]];
  long long a, b;
  x_tile_range(c, tile, a, b);
  // the approximate running sum at the tile's start (the approximate sums of the earlier tiles)
  double pre = 0.0;
  for (int k = c.tile0 + static_cast<int>(threadIdx.x); k < tile; k += blockDim.x) pre += st[k].sum;
  pre = x_block_reduce(pre, [](double x, double y) { return x + y; }, shd);
  const double s0 = c.init + pre;
  int e0;
  XTileAgg g;
  g.u = g.u1 = 0.0;
  g.split = -1;
  g.pad = 0;
  g.pre = g.suf = x_identity();
  if (!x_binade(s0, e0)) {  // uniform over the block
    if (threadIdx.x == 0) g.pre.bad = 1, ag[tile] = g;
    return;
  }
  const long long i0 = a + static_cast<long long>(threadIdx.x) * kXPer;
  double v[kXPer];
  double run = 0.0;
#pragma unroll
  for (int q = 0; q < kXPer; ++q) {
    v[q] = i0 + q < b ? c.t[i0 + q] : 0.0;
    run += v[q];
  }
  // approximate running sums: the first position whose running sum leaves e0's binade
  double total;
  const double before = x_block_excl(run, total, shd);
  const int base = static_cast<int>(threadIdx.x) * kXPer;
  int first = INT_MAX;
  double acc = s0 + before;
#pragma unroll
  for (int q = 0; q < kXPer; ++q)
    if (i0 + q < b) {
      acc += v[q];
      int e;
      if (first == INT_MAX && !(x_binade(acc, e) && e == e0 && (acc > 0) == (s0 > 0))) first = base + q;
    }
  const int split = x_block_reduce(first, [](int x, int y) { return x < y ? x : y; }, shi);
  // the binade after the split: all later approximate running sums must share it
  int e1 = e0, ok1 = 1;
  if (split != INT_MAX) {
    if (split >= base && split < base + kXPer) {
      double acc2 = s0 + before;
#pragma unroll
      for (int q = 0; q < kXPer; ++q)
        if (q <= split - base) acc2 += v[q];
      sh_at_split = acc2;
    }
    __syncthreads();
    const double after = sh_at_split;
    ok1 = x_binade(after, e1) ? 1 : 0;
    double acc3 = s0 + before;
#pragma unroll
    for (int q = 0; q < kXPer; ++q)
      if (i0 + q < b) {
        acc3 += v[q];
        int e;
        if (base + q > split && !(x_binade(acc3, e) && e == e1 && (acc3 > 0) == (after > 0))) ok1 = 0;
      }
    ok1 = x_block_reduce(ok1, [](int x, int y) { return x & y; }, shi);
  }
  unsigned mpre = 0, msuf = 0;
#pragma unroll
  for (int q = 0; q < kXPer; ++q)
    if (i0 + q < b) {
      if (base + q < split) mpre |= 1u << q;
      else if (split != INT_MAX && base + q > split) msuf |= 1u << q;
    }
  const XRun rp = x_block_ordered(x_run_masked(v, mpre, x_pow2(52 - e0)), shr);
  XRun rs = x_identity();
  if (split != INT_MAX && ok1) rs = x_block_ordered(x_run_masked(v, msuf, x_pow2(52 - e1)), shr);
  if (threadIdx.x == 0) {
    g.u = x_pow2(e0 - 52);
    g.pre = rp;
    if (split != INT_MAX) {
      g.split = split;
      g.u1 = ok1 ? x_pow2(e1 - 52) : 0.0;
      g.suf = rs;
      if (!ok1) g.suf.bad = 1;
    }
    ag[tile] = g;
  }
}

// The chain over t[a, b) from the exact partial sum s, by windows of 32·kXPer terms (all 32 lanes
// call it with the same s and return the same s). The next window's terms are requested before
// the current one is evaluated, so a run of valid windows waits on memory once.
__device__ __forceinline__ void x_load_window(const double* __restrict__ t, long long pos, long long b,
                                              double (&v)[kXPer]) {
  const long long i0 = pos + static_cast<long long>(threadIdx.x & 31) * kXPer;
#pragma unroll
  for (int q = 0; q < kXPer; ++q) v[q] = i0 + q < b ? t[i0 + q] : 0.0;
}
__device__ __forceinline__ double x_window_walk(const double* __restrict__ t, long long a, long long b, double s) {
  const int lane = threadIdx.x & 31;
  long long pos = a;
  double v[kXPer], nx[kXPer];
  x_load_window(t, pos, b, v);
  while (pos < b) {
    int e;
    if (!x_binade(s, e)) {  // zero, subnormal, inf or NaN: a plain sequential run of up to 32 terms
      const long long rem = b - pos;
      const int cnt = rem < 32 ? static_cast<int>(rem) : 32;
      const double w = lane < cnt ? t[pos + lane] : 0.0;
      for (int j = 0; j < cnt; ++j) s += __shfl_sync(kFull, w, j);
      pos += cnt;
      x_load_window(t, pos, b, v);
      continue;
    }
    x_load_window(t, pos + 32LL * kXPer, b, nx);  // the next window, if this one is valid
    const double u = x_pow2(e - 52), inv_u = x_pow2(52 - e);
    const long long S0 = static_cast<long long>(s * inv_u);
    const int p0 = static_cast<int>(S0 & 1);
    const long long i0 = pos + static_cast<long long>(lane) * kXPer;
    int cnt = 0;
#pragma unroll
    for (int q = 0; q < kXPer; ++q) cnt += i0 + q < b ? 1 : 0;
    XRun inc = x_run_of(v, cnt, inv_u);  // warp inclusive scan in lane order
    for (int off = 1; off < 32; off <<= 1) {
      const XRun o = x_shfl_up(inc, off);
      if (lane >= off) inc = x_compose(o, inc);
    }
    XRun ex = x_shfl_up(inc, 1);
    if (lane == 0) ex = x_identity();
    // this lane's terms with its exact incoming state: the first invalid position
    long long run = p0 ? ex.K[1] : ex.K[0], committed = run;
    int par = p0 ? ex.out[1] : ex.out[0], first = kXPer;
    double vf = 0.0;
#pragma unroll
    for (int q = 0; q < kXPer; ++q) {
      if (q < cnt && first == kXPer) {
        long long kf;
        bool tie;
        bool ok = x_term(v[q], inv_u, kf, tie);
        if (ok) {
          int p2 = par;
          const long long k = x_step(kf, tie, p2);
          ok = x_inside(S0, S0 + run + k);
          if (ok) run += k, par = p2;
        }
        if (!ok) first = q, committed = run, vf = v[q];
      }
    }
    const unsigned fail = __ballot_sync(kFull, first < kXPer);
    if (fail == 0) {
      const long long total = __shfl_sync(kFull, p0 ? inc.K[1] : inc.K[0], 31);
      s = static_cast<double>(S0 + total) * u;
      pos = pos + 32LL * kXPer < b ? pos + 32LL * kXPer : b;
#pragma unroll
      for (int q = 0; q < kXPer; ++q) v[q] = nx[q];
      continue;
    }
    const int fl = __ffs(fail) - 1;
    const int fq = __shfl_sync(kFull, first, fl);
    committed = __shfl_sync(kFull, committed, fl);
    vf = __shfl_sync(kFull, vf, fl);
    s = static_cast<double>(S0 + committed) * u;  // the valid prefix (nothing when it is empty)
    s += vf;                                      // the failing term, as the sequential chain adds it
    const long long f = static_cast<long long>(fl) * kXPer + fq;
    pos += f + 1;
    if (f < kXPer) {  // little progress: a plain run of up to 32 terms before the next window
      const long long rem = b - pos;
      const int n2 = rem <= 0 ? 0 : (rem < 32 ? static_cast<int>(rem) : 32);
      const double w = lane < n2 ? t[pos + lane] : 0.0;
      for (int j = 0; j < n2; ++j) s += __shfl_sync(kFull, w, j);
      pos += n2;
    }
    x_load_window(t, pos, b, v);
  }
  return s;
}

// Commits the run r (counted in the grid u) onto the exact s when s lies in u's binade and every
// running S stays inside it; returns false (s unchanged) otherwise.
__device__ __forceinline__ bool x_commit(double& s, double u, const XRun& r) {
  int e;
  if (r.bad || u == 0.0 || !x_binade(s, e) || x_pow2(e - 52) != u) return false;
  const long long S0 = static_cast<long long>(s * x_pow2(52 - e));
  const bool odd = (S0 & 1) != 0;
  if (r.mn[0] == LLONG_MAX) return true;  // an empty run
  const long long mn = odd ? r.mn[1] : r.mn[0], mx = odd ? r.mx[1] : r.mx[0];
  if (!x_inside(S0, S0 + mn) || !x_inside(S0, S0 + mx)) return false;
  s = static_cast<double>(S0 + (odd ? r.K[1] : r.K[0])) * u;
  return true;
}

// One warp per group of kXGroup tiles: lane l composes tile l's run in order (an ordered warp
// reduction); the group is whole when every tile counts in lane 0's grid, has no split and no bad
// term. group_chain[g]: the chain of group g.
static __global__ void __launch_bounds__(32 * kXChainWarps) k_xgroup(const XChain* ch, const int* group_chain,
                                                                      int ngroups, const XTileAgg* ag,
                                                                      XGroupAgg* gg, const int* skip) {
  if (skip && *skip) return;
  const int g = static_cast<int>((blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (g >= ngroups) return;
  const XChain c = ch[group_chain[g]];
  const int tile = c.tile0 + (g - c.group0) * kXGroup + lane;
  const bool mine = tile < c.tile0 + c.ntiles;
  XRun r = x_identity();
  double u = 0.0;
  bool ok = true;
  if (mine) {
    const XTileAgg& G = ag[tile];
    r = G.pre;
    u = G.u;
    ok = !G.pre.bad && G.split < 0 && G.u != 0.0;
  }
  const double u0 = __shfl_sync(kFull, u, 0);
  ok = __all_sync(kFull, !mine || (ok && u == u0)) != 0;
  for (int off = 1; off < 32; off <<= 1) {  // ordered reduction: lane 0 ends with tiles 0 … 31
    const XRun o = x_shfl_down(r, off);
    if ((lane & (2 * off - 1)) == 0 && lane + off < 32) r = x_compose(r, o);
  }
  if (lane == 0) {
    XGroupAgg out;
    out.u = ok ? u0 : 0.0;
    out.run = r;
    gg[g] = out;
  }
}

// One warp per chain (4 warps per block): tiles in order, the rest walked in windows. The tile
// summaries are brought into shared memory 32 at a time; the lanes take one tile each and a warp
// scan of their XRuns gives every tile its exact incoming S, so one step commits every tile up
// to the first one that is not valid for the exact s or whose running sum changes binade. Such a
// tile is taken on its own: its part before the change, the changing term as a plain addition,
// its part after; what does not commit is walked in windows.
static __global__ void __launch_bounds__(32 * kXChainWarps) k_xchain(const XChain* ch, int nch, const XTileAgg* ag,
                                                                      const XGroupAgg* gg, const int* skip) {
  __shared__ XTileAgg sg[kXChainWarps][32];
  if (skip && *skip) return;
  const int warp = static_cast<int>((blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31, wl = threadIdx.x >> 5;
  if (warp >= nch) return;
  const XChain c = ch[warp];
  double s = c.init;
  if (c.ntiles == 0) {
    s = x_window_walk(c.t, c.lo, c.hi, s);
  } else {
    int g0 = 0;  // the next tile, a multiple of kXGroup
    while (g0 < c.ntiles) {
      if (gg && c.ngroups > 0) {
        // whole groups first: up to 32 groups (32 · kXGroup tiles) per scan, committed up to the
        // first group that is not whole, not in this binade, or whose running sum leaves it
        const int gi = g0 / kXGroup;
        const int cntg = c.ngroups - gi < 32 ? c.ngroups - gi : 32;
        int e;
        const bool have = x_binade(s, e);
        const double u = have ? x_pow2(e - 52) : 0.0;
        const long long S0 = have ? static_cast<long long>(s * x_pow2(52 - e)) : 0;
        const int p0 = static_cast<int>(S0 & 1);
        XRun r = x_identity();
        bool mine_ok = false;
        if (lane < cntg) {
          const XGroupAgg& G = gg[c.group0 + gi + lane];
          mine_ok = have && G.u == u && !G.run.bad;
          r = G.run;
        }
        XRun inc = r;
        for (int off = 1; off < 32; off <<= 1) {
          const XRun o = x_shfl_up(inc, off);
          if (lane >= off) inc = x_compose(o, inc);
        }
        XRun ex = x_shfl_up(inc, 1);
        if (lane == 0) ex = x_identity();
        const long long Kb = p0 ? ex.K[1] : ex.K[0];
        const int pb = p0 ? ex.out[1] : ex.out[0];
        bool valid = false;
        if (mine_ok) {
          const long long mn = pb ? r.mn[1] : r.mn[0], mx = pb ? r.mx[1] : r.mx[0];
          valid = x_inside(S0, S0 + Kb + mn) && x_inside(S0, S0 + Kb + mx);
        }
        const unsigned bad = __ballot_sync(kFull, lane < cntg && !valid);
        const int f = bad ? __ffs(bad) - 1 : cntg;  // first group not committed
        if (f > 0) {
          const long long K = f < 32 ? __shfl_sync(kFull, Kb, f & 31) : __shfl_sync(kFull, p0 ? inc.K[1] : inc.K[0], 31);
          s = static_cast<double>(S0 + K) * u;
        }
        g0 += f * kXGroup;
        if (f == cntg) continue;  // every loaded group taken: the next 32 groups
      }
      if (g0 >= c.ntiles) break;
      // tiles g0 … g0 + 31 one by one
      const int cnt = c.ntiles - g0 < 32 ? c.ntiles - g0 : 32;
      __syncwarp();
      if (lane < cnt) sg[wl][lane] = ag[c.tile0 + g0 + lane];
      __syncwarp();
      int j = 0;
      while (j < cnt) {
        int e;
        const bool have = x_binade(s, e);
        const double u = have ? x_pow2(e - 52) : 0.0;
        const long long S0 = have ? static_cast<long long>(s * x_pow2(52 - e)) : 0;
        const int p0 = static_cast<int>(S0 & 1);
        // lane l >= j: tile l's run if it stays in this binade; lanes below j: nothing
        XRun r = x_identity();
        bool mine_ok = false;
        if (lane >= j && lane < cnt) {
          const XTileAgg& G = sg[wl][lane];
          mine_ok = have && !G.pre.bad && G.split < 0 && G.u == u;
          r = G.pre;
        }
        XRun inc = r;
        for (int off = 1; off < 32; off <<= 1) {
          const XRun o = x_shfl_up(inc, off);
          if (lane >= off) inc = x_compose(o, inc);
        }
        XRun ex = x_shfl_up(inc, 1);
        if (lane == 0) ex = x_identity();
        const long long Kb = p0 ? ex.K[1] : ex.K[0];
        const int pb = p0 ? ex.out[1] : ex.out[0];
        bool valid = false;
        if (mine_ok) {
          const long long mn = pb ? r.mn[1] : r.mn[0], mx = pb ? r.mx[1] : r.mx[0];
          valid = x_inside(S0, S0 + Kb + mn) && x_inside(S0, S0 + Kb + mx);
        }
        const unsigned bad = __ballot_sync(kFull, lane >= j && lane < cnt && !valid);
        const int f = bad ? __ffs(bad) - 1 : cnt;  // first tile not committed
        if (f > j) {  // tiles j … f−1: S0 plus the exclusive change at tile f (or the total)
          const long long K = f < 32 ? __shfl_sync(kFull, Kb, f & 31) : __shfl_sync(kFull, p0 ? inc.K[1] : inc.K[0], 31);
          s = static_cast<double>(S0 + K) * u;
        }
        if (f < cnt) {  // tile f on its own
          long long a, b;
          x_tile_range(c, c.tile0 + g0 + f, a, b);
          long long resume = a;
          if (lane == 0) {
            const XTileAgg& G = sg[wl][f];
            double s2 = s;
            if (x_commit(s2, G.u, G.pre)) {
              if (G.split < 0) {
                resume = b;
              } else {
                s2 += c.t[a + G.split];  // the term that changes the binade, as the chain adds it
                resume = a + G.split + 1;
                if (x_commit(s2, G.u1, G.suf)) resume = b;
              }
              s = s2;
            }
          }
          s = __shfl_sync(kFull, s, 0);
          resume = __shfl_sync(kFull, resume, 0);
          if (resume < b) s = x_window_walk(c.t, resume, b, s);
        }
        j = f + 1;
      }
      g0 += 32;
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
        XChain c{t, lo, hi, init, out, static_cast<int>(tile_chain.size()), 0, 0, 0};
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
          phase2.push_back({part, 0, chunks, j.init, j.out, 0, 0, 0, 0});
          ++slot;
        }
      }
      ntiles_ = static_cast<int>(tile_chain.size());
      // chains of more than one group of tiles also get group summaries (k_xgroup)
      std::vector<int> group_chain;
      for (std::size_t k = 0; k < phase1.size(); ++k) {
        XChain& c = phase1[k];
        if (c.ntiles <= kXGroup) continue;
        c.group0 = static_cast<int>(group_chain.size());
        c.ngroups = (c.ntiles + kXGroup - 1) / kXGroup;
        for (int g = 0; g < c.ngroups; ++g) group_chain.push_back(static_cast<int>(k));
      }
      ngroups_ = static_cast<int>(group_chain.size());
      upload(group_chain, group_chain_, st);
      group_agg_.alloc(static_cast<std::size_t>(ngroups_ > 0 ? ngroups_ : 1) * sizeof(XGroupAgg));
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
      XGroupAgg* tg = ngroups_ > 0 ? reinterpret_cast<XGroupAgg*>(group_agg_.get()) : nullptr;
      if (ntiles_ > 0) {
        k_xstat<<<ntiles_, kXThreads, 0, st>>>(c1, tc, ts, skip_);
        k_xagg<<<ntiles_, kXThreads, 0, st>>>(c1, tc, ts, ta, skip_);
        B200_LAUNCH_CHECK();
      }
      if (ngroups_ > 0) {
        k_xgroup<<<(ngroups_ + kXChainWarps - 1) / kXChainWarps, 32 * kXChainWarps, 0, st>>>(
            c1, reinterpret_cast<const int*>(group_chain_.get()), ngroups_, ta, tg, skip_);
        B200_LAUNCH_CHECK();
      }
      if (n1_ > 0) {
        k_xchain<<<(n1_ + kXChainWarps - 1) / kXChainWarps, 32 * kXChainWarps, 0, st>>>(c1, n1_, ta, tg, skip_);
        B200_LAUNCH_CHECK();
      }
      if (n2_ > 0) {
        k_xchain<<<(n2_ + kXChainWarps - 1) / kXChainWarps, 32 * kXChainWarps, 0, st>>>(
            reinterpret_cast<const XChain*>(seg2_.get()), n2_, ta, nullptr, skip_);
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
  int kernel_count() const {
    return exact_ ? 2 * (ntiles_ > 0) + (ngroups_ > 0) + (n1_ > 0) + (n2_ > 0) : (nt_ > 0 ? 2 : 0);
  }
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
  DevBuf<unsigned char> seg1_, seg2_, tseg_, tile_chain_, group_chain_;
  mutable DevBuf<unsigned char> tile_stat_, tile_agg_, group_agg_;
  mutable DevBuf<double> partials_;
  int n1_ = 0, n2_ = 0, nt_ = 0, ntiles_ = 0, ngroups_ = 0;
};

}  // namespace b200
