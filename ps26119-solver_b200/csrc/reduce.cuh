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
//   k_xchain  one warp per chain walks its tiles in order with the EXACT s: a tile is committed
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
  int tile0, ntiles;  // this chain's tiles in the tile arrays (ntiles = 0: windows only)
};
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
struct XTileAgg {
  double u;  // the binade's ulp the run is counted in (0: no guess)
  XRun r;
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
  __shared__ XRun shr[kXThreads / 32];
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
    if (threadIdx.x == 0) {
      XTileAgg g;
      g.u = 0.0;
      g.r = x_identity();
      g.r.bad = 1;
      ag[tile] = g;
    }
    return;
  }
  const double inv_u = x_pow2(52 - e0);
  const long long i0 = a + static_cast<long long>(threadIdx.x) * kXPer;
  double v[kXPer];
  int cnt = 0;
#pragma unroll
  for (int q = 0; q < kXPer; ++q) {
    v[q] = i0 + q < b ? c.t[i0 + q] : 0.0;
    cnt += i0 + q < b ? 1 : 0;
  }
  XRun r = x_run_of(v, cnt, inv_u);
  // ordered reduction: lanes, then the block's warps in order
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int off = 1; off < 32; off <<= 1) {
    const XRun o = x_shfl_down(r, off);
    if ((lane & (2 * off - 1)) == 0 && lane + off < 32) r = x_compose(r, o);
  }
  if (lane == 0) shr[wid] = r;
  __syncthreads();
  if (threadIdx.x == 0) {
    XRun t = shr[0];
    for (int w = 1; w < kXThreads / 32; ++w) t = x_compose(t, shr[w]);
    XTileAgg g;
    g.u = x_pow2(e0 - 52);
    g.r = t;
    ag[tile] = g;
  }
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
    const int p0 = static_cast<int>(S0 & 1);
    const long long i0 = pos + static_cast<long long>(lane) * kXPer;
    double v[kXPer];
    int cnt = 0;
#pragma unroll
    for (int q = 0; q < kXPer; ++q) {
      v[q] = i0 + q < b ? t[i0 + q] : 0.0;
      cnt += i0 + q < b ? 1 : 0;
    }
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
  }
  return s;
}

// One warp per chain (4 warps per block): tiles in order (committed whole when valid for the
// exact s), the rest walked in windows. The tile summaries are brought into shared memory 32 at a
// time, so the walk over them waits on no global load.
constexpr int kXChainWarps = 4;
static __global__ void __launch_bounds__(32 * kXChainWarps) k_xchain(const XChain* ch, int nch, const XTileAgg* ag,
                                                                      const int* skip) {
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
    for (int g0 = 0; g0 < c.ntiles; g0 += 32) {
      const int cnt = c.ntiles - g0 < 32 ? c.ntiles - g0 : 32;
      __syncwarp();
      if (lane < cnt) sg[wl][lane] = ag[c.tile0 + g0 + lane];
      __syncwarp();
      for (int j = 0; j < cnt; ++j) {
        // lane 0 decides from the tile's summary; every lane follows its decision
        int commit = 0;
        if (lane == 0) {
          const XTileAgg& G = sg[wl][j];
          int e;
          if (!G.r.bad && G.u != 0.0 && x_binade(s, e) && x_pow2(e - 52) == G.u) {
            const long long S0 = static_cast<long long>(s * x_pow2(52 - e));
            const bool odd = (S0 & 1) != 0;
            const long long mn = odd ? G.r.mn[1] : G.r.mn[0], mx = odd ? G.r.mx[1] : G.r.mx[0];
            if (x_inside(S0, S0 + mn) && x_inside(S0, S0 + mx)) {
              s = static_cast<double>(S0 + (odd ? G.r.K[1] : G.r.K[0])) * G.u;
              commit = 1;
            }
          }
        }
        commit = __shfl_sync(kFull, commit, 0);
        s = __shfl_sync(kFull, s, 0);
        if (!commit) {
          long long a, b;
          x_tile_range(c, c.tile0 + g0 + j, a, b);
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
        k_xchain<<<(n1_ + kXChainWarps - 1) / kXChainWarps, 32 * kXChainWarps, 0, st>>>(c1, n1_, ta, skip_);
        B200_LAUNCH_CHECK();
      }
      if (n2_ > 0) {
        k_xchain<<<(n2_ + kXChainWarps - 1) / kXChainWarps, 32 * kXChainWarps, 0, st>>>(
            reinterpret_cast<const XChain*>(seg2_.get()), n2_, ta, skip_);
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
