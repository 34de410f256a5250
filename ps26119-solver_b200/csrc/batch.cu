// batch.cu — lockstep r²HPDHG over K scenarios that share one constraint matrix
// (≙ ps26119::solve_batch, reference src/pdhg/batch.cpp:129-441), on the device.
//
// Layout: every per-scenario vector is an interleaved (rows × W) block, element (r, t) at
// r·W + t, where W is the number of scenarios still running ("slots"). A nonzero of Ã is read
// once per iteration and multiplied with W contiguous values: the reference's SpMM
// (spmm_fixed, batch.cpp:40-57) as one coalesced W-wide gather per nonzero. When scenarios
// finish, every block is compacted to the remaining slots (compact, batch.cpp:94-101).
//
// Per iteration: k_bspmm with the primal epilogue (Ãᵀy, projection, reflection, Halpern) and
// with the dual epilogue (Ãx̄, dual update): two launches. The per-slot step sizes and Halpern
// counters live in device arrays written at each check. An epoch of K iterations is one CUDA
// graph (two variants: with and without the r⁰ section after the first step), captured for the
// current slot count and blocks and captured again after a compaction moves them.
// Per check (every K iterations): fixed-point residuals (one SpMM), restart distances, the
// KKT statistics of every slot on the ORIGINAL matrix (two SpMMs), all per-slot sums in one
// launch, one download of W×32 doubles; the host then takes the reference's per-scenario
// decisions (termination, restart, PID primal weight).
//
// Sums: exact mode walks each slot's terms in the reference's order (one lane per slot,
// sequential over rows), so every scenario's trajectory is bit-identical to the reference;
// fast mode uses a fixed two-level split (deterministic run to run, different rounding).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <limits>
#include <string>

#include "batch.hpp"

#include <type_traits>
#include "checks.cuh"
#include "problem.cuh"
#include "tune.hpp"

namespace b200 {
namespace {

constexpr int kMaxSlots = 256;  // slots of one lockstep group (k_bspmm: 32 lanes × 8)
constexpr int kRes = 32;        // per-slot result block (doubles)
enum BSlot : int {
  kBPx0 = 0, kBPy0, kBCr0,  // residual after the first step of an epoch
  kBPx, kBPy, kBCr,         // residual at the check
  kBDxn, kBDyn,             // restart distances ‖x̂ − x0‖², ‖ŷ − y0‖²
  kBRp2, kBD, kBRd2, kBP,   // kkt_general sums
  kBB2, kBC2,               // kkt_general ‖b‖², ‖c‖² (constant per scenario)
  kBSb2, kBSc2,             // bound / objective rescaling sums (setup)
  kBPmax = 24, kBDmax, kBCinf
};
constexpr double kFirstOrderFast = 1e-4;
constexpr double kVerifyPrimal = 1e-6, kVerifyDual = 1e-6, kVerifyGap = 1e-6;

// ---------------------------------------------------------------------------------- SpMM
// Y(rows × W) = M · X(cols × W) row by row in CSR order, G = 2^lg lanes per row, S slots per
// lane (slot t = g + s·G). Each (row, slot) sum is the reference's acc[k] += a·x[k] over the
// row's nonzeros in order. Epi::kMax per-slot maxima are folded per warp and then into
// atomic keys (order-independent and exact).
// Latency: an epilogue with `Pre load(q, t)` has its operands loaded before the row walk, and
// the walk loads kBatchNz (col, val) pairs, then their gathers, then adds them in order, so a
// row costs two dependent round trips per kBatchNz nonzeros instead of two per nonzero.
#ifndef B200_BATCH_NZ
#define B200_BATCH_NZ 2
#endif
constexpr int kBatchNz = B200_BATCH_NZ;
// 1: the step epilogues load their streamed operands evict-first and store the block the next
// kernel gathers (x̄, y) evict-last, so that it stays in L2 (as the single-LP kernels do).
#ifndef B200_BATCH_HINTS
#define B200_BATCH_HINTS 1
#endif
template <class T>
__device__ __forceinline__ T bstream(const T* p) {
#if B200_BATCH_HINTS
  return ld_stream(p);
#else
  return *p;
#endif
}
template <class T>
__device__ __forceinline__ void bkeep(T* p, T v) {
#if B200_BATCH_HINTS
  st_keep(p, v);
#else
  *p = v;
#endif
}
struct BNoPre {};
template <class E>
__device__ __forceinline__ auto bload(const E& e, long long q, int t, int) -> decltype(e.load(q, t)) {
  return e.load(q, t);
}
template <class E>
__device__ __forceinline__ BNoPre bload(const E&, long long, int, long) {
  return BNoPre{};
}
template <class E, class P>
__device__ __forceinline__ void bapply(const E& e, long long r, int t, long long q, double acc, double* mx, const P& p) {
  if constexpr (std::is_same<P, BNoPre>::value) e(r, t, q, acc, mx);
  else e(r, t, q, acc, mx, p);
}

// TV / TX: the matrix values and the gathered block in the working precision (double, or float
// in the mixed form's first phase); products and sums in fp64 either way.
template <int S, class Epi, class TV, class TX>
__global__ void __launch_bounds__(256) k_bspmm(int rows, int W, int lg, const int* __restrict__ rp,
                                               const int* __restrict__ col, const TV* __restrict__ val,
                                               const TX* __restrict__ X, Epi epi) {
  const int G = 1 << lg, g = threadIdx.x & (G - 1);
  const long long gid = (blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x) >> lg;
  const long long ng = (static_cast<long long>(gridDim.x) * blockDim.x) >> lg;
  constexpr int NM = Epi::kMax > 0 ? Epi::kMax : 1;
  double mx[S][NM];
#pragma unroll
  for (int s = 0; s < S; ++s)
#pragma unroll
    for (int k = 0; k < NM; ++k) mx[s][k] = 0.0;
  for (long long r = gid; r < rows; r += ng) {
    using Pre = decltype(bload(epi, 0LL, 0, 0));
    Pre pre[S];
#pragma unroll
    for (int s = 0; s < S; ++s) {
      const int t = g + s * G;
      if (t < W) pre[s] = bload(epi, r * W + t, t, 0);
    }
    double acc[S];
#pragma unroll
    for (int s = 0; s < S; ++s) acc[s] = 0.0;
    const int b = rp[r], e = rp[r + 1];
    for (int p = b; p < e; p += kBatchNz) {
      int cc[kBatchNz];
      double aa[kBatchNz];
#pragma unroll
      for (int u = 0; u < kBatchNz; ++u) {
        cc[u] = p + u < e ? col[p + u] : 0;
        aa[u] = p + u < e ? static_cast<double>(val[p + u]) : 0.0;
      }
      double xv[kBatchNz][S];
#pragma unroll
      for (int u = 0; u < kBatchNz; ++u)
#pragma unroll
        for (int s = 0; s < S; ++s) {
          const int t = g + s * G;
          xv[u][s] = (p + u < e && t < W) ? static_cast<double>(X[static_cast<long long>(cc[u]) * W + t]) : 0.0;
        }
#pragma unroll
      for (int u = 0; u < kBatchNz; ++u)
        if (p + u < e)
#pragma unroll
          for (int s = 0; s < S; ++s) acc[s] += aa[u] * xv[u][s];  // in CSR order
    }
#pragma unroll
    for (int s = 0; s < S; ++s) {
      const int t = g + s * G;
      if (t < W) bapply(epi, r, t, r * W + t, acc[s], mx[s], pre[s]);
    }
  }
  if constexpr (Epi::kMax > 0) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int s = 0; s < S; ++s)
#pragma unroll
      for (int k = 0; k < Epi::kMax; ++k) {
        unsigned long long key = mx[s][k] > 0.0 ? nonneg_key(mx[s][k]) : 0ULL;
        for (int off = 16; off >= G; off >>= 1) {
          const unsigned long long o = __shfl_xor_sync(kFull, key, off);
          key = o > key ? o : key;
        }
        const int t = lane + s * G;
        if (lane < G && t < W && key != 0ULL) atomicMax(epi.key(t, k), key);
      }
  }
}

// Primal step of every slot (batch.cpp:331-343), acc = (Ãᵀy)_j, in the working precision T
// (double: the reference's arithmetic; float: the mixed form's first phase, as the single-LP
// engine's fp32 kernels).
template <class T>
struct EpiBPrimal {
  static constexpr int kMax = 0;
  const T *C, *L, *U, *X0;
  const double* tau;
  T *X, *XH, *XB;
  const long long* inner0;
  int step, last;  // last: the epoch's last step
  double a2, b2;
  struct Pre {
    T x, c, l, u, x0;
  };
  __device__ Pre load(long long q, int) const {
    return Pre{bstream(X + q), bstream(C + q), bstream(L + q), bstream(U + q), bstream(X0 + q)};
  }
  __device__ void operator()(long long, int t, long long q, double aty, double*, const Pre& p) const {
    const long long in = inner0[t] + step;
    const T w = static_cast<T>(static_cast<double>(in + 1) / static_cast<double>(in + 2));
    const T x = p.x;
    const T h = ref_clamp<T>(x - static_cast<T>(tau[t]) * (p.c - static_cast<T>(aty)), p.l, p.u);
    // x̂ is read only by the residual, check and restart that follow the epoch's last step and
    // the first step of a slot's Halpern cycle; on the other steps it is not stored
    if (step == last || in == 0) XH[q] = h;
    bkeep(XB + q, static_cast<T>(static_cast<T>(2) * h - x));  // gathered by the dual kernel next
    X[q] = w * (static_cast<T>(a2) * h + static_cast<T>(b2) * x) + (static_cast<T>(1) - w) * p.x0;
  }
};
// Dual step of every slot (batch.cpp:345-358), acc = (Ãx̄)_i.
template <class T>
struct EpiBDual {
  static constexpr int kMax = 0;
  const T *RL, *RU, *Y0;
  const double* sigma;
  T *Y, *YH, *YB;
  const long long* inner0;
  int step, last;
  double a2, b2;
  struct Pre {
    T y, rl, ru, y0;
  };
  __device__ Pre load(long long q, int) const { return Pre{bstream(Y + q), bstream(RL + q), bstream(RU + q), bstream(Y0 + q)}; }
  __device__ void operator()(long long, int t, long long q, double axd, double*, const Pre& p) const {
    const long long in = inner0[t] + step;
    const T w = static_cast<T>(static_cast<double>(in + 1) / static_cast<double>(in + 2));
    const T sg = static_cast<T>(sigma[t]), ax = static_cast<T>(axd);
    const T y = p.y;
    const T v = ax - y / sg;
    const T h = y - sg * ax + sg * ref_clamp<T>(v, p.rl, p.ru);
    if (step == last || in == 0) {  // ŷ, ȳ: read only after those steps (as x̂ above)
      YH[q] = h;
      YB[q] = static_cast<T>(2) * h - y;
    }
    bkeep(Y + q, static_cast<T>(w * (static_cast<T>(a2) * h + static_cast<T>(b2) * y) + (static_cast<T>(1) - w) * p.y0));
  }
};
// Residual rows after adx = Ã·Δx (compute_residuals, batch.cpp:305-318): terms Δy², Δy·(AΔx)
// and, at a check, the restart distance (ŷ − y0)² (batch.cpp:399-403); fp64 terms.
template <class T>
struct EpiBRes {
  static constexpr int kMax = 0;
  const T *YB, *YH, *Y0;
  double *t_py, *t_cr, *t_dyn;
  __device__ void operator()(long long, int, long long q, double adx, double*) const {
    const double dy = static_cast<double>(static_cast<T>(YB[q] - YH[q]));
    t_py[q] = dy * dy;
    t_cr[q] = dy * static_cast<double>(static_cast<T>(adx));
    if (t_dyn) {
      const double e = static_cast<double>(YH[q]) - static_cast<double>(Y0[q]);
      t_dyn[q] = e * e;
    }
  }
};
// kkt_general rows (cpu_backend.cpp:238-252) per slot, acc = (A x)_i on the original matrix.
struct EpiBKktRows {
  static constexpr int kMax = 2;  // pmax, dmax
  const double *YO, *RL, *RU;
  double *t_rp2, *t_d, *t_rd2;
  double* res;
  __device__ void operator()(long long, int, long long q, double ax, double* mx) const {
    const double lo = RL[q], up = RU[q];
    const double viol = ax < lo ? lo - ax : (ax > up ? ax - up : 0.0);
    t_rp2[q] = viol * viol;
    mx[0] = std_max(mx[0], elem_viol(ax, lo, up));
    const double yi = YO[q];
    double d = 0.0, rd = 0.0;
    if (yi > 0) {
      if (isfinite(lo)) d = yi * lo;
      else rd = yi * yi, mx[1] = std_max(mx[1], yi);
    } else if (yi < 0) {
      if (isfinite(up)) d = yi * up;
      else rd = yi * yi, mx[1] = std_max(mx[1], -yi);
    }
    t_d[q] = d;
    t_rd2[q] = rd;
  }
  __device__ unsigned long long* key(int t, int k) const {
    return reinterpret_cast<unsigned long long*>(res + static_cast<long long>(t) * kRes + kBPmax + k);
  }
};
// kkt_general columns (cpu_backend.cpp:253-271), acc = (Aᵀy)_j in the caller's CSC order.
struct EpiBKktCols {
  static constexpr int kMax = 2;
  const double *XO, *OC, *CL, *CU;
  double sense;
  double *t_p, *t_d, *t_rd2;
  double* res;
  __device__ void operator()(long long, int, long long q, double aty, double* mx) const {
    const double cj = sense * OC[q];
    const double x = XO[q], lo = CL[q], up = CU[q];
    t_p[q] = cj * x;
    mx[0] = std_max(mx[0], elem_viol(x, lo, up));
    const double lam = cj - aty;
    double z;
    if (isfinite(lo) && isfinite(up)) z = lam;
    else if (isfinite(lo)) z = std_max(lam, 0.0);
    else if (isfinite(up)) z = std_min(lam, 0.0);
    else z = 0.0;
    t_rd2[q] = (lam - z) * (lam - z);
    mx[1] = std_max(mx[1], fabs(lam - z));
    t_d[q] = z > 0 ? z * lo : (z < 0 ? z * up : 0.0);
  }
  __device__ unsigned long long* key(int t, int k) const {
    return reinterpret_cast<unsigned long long*>(res + static_cast<long long>(t) * kRes + kBPmax + k);
  }
};

// ------------------------------------------------------------------------- per-slot sums
// A sum of one slot's terms over rows a[0, na) then b[0, nb) of interleaved blocks, into
// res[t·kRes + out]. Up to kMaxSeg sums per launch (passed by value).
constexpr int kMaxSeg = 12;
struct ISeg {
  const double* a;
  long long na;
  const double* b;
  long long nb;
  double init;
  int out;
};
struct ISegs {
  ISeg s[kMaxSeg];
  int n;
};
__device__ __forceinline__ double iterm(const ISeg& g, long long r, int W, int t) {
  return r < g.na ? g.a[r * W + t] : g.b[(r - g.na) * W + t];
}
// exact: one lane per slot walks r = 0, 1, … in order (kkt_general / compute_residuals loops)
__global__ void k_isum_seq(ISegs segs, int W, double* res) {
  const ISeg g = segs.s[blockIdx.y];
  const int t = blockIdx.x * 32 + threadIdx.x;
  if (t >= W) return;
  double s = g.init;
#pragma unroll 8
  for (long long r = 0; r < g.na; ++r) s += g.a[r * W + t];
#pragma unroll 8
  for (long long r = 0; r < g.nb; ++r) s += g.b[r * W + t];
  res[static_cast<long long>(t) * kRes + g.out] = s;
}
// fast, level 1: chunk c of P, 8 warps split it, lane = slot; partials in a fixed order
__global__ void k_isum_part(ISegs segs, int W, int P, double* part) {
  __shared__ double sh[8][32];
  const ISeg g = segs.s[blockIdx.z];
  const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
  const int t = blockIdx.y * 32 + lane;
  const long long len = g.na + g.nb, c = blockIdx.x;
  const long long a = len * c / P, e = len * (c + 1) / P;
  const long long wa = a + (e - a) * wp / 8, we = a + (e - a) * (wp + 1) / 8;
  double s = 0.0;
  if (t < W)
    for (long long r = wa; r < we; ++r) s += iterm(g, r, W, t);
  sh[wp][lane] = s;
  __syncthreads();
  if (wp == 0 && t < W) {
    double v = 0.0;
    for (int k = 0; k < 8; ++k) v += sh[k][lane];
    part[(static_cast<long long>(blockIdx.z) * P + c) * W + t] = v;
  }
}
__global__ void k_isum_fin(ISegs segs, int W, int P, const double* part, double* res) {
  const ISeg g = segs.s[blockIdx.y];
  const int t = blockIdx.x * 32 + threadIdx.x;
  if (t >= W) return;
  double s = g.init;
  for (int c = 0; c < P; ++c) s += part[(static_cast<long long>(blockIdx.y) * P + c) * W + t];
  res[static_cast<long long>(t) * kRes + g.out] = s;
}

// ---------------------------------------------------------------------- element-wise
// Per-scenario kkt_general constants and the bound/objective rescaling sums (batch.cpp:208-223).
__global__ void k_bconst_rows(long long mw, int W, const double* RLo, const double* RUo, const double* row_scale,
                              double* t_b2, double* t_sb2) {
  B200_FOR(q, mw) {
    const long long i = q / W;
    const double lo = RLo[q], up = RUo[q];
    const double bl = isfinite(lo) ? fabs(lo) : 0.0, bu = isfinite(up) ? fabs(up) : 0.0;
    t_b2[q] = std_max(bl, bu) * std_max(bl, bu);
    const double b = row_scale[i] * std_max(bl, bu);
    t_sb2[q] = b * b;
  }
}
__global__ void k_bconst_cols(long long nw, int W, double sense, const double* OC, const double* col_scale,
                              double* t_c2, double* t_sc2, double* res) {
  B200_FOR(q, nw) {
    const long long j = q / W;
    const double cj = sense * OC[q];
    t_c2[q] = cj * cj;
    const double c = col_scale[j] * OC[q];
    t_sc2[q] = c * c;
    const int t = static_cast<int>(q % W);
    atomic_max_nonneg(reinterpret_cast<unsigned long long*>(res + static_cast<long long>(t) * kRes + kBCinf), fabs(cj));
  }
}
// Scaled scenario vectors and the start point (batch.cpp:224-249).
__global__ void k_bscale_cols(long long nw, int W, double sense, const double* OC, const double* CLo, const double* CUo,
                              const double* col_scale, const double* bs, const double* os, double* C, double* L,
                              double* U, double* X, double* X0, double* XH, double* XB) {
  B200_FOR(q, nw) {
    const long long j = q / W;
    const int t = static_cast<int>(q % W);
    C[q] = os[t] * col_scale[j] * sense * OC[q];
    const double l = bs[t] * CLo[q] / col_scale[j], u = bs[t] * CUo[q] / col_scale[j];
    L[q] = l;
    U[q] = u;
    const double x = ref_clamp(0.0, l, u);
    X[q] = x, X0[q] = x, XH[q] = x, XB[q] = 0.0;
  }
}
__global__ void k_bscale_rows(long long mw, int W, const double* RLo, const double* RUo, const double* row_scale,
                              const double* bs, double* RL, double* RU, double* Y, double* Y0, double* YH,
                              double* YB) {
  B200_FOR(q, mw) {
    const long long i = q / W;
    const int t = static_cast<int>(q % W);
    RL[q] = bs[t] * row_scale[i] * RLo[q];
    RU[q] = bs[t] * row_scale[i] * RUo[q];
    Y[q] = 0.0, Y0[q] = 0.0, YH[q] = 0.0, YB[q] = 0.0;
  }
}
// Δx = x̄ − x̂ and its terms; at a check also (x̂ − x0)² (batch.cpp:306, 395-398).
template <class T>
__global__ void k_bres_x(long long nw, const T* XB, const T* XH, const T* X0, T* DX, double* t_px, double* t_dxn) {
  B200_FOR(q, nw) {
    const T d = XB[q] - XH[q];
    DX[q] = d;
    t_px[q] = static_cast<double>(d) * static_cast<double>(d);
    if (t_dxn) {
      const double e = static_cast<double>(XH[q]) - static_cast<double>(X0[q]);
      t_dxn[q] = e * e;
    }
  }
}
// unscale (batch.cpp:267-275): x = clamp(C x̂ / bs, l, u), y_min = R ŷ / os
template <class T>
__global__ void k_bunscale_x(long long nw, int W, const T* XH, const double* col_scale, const double* bs,
                             const double* CLo, const double* CUo, double* XO) {
  B200_FOR(q, nw) {
    const long long j = q / W;
    const int t = static_cast<int>(q % W);
    XO[q] = ref_clamp(col_scale[j] * static_cast<double>(XH[q]) / bs[t], CLo[q], CUo[q]);
  }
}
template <class T>
__global__ void k_bunscale_y(long long mw, int W, const T* YH, const double* row_scale, const double* os,
                             double* YO) {
  B200_FOR(q, mw) {
    const long long i = q / W;
    const int t = static_cast<int>(q % W);
    YO[q] = row_scale[i] * static_cast<double>(YH[q]) / os[t];
  }
}
// restart of the flagged slots: x = x0 = x̂, y = y0 = ŷ (batch.cpp:413-420)
template <class T>
__global__ void k_brestart(long long nw, long long mw, int W, const int* flag, const T* XH, T* X, T* X0, const T* YH,
                           T* Y, T* Y0) {
  B200_FOR(q, (nw > mw ? nw : mw)) {
    const int t = static_cast<int>(q % W);
    if (!flag[t]) continue;
    if (q < nw) X[q] = XH[q], X0[q] = XH[q];
    if (q < mw) Y[q] = YH[q], Y0[q] = YH[q];
  }
}
template <class T>
__global__ void k_bgather(long long rows, int W, int W2, const int* keep, const T* src, T* dst) {
  B200_FOR(q, rows * W2) {
    const long long r = q / W2;
    const int t2 = static_cast<int>(q % W2);
    dst[q] = src[r * W + keep[t2]];
  }
}
// element-wise precision change of a whole block (the mixed form's start and promotion)
template <class D, class S>
__global__ void k_bconvert(long long len, const S* src, D* dst) {
  B200_FOR(q, len) dst[q] = static_cast<D>(src[q]);
}
__global__ void k_bcolumn(long long rows, int W, int t, const double* src, double* dst) {
  B200_FOR(r, rows) dst[r] = src[r * W + t];
}
__global__ void k_bzero_keys(int W, double* res) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < W) res[static_cast<long long>(t) * kRes + kBPmax] = 0.0, res[static_cast<long long>(t) * kRes + kBDmax] = 0.0;
}

struct BKkt {  // pdhg::KktStats (termination.h:35-60) with obj_shift = 0
  double primal_residual = 0, dual_residual = 0, primal_obj = 0, dual_obj = 0, b_norm = 0, c_norm = 0;
  double primal_max_rel = 0, dual_max_rel = 0;
  double rel_primal() const { return primal_residual / (1.0 + b_norm); }
  double rel_dual() const { return dual_residual / (1.0 + c_norm); }
  double rel_gap() const { return std::fabs(primal_obj - dual_obj) / (1.0 + std::fabs(primal_obj) + std::fabs(dual_obj)); }
  double rel_kkt() const { return std::max({rel_primal(), rel_dual(), rel_gap()}); }
  bool converged(double eps) const {
    if (rel_kkt() > eps) return false;
    if (eps >= kVerifyPrimal) return true;
    return primal_max_rel <= kVerifyPrimal && dual_max_rel <= kVerifyDual && rel_gap() <= kVerifyGap;
  }
  bool finite() const {
    return std::isfinite(primal_residual) && std::isfinite(dual_residual) && std::isfinite(primal_obj) &&
           std::isfinite(dual_obj);
  }
};

// ------------------------------------------------------------------------- the engine
class BatchEngine {
 public:
  BatchEngine(const HostModelView& base, const std::vector<BatchScenarioView>& sc, const std::vector<int>& sid,
              const EngineOptions& o, cudaStream_t st, std::chrono::steady_clock::time_point t0)
      : B_(base), S_(sc), sid_(sid), o_(o), st_(st), t0_(t0) {
    for (auto& e : ev_) B200_CHECK(cudaEventCreate(&e));
  }
  ~BatchEngine() {
    drop_graphs();
    for (auto& e : ev_) cudaEventDestroy(e);
  }
  BatchEngine(const BatchEngine&) = delete;
  BatchEngine& operator=(const BatchEngine&) = delete;

  void run(std::vector<BatchOutcome>& out);
  // Bulk-copy waits of this batch's setup kernels that ran out (synchronises the stream).
  unsigned stage_errors() {
    unsigned v = 0;
    if (stage_err_.get()) {
      B200_CHECK(cudaMemcpyAsync(&v, stage_err_.get(), sizeof v, cudaMemcpyDeviceToHost, st_));
      B200_CHECK(cudaStreamSynchronize(st_));
    }
    return v;
  }

 private:
  double elapsed() const { return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0_).count(); }
  void upload_model();
  void setup();
  void launch_sums(const ISegs& segs, bool exact);
  void launch_residual(bool distances);
  void launch_kkt();
  template <class Epi, class TV, class TX>
  void spmm(int rows, const int* rp, const int* col, const TV* val, const TX* X, const Epi& epi, bool capped,
            int shape = 0);
  void tune_spmm();
  void step(int s);
  void epoch_body(bool r0_section);
  void launch_epoch(bool r0_section);
  void drop_graphs() {
    for (auto& g : graph_)
      if (g) cudaGraphExecDestroy(g), g = nullptr;
  }
  void compact(const std::vector<int>& keep);
  void start_mixed();
  void promote();
  void finish_slot(int t, BatchOutcome& o, Status st, const BKkt& kk, long long it, const std::string& msg);

  const HostModelView& B_;
  const std::vector<BatchScenarioView>& S_;
  std::vector<int> sid_;
  const EngineOptions& o_;
  cudaStream_t st_;
  cudaEvent_t ev_[4] = {};  // SpMM time of an epoch: [0,1] step 0, [2,3] steps 1..K-1
  cudaGraphExec_t graph_[2] = {nullptr, nullptr};  // epoch without / with the r⁰ section
  long long graph_kernels_[2] = {0, 0};
  double spmm_ms_ = 0.0;
  long long spmm_launches_ = 0;
  std::chrono::steady_clock::time_point t0_;
  int m_ = 0, n_ = 0, W_ = 0;
  double eta_ = 1.0, setup_s_ = 0.0;
  long long launches_ = 0;
  int shape_[2] = {0, 0};  // SpMM shapes of the primal and dual step kernels (tune_spmm)

  DevBuf<double> c_, cl_, cu_, rl_, ru_, v_;
  DevBuf<int> cs_, ri_;
  DevBuf<unsigned> stage_err_;  // this batch's bulk-copy timeouts (see count_stage_timeout)
  ScaledDevice sp_;
  // interleaved blocks: original data, scaled data, iterates, work and term arrays
  enum NVec { OC, OCL, OCU, C, L, U, X, X0, XH, XB, DX, XO, TPX, TDXN, TP, TDC, TRDC, TC2, TSC2, kNVec };
  enum MVec { ORL, ORU, RL, RU, Y, Y0, YH, YB, YO, TPY, TCR, TDYN, TRP2, TDR, TRDR, TB2, TSB2, kMVec };
  DevBuf<double> nv_[kNVec], mv_[kMVec], spare_n_, spare_m_;
  // the mixed form's first phase: fp32 copies of the scaled data and of the iterate blocks
  enum FN { FC, FL, FU, FX, FX0, FXH, FXB, FDX, kFN };
  enum FM { FRL, FRU, FY, FY0, FYH, FYB, kFM };
  DevBuf<float> fn_[kFN], fm_[kFM], fspare_n_, fspare_m_;
  bool mixed_now_ = false;
  long long switch_it_ = -1;
  DevBuf<double> res_, part_, tau_, sigma_, bs_, os_, col_buf_n_, col_buf_m_, col_buf_c_, obj_t_, obj_out_;
  DevBuf<long long> inner0_;
  DevBuf<int> flag_, keep_;
  PinnedBuf<double> h_res_, h_par_;
  PinnedBuf<long long> h_inner_;
  PinnedBuf<int> h_int_;
  std::vector<double> hbs_, hos_;
};

// `shape`: how the W slots of a row are spread over lanes. 0: G = 32 lanes per row (fewer for
// W < 32) with S = ⌈W/G⌉ slots per lane; c > 0: G/2^c lanes with 2^c times the slots (while
// S ≤ 8). Every shape sums each (row, slot) in the same order; the iteration kernels use the
// shape the autotuner measured fastest on this matrix (tune_spmm).
template <class Epi, class TV, class TX>
void BatchEngine::spmm(int rows, const int* rp, const int* col, const TV* val, const TX* X, const Epi& epi,
                       bool capped, int shape) {
  if (rows <= 0) return;
  int lg = 0, S = 1;
  if (W_ >= 32) {
    lg = 5;
    const int need = (W_ + 31) / 32;
    S = need <= 1 ? 1 : need <= 2 ? 2 : need <= 4 ? 4 : 8;
  } else {
    while ((1 << lg) < W_) ++lg;
  }
  for (int c = 0; c < shape && lg > 0 && S < 8; ++c) --lg, S *= 2;
  const long long threads = static_cast<long long>(rows) << lg;
  long long blocks = (threads + 255) / 256;
  if (capped) blocks = std::min<long long>(blocks, 148 * 8);
  blocks = std::max<long long>(1, std::min<long long>(blocks, 1LL << 30));
  const int nb = static_cast<int>(blocks);
  switch (S) {
    case 1: k_bspmm<1, Epi, TV, TX><<<nb, 256, 0, st_>>>(rows, W_, lg, rp, col, val, X, epi); break;
    case 2: k_bspmm<2, Epi, TV, TX><<<nb, 256, 0, st_>>>(rows, W_, lg, rp, col, val, X, epi); break;
    case 4: k_bspmm<4, Epi, TV, TX><<<nb, 256, 0, st_>>>(rows, W_, lg, rp, col, val, X, epi); break;
    default: k_bspmm<8, Epi, TV, TX><<<nb, 256, 0, st_>>>(rows, W_, lg, rp, col, val, X, epi); break;
  }
  B200_LAUNCH_CHECK();
  ++launches_;
}

// exact: each slot's sums in the reference's order (one lane per slot); else the fixed split.
void BatchEngine::launch_sums(const ISegs& segs, bool exact) {
  if (segs.n == 0 || W_ == 0) return;
  const int gx = (W_ + 31) / 32;
  if (exact) {
    k_isum_seq<<<dim3(gx, segs.n), 32, 0, st_>>>(segs, W_, res_.get());
    B200_LAUNCH_CHECK();
    ++launches_;
    return;
  }
  long long len = 0;
  for (int k = 0; k < segs.n; ++k) len = std::max(len, segs.s[k].na + segs.s[k].nb);
  const int P = static_cast<int>(std::max<long long>(1, std::min<long long>(64, len / 2048)));
  k_isum_part<<<dim3(P, gx, segs.n), 256, 0, st_>>>(segs, W_, P, part_.get());
  k_isum_fin<<<dim3(gx, segs.n), 32, 0, st_>>>(segs, W_, P, part_.get(), res_.get());
  B200_LAUNCH_CHECK();
  launches_ += 2;
}

void BatchEngine::upload_model() {
  const std::size_t mm = m_, nn = n_, nz = static_cast<std::size_t>(B_.col_start[n_]);
  c_.upload(B_.c, nn, st_), cl_.upload(B_.col_lower, nn, st_), cu_.upload(B_.col_upper, nn, st_);
  rl_.upload(B_.row_lower, mm, st_), ru_.upload(B_.row_upper, mm, st_);
  cs_.upload(B_.col_start, nn + 1, st_), ri_.upload(B_.row_index, nz, st_), v_.upload(B_.value, nz, st_);
}

void BatchEngine::setup() {
  m_ = B_.m, n_ = B_.n;
  W_ = static_cast<int>(sid_.size());
  upload_model();
  DeviceModel dm;
  dm.m = m_, dm.n = n_, dm.sense = B_.sense, dm.offset = B_.offset;
  dm.c = c_.get(), dm.col_lower = cl_.get(), dm.col_upper = cu_.get(), dm.row_lower = rl_.get(),
  dm.row_upper = ru_.get(), dm.col_start = cs_.get(), dm.row_index = ri_.get(), dm.value = v_.get();
  dm.nnz = B_.col_start[n_];
  // shared scaling of A only: bound/objective scalars are per scenario (batch.cpp:196-200)
  ScalingOptions so = o_.scaling;
  so.bound_objective_rescaling = false;
  sp_.build(dm, so, o_.exact, st_);
  stage_err_.alloc(1);
  B200_CHECK(cudaMemsetAsync(stage_err_.get(), 0, sizeof(unsigned), st_));
  const double norm = sp_.lanczos(st_, stage_err_.get());
  eta_ = norm > 0 ? 0.998 / norm : 1.0;
  setup_s_ = elapsed();

  const std::size_t NW = static_cast<std::size_t>(n_) * W_, MW = static_cast<std::size_t>(m_) * W_;
  for (auto& v : nv_) v.alloc(NW);
  for (auto& v : mv_) v.alloc(MW);
  spare_n_.alloc(NW), spare_m_.alloc(MW);
  res_.alloc(static_cast<std::size_t>(W_) * kRes);
  part_.alloc(static_cast<std::size_t>(kMaxSeg) * 64 * W_);
  tau_.alloc(W_), sigma_.alloc(W_), bs_.alloc(W_), os_.alloc(W_), inner0_.alloc(W_), flag_.alloc(W_), keep_.alloc(W_);
  const std::size_t n1 = static_cast<std::size_t>(std::max(n_, 1));
  col_buf_n_.alloc(n1), col_buf_m_.alloc(static_cast<std::size_t>(std::max(m_, 1))), col_buf_c_.alloc(n1);
  obj_t_.alloc(n1), obj_out_.alloc(1);
  h_res_.alloc(static_cast<std::size_t>(W_) * kRes);
  h_par_.alloc(static_cast<std::size_t>(W_) * 4);
  h_inner_.alloc(W_);
  h_int_.alloc(W_);
  B200_CHECK(cudaMemsetAsync(res_.get(), 0, static_cast<std::size_t>(W_) * kRes * sizeof(double), st_));

  // ---- original scenario data, interleaved (host assembly, one upload per block)
  {
    std::vector<double> hn(NW), hm(MW);
    auto put_n = [&](NVec which, auto pick) {
      for (int t = 0; t < W_; ++t) {
        const double* src = pick(S_[sid_[t]]);
        for (int j = 0; j < n_; ++j) hn[static_cast<std::size_t>(j) * W_ + t] = src[j];
      }
      nv_[which].upload(hn.data(), NW, st_);
      B200_CHECK(cudaStreamSynchronize(st_));
    };
    auto put_m = [&](MVec which, auto pick) {
      for (int t = 0; t < W_; ++t) {
        const double* src = pick(S_[sid_[t]]);
        for (int i = 0; i < m_; ++i) hm[static_cast<std::size_t>(i) * W_ + t] = src[i];
      }
      mv_[which].upload(hm.data(), MW, st_);
      B200_CHECK(cudaStreamSynchronize(st_));
    };
    put_n(OC, [&](const BatchScenarioView& s) { return s.c ? s.c : B_.c; });
    put_n(OCL, [&](const BatchScenarioView& s) { return s.col_lower ? s.col_lower : B_.col_lower; });
    put_n(OCU, [&](const BatchScenarioView& s) { return s.col_upper ? s.col_upper : B_.col_upper; });
    put_m(ORL, [&](const BatchScenarioView& s) { return s.row_lower ? s.row_lower : B_.row_lower; });
    put_m(ORU, [&](const BatchScenarioView& s) { return s.row_upper ? s.row_upper : B_.row_upper; });
  }
  const long long nw = static_cast<long long>(NW), mw = static_cast<long long>(MW);
  // ---- per-scenario constants: kkt_general ‖b‖², ‖c‖², ‖c‖∞ and the rescaling sums
  k_bconst_rows<<<grid_for(mw), kBlock, 0, st_>>>(mw, W_, mv_[ORL].get(), mv_[ORU].get(), sp_.row_scale.get(),
                                                  mv_[TB2].get(), mv_[TSB2].get());
  k_bconst_cols<<<grid_for(nw), kBlock, 0, st_>>>(nw, W_, static_cast<double>(B_.sense), nv_[OC].get(),
                                                  sp_.col_scale.get(), nv_[TC2].get(), nv_[TSC2].get(), res_.get());
  B200_LAUNCH_CHECK();
  launches_ += 2;
  ISegs segs{};
  segs.s[0] = {mv_[TB2].get(), m_, nullptr, 0, 0.0, kBB2};
  segs.s[1] = {nv_[TC2].get(), n_, nullptr, 0, 0.0, kBC2};
  segs.s[2] = {mv_[TSB2].get(), m_, nullptr, 0, 0.0, kBSb2};
  segs.s[3] = {nv_[TSC2].get(), n_, nullptr, 0, 0.0, kBSc2};
  segs.n = 4;
  launch_sums(segs, true);  // the rescaling sums enter the scaled data: always the reference's order
  B200_CHECK(cudaMemcpyAsync(h_res_.get(), res_.get(), static_cast<std::size_t>(W_) * kRes * sizeof(double),
                             cudaMemcpyDeviceToHost, st_));
  B200_CHECK(cudaStreamSynchronize(st_));
  hbs_.assign(W_, 1.0), hos_.assign(W_, 1.0);
  if (o_.scaling.bound_objective_rescaling) {
    for (int t = 0; t < W_; ++t) {
      hbs_[t] = 1.0 / (std::sqrt(h_res_[static_cast<std::size_t>(t) * kRes + kBSb2]) + 1.0);
      hos_[t] = 1.0 / (std::sqrt(h_res_[static_cast<std::size_t>(t) * kRes + kBSc2]) + 1.0);
    }
  }
  bs_.upload(hbs_.data(), W_, st_), os_.upload(hos_.data(), W_, st_);
  tune_spmm();  // before the start point is written: the timed launches overwrite the iterates
  k_bscale_cols<<<grid_for(nw), kBlock, 0, st_>>>(nw, W_, static_cast<double>(B_.sense), nv_[OC].get(),
                                                  nv_[OCL].get(), nv_[OCU].get(), sp_.col_scale.get(), bs_.get(),
                                                  os_.get(), nv_[C].get(), nv_[L].get(), nv_[U].get(), nv_[X].get(),
                                                  nv_[X0].get(), nv_[XH].get(), nv_[XB].get());
  k_bscale_rows<<<grid_for(mw), kBlock, 0, st_>>>(mw, W_, mv_[ORL].get(), mv_[ORU].get(), sp_.row_scale.get(),
                                                  bs_.get(), mv_[RL].get(), mv_[RU].get(), mv_[Y].get(),
                                                  mv_[Y0].get(), mv_[YH].get(), mv_[YB].get());
  B200_LAUNCH_CHECK();
  launches_ += 2;
  if (o_.mixed) start_mixed();
  B200_CHECK(cudaStreamSynchronize(st_));
}

// The mixed form starts in fp32: the scaled matrix and every scaled-data and iterate block are
// converted once (the fp64 blocks stay, for the checks and for the promotion).
void BatchEngine::start_mixed() {
  sp_.make_f32(st_);
  const long long nw = static_cast<long long>(n_) * W_, mw = static_cast<long long>(m_) * W_;
  const NVec ns[kFN] = {C, L, U, X, X0, XH, XB, DX};
  const MVec ms[kFM] = {RL, RU, Y, Y0, YH, YB};
  for (int k = 0; k < kFN; ++k) {
    fn_[k].alloc(static_cast<std::size_t>(nw));
    k_bconvert<float, double><<<grid_for(nw), kBlock, 0, st_>>>(nw, nv_[ns[k]].get(), fn_[k].get());
  }
  for (int k = 0; k < kFM; ++k) {
    fm_[k].alloc(static_cast<std::size_t>(mw));
    k_bconvert<float, double><<<grid_for(mw), kBlock, 0, st_>>>(mw, mv_[ms[k]].get(), fm_[k].get());
  }
  B200_LAUNCH_CHECK();
  launches_ += kFN + kFM;
  fspare_n_.alloc(static_cast<std::size_t>(nw)), fspare_m_.alloc(static_cast<std::size_t>(mw));
  mixed_now_ = true;
}

// Promotion to fp64 (PrecisionPolicy's switch, engine.cpp:61-79, taken by the whole batch at
// once): every iterate block converted float → double; the caller restarts every slot.
void BatchEngine::promote() {
  const long long nw = static_cast<long long>(n_) * W_, mw = static_cast<long long>(m_) * W_;
  const std::pair<int, int> np[] = {{FX, X}, {FX0, X0}, {FXH, XH}, {FXB, XB}};
  const std::pair<int, int> mp[] = {{FY, Y}, {FY0, Y0}, {FYH, YH}, {FYB, YB}};
  for (const auto& pr : np)
    k_bconvert<double, float><<<grid_for(nw), kBlock, 0, st_>>>(nw, fn_[pr.first].get(), nv_[pr.second].get());
  for (const auto& pr : mp)
    k_bconvert<double, float><<<grid_for(mw), kBlock, 0, st_>>>(mw, fm_[pr.first].get(), mv_[pr.second].get());
  B200_LAUNCH_CHECK();
  launches_ += 8;
  mixed_now_ = false;
  drop_graphs();  // the epoch graphs run the fp32 kernels
}

// The autotuner for the two step kernels (tune.hpp): every SpMM shape timed on this matrix and
// slot count, unless the shape class was measured before in this process. The choice stays
// for the whole batch (later compactions keep the shape index).
void BatchEngine::tune_spmm() {
  const int forced = tune_forced();
  if (forced >= 0) {
    shape_[0] = shape_[1] = forced < 3 ? forced : 0;
    return;
  }
  if (!tune_enabled()) return;
  const long long nnz = B_.col_start[n_];
  // the batch step kernels are classes 10 and 11, with the slot count in the precision field
  const TuneKey k0 = tune_key(10 + 0, W_, n_, nnz), k1 = tune_key(10 + 1, W_, m_, nnz);
  TuneCache& cache = TuneCache::instance();
  if (cache.get(k0, shape_[0]) && cache.get(k1, shape_[1])) return;
  cudaEvent_t a, b;
  B200_CHECK(cudaEventCreate(&a));
  B200_CHECK(cudaEventCreate(&b));
  auto measure = [&](auto&& launch) {
    double ms[3];
    for (int c = 0; c < 3; ++c) {
      launch(c);
      B200_CHECK(cudaEventRecord(a, st_));
      for (int r = 0; r < 3; ++r) launch(c);
      B200_CHECK(cudaEventRecord(b, st_));
      B200_CHECK(cudaEventSynchronize(b));
      float t = 0;
      B200_CHECK(cudaEventElapsedTime(&t, a, b));
      ms[c] = t / 3.0;
    }
    return pick_variant(ms, 3);
  };
  const int Kc = o_.check_every;
  shape_[0] = measure([&](int c) {
    EpiBPrimal<double> ep{nv_[C].get(), nv_[L].get(), nv_[U].get(), nv_[X0].get(), tau_.get(), nv_[X].get(), nv_[XH].get(),
                  nv_[XB].get(), inner0_.get(), 1, Kc - 1, 2 * o_.reflection, 1 - 2 * o_.reflection};
    spmm(n_, cs_.get(), sp_.t_ri.get(), sp_.sat.get(), mv_[Y].get(), ep, false, c);
  });
  shape_[1] = measure([&](int c) {
    EpiBDual<double> ed{mv_[RL].get(), mv_[RU].get(), mv_[Y0].get(), sigma_.get(), mv_[Y].get(), mv_[YH].get(), mv_[YB].get(),
                inner0_.get(), 1, Kc - 1, 2 * o_.reflection, 1 - 2 * o_.reflection};
    spmm(m_, sp_.a_rp.get(), sp_.a_col.get(), sp_.sa.get(), nv_[XB].get(), ed, false, c);
  });
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cache.put(k0, shape_[0]);
  cache.put(k1, shape_[1]);
}

void BatchEngine::step(int s) {
  const int last = o_.check_every - 1;
  const double a2 = 2 * o_.reflection, b2 = 1 - 2 * o_.reflection;
  if (mixed_now_) {
    EpiBPrimal<float> ep{fn_[FC].get(), fn_[FL].get(), fn_[FU].get(), fn_[FX0].get(), tau_.get(), fn_[FX].get(),
                         fn_[FXH].get(), fn_[FXB].get(), inner0_.get(), s, last, a2, b2};
    spmm(n_, cs_.get(), sp_.t_ri.get(), sp_.satf.get(), fm_[FY].get(), ep, false, shape_[0]);
    EpiBDual<float> ed{fm_[FRL].get(), fm_[FRU].get(), fm_[FY0].get(), sigma_.get(), fm_[FY].get(), fm_[FYH].get(),
                       fm_[FYB].get(), inner0_.get(), s, last, a2, b2};
    spmm(m_, sp_.a_rp.get(), sp_.a_col.get(), sp_.saf.get(), fn_[FXB].get(), ed, false, shape_[1]);
    return;
  }
  EpiBPrimal<double> ep{nv_[C].get(), nv_[L].get(), nv_[U].get(), nv_[X0].get(), tau_.get(), nv_[X].get(), nv_[XH].get(),
                        nv_[XB].get(), inner0_.get(), s, last, a2, b2};
  spmm(n_, cs_.get(), sp_.t_ri.get(), sp_.sat.get(), mv_[Y].get(), ep, false, shape_[0]);
  EpiBDual<double> ed{mv_[RL].get(), mv_[RU].get(), mv_[Y0].get(), sigma_.get(), mv_[Y].get(), mv_[YH].get(),
                      mv_[YB].get(), inner0_.get(), s, last, a2, b2};
  spmm(m_, sp_.a_rp.get(), sp_.a_col.get(), sp_.sa.get(), nv_[XB].get(), ed, false, shape_[1]);
}

// The K iterations of an epoch (the body of the epoch graph), with the r⁰ residual right after
// the first step when a slot starts a Halpern cycle (batch.cpp:359-366).
void BatchEngine::epoch_body(bool r0_section) {
  const int Kc = o_.check_every;
  B200_CHECK(cudaEventRecordWithFlags(ev_[0], st_, cudaEventRecordExternal));
  for (int s = 0; s < Kc; ++s) {
    step(s);
    if (s == 0) B200_CHECK(cudaEventRecordWithFlags(ev_[1], st_, cudaEventRecordExternal));
    if (s == 0 && r0_section) {
      launch_residual(false);
      ISegs g{};
      g.s[0] = {nv_[TPX].get(), n_, nullptr, 0, 0.0, kBPx0};
      g.s[1] = {mv_[TPY].get(), m_, nullptr, 0, 0.0, kBPy0};
      g.s[2] = {mv_[TCR].get(), m_, nullptr, 0, 0.0, kBCr0};
      g.n = 3;
      launch_sums(g, o_.exact);
    }
    if (s == 0) B200_CHECK(cudaEventRecordWithFlags(ev_[2], st_, cudaEventRecordExternal));
  }
  B200_CHECK(cudaEventRecordWithFlags(ev_[3], st_, cudaEventRecordExternal));
}

// Replays the epoch graph of this variant, capturing it first for the current slots.
void BatchEngine::launch_epoch(bool r0_section) {
  const int v = r0_section ? 1 : 0;
  if (!graph_[v]) {
    const long long before = launches_;
    cudaGraph_t g;
    {
      CaptureScope scope;  // no device-wide synchronisation elsewhere meanwhile
      B200_CHECK(cudaStreamBeginCapture(st_, cudaStreamCaptureModeThreadLocal));
      try {
        epoch_body(r0_section);
      } catch (...) {
        cudaGraph_t dead = nullptr;
        cudaStreamEndCapture(st_, &dead);
        if (dead) cudaGraphDestroy(dead);
        throw;
      }
      B200_CHECK(cudaStreamEndCapture(st_, &g));
    }
    const cudaError_t e = cudaGraphInstantiate(&graph_[v], g, 0);
    cudaGraphDestroy(g);
    B200_CHECK(e);
    graph_kernels_[v] = launches_ - before;
    launches_ = before;
  }
  B200_CHECK(cudaGraphLaunch(graph_[v], st_));
  launches_ += graph_kernels_[v];
}

void BatchEngine::launch_residual(bool distances) {
  const long long nw = static_cast<long long>(n_) * W_;
  double* tdxn = distances ? nv_[TDXN].get() : nullptr;
  double* tdyn = distances ? mv_[TDYN].get() : nullptr;
  if (mixed_now_) {
    k_bres_x<float><<<grid_for(nw), kBlock, 0, st_>>>(nw, fn_[FXB].get(), fn_[FXH].get(), fn_[FX0].get(),
                                                      fn_[FDX].get(), nv_[TPX].get(), tdxn);
    B200_LAUNCH_CHECK();
    ++launches_;
    EpiBRes<float> er{fm_[FYB].get(), fm_[FYH].get(), fm_[FY0].get(), mv_[TPY].get(), mv_[TCR].get(), tdyn};
    spmm(m_, sp_.a_rp.get(), sp_.a_col.get(), sp_.saf.get(), fn_[FDX].get(), er, false);
    return;
  }
  k_bres_x<double><<<grid_for(nw), kBlock, 0, st_>>>(nw, nv_[XB].get(), nv_[XH].get(), nv_[X0].get(), nv_[DX].get(),
                                                     nv_[TPX].get(), tdxn);
  B200_LAUNCH_CHECK();
  ++launches_;
  EpiBRes<double> er{mv_[YB].get(), mv_[YH].get(), mv_[Y0].get(), mv_[TPY].get(), mv_[TCR].get(), tdyn};
  spmm(m_, sp_.a_rp.get(), sp_.a_col.get(), sp_.sa.get(), nv_[DX].get(), er, false);
}

void BatchEngine::launch_kkt() {
  const long long nw = static_cast<long long>(n_) * W_, mw = static_cast<long long>(m_) * W_;
  if (mixed_now_) {
    k_bunscale_x<float><<<grid_for(nw), kBlock, 0, st_>>>(nw, W_, fn_[FXH].get(), sp_.col_scale.get(), bs_.get(),
                                                          nv_[OCL].get(), nv_[OCU].get(), nv_[XO].get());
    k_bunscale_y<float><<<grid_for(mw), kBlock, 0, st_>>>(mw, W_, fm_[FYH].get(), sp_.row_scale.get(), os_.get(),
                                                          mv_[YO].get());
  } else {
    k_bunscale_x<double><<<grid_for(nw), kBlock, 0, st_>>>(nw, W_, nv_[XH].get(), sp_.col_scale.get(), bs_.get(),
                                                           nv_[OCL].get(), nv_[OCU].get(), nv_[XO].get());
    k_bunscale_y<double><<<grid_for(mw), kBlock, 0, st_>>>(mw, W_, mv_[YH].get(), sp_.row_scale.get(), os_.get(),
                                                           mv_[YO].get());
  }
  k_bzero_keys<<<(W_ + 127) / 128, 128, 0, st_>>>(W_, res_.get());
  B200_LAUNCH_CHECK();
  launches_ += 3;
  EpiBKktRows er{mv_[YO].get(), mv_[ORL].get(), mv_[ORU].get(), mv_[TRP2].get(), mv_[TDR].get(), mv_[TRDR].get(),
                 res_.get()};
  spmm(m_, sp_.a_rp.get(), sp_.a_col.get(), sp_.a_v0.get(), nv_[XO].get(), er, true);
  EpiBKktCols ec{nv_[XO].get(), nv_[OC].get(), nv_[OCL].get(), nv_[OCU].get(), static_cast<double>(B_.sense),
                 nv_[TP].get(), nv_[TDC].get(), nv_[TRDC].get(), res_.get()};
  spmm(n_, cs_.get(), ri_.get(), v_.get(), mv_[YO].get(), ec, true);
}

void BatchEngine::compact(const std::vector<int>& keep) {
  const int W2 = static_cast<int>(keep.size());
  for (int t = 0; t < W2; ++t) h_int_[t] = keep[t];
  B200_CHECK(cudaMemcpyAsync(keep_.get(), h_int_.get(), W2 * sizeof(int), cudaMemcpyHostToDevice, st_));
  auto gather = [&](auto& v, long long rows, auto& spare) {
    k_bgather<<<grid_for(rows * W2), kBlock, 0, st_>>>(rows, W_, W2, keep_.get(), v.get(), spare.get());
    B200_LAUNCH_CHECK();
    ++launches_;
    std::swap(v, spare);
  };
  for (auto& v : nv_) gather(v, n_, spare_n_);
  for (auto& v : mv_) gather(v, m_, spare_m_);
  if (mixed_now_) {
    for (auto& v : fn_) gather(v, n_, fspare_n_);
    for (auto& v : fm_) gather(v, m_, fspare_m_);
  }
  drop_graphs();  // the blocks moved and the slot count changed: capture again
  std::vector<double> nbs(W2), nos(W2);
  for (int t = 0; t < W2; ++t) nbs[t] = hbs_[keep[t]], nos[t] = hos_[keep[t]];
  hbs_.swap(nbs), hos_.swap(nos);
  bs_.upload(hbs_.data(), W2, st_), os_.upload(hos_.data(), W2, st_);
  B200_CHECK(cudaStreamSynchronize(st_));  // the host vectors above are pageable
  std::vector<int> nsid(W2);
  for (int t = 0; t < W2; ++t) nsid[t] = sid_[keep[t]];
  sid_.swap(nsid);
  W_ = W2;
}

void BatchEngine::finish_slot(int t, BatchOutcome& so, Status st, const BKkt& kk, long long it,
                              const std::string& msg) {
  // batch.cpp:276-298: x, y = sense·y_min, z = c − Aᵀy (CSC order), objective = offset + Σ c x
  const int m = m_, n = n_;
  so.status = st;
  so.message = msg;
  k_bcolumn<<<grid_for(n), kBlock, 0, st_>>>(n, W_, t, nv_[XO].get(), col_buf_n_.get());
  k_bcolumn<<<grid_for(m), kBlock, 0, st_>>>(m, W_, t, mv_[YO].get(), col_buf_m_.get());
  k_bcolumn<<<grid_for(n), kBlock, 0, st_>>>(n, W_, t, nv_[OC].get(), col_buf_c_.get());
  k_dual_out<<<grid_for(m), kBlock, 0, st_>>>(m, static_cast<double>(B_.sense), col_buf_m_.get(), col_buf_m_.get());
  k_obj_terms<<<grid_for(n), kBlock, 0, st_>>>(n, col_buf_c_.get(), col_buf_n_.get(), obj_t_.get());
  B200_LAUNCH_CHECK();
  launches_ += 5;
  SumPlan p;
  p.add(obj_t_.get(), 0, n, B_.offset, SumOrder::kSeq, obj_out_.get());
  p.build(o_.exact, nullptr, st_);
  p.launch(st_);
  launches_ += p.kernel_count();
  so.x.resize(n), so.y.resize(m), so.z.resize(n);
  if (n) B200_CHECK(cudaMemcpyAsync(so.x.data(), col_buf_n_.get(), n * sizeof(double), cudaMemcpyDeviceToHost, st_));
  if (m) B200_CHECK(cudaMemcpyAsync(so.y.data(), col_buf_m_.get(), m * sizeof(double), cudaMemcpyDeviceToHost, st_));
  // z after the objective sum has read obj_t_: obj_t_ is reused as z's output
  k_reduced_costs<<<grid_for(n), kBlock, 0, st_>>>(n, cs_.get(), ri_.get(), v_.get(), col_buf_c_.get(),
                                                   col_buf_m_.get(), obj_t_.get());
  B200_LAUNCH_CHECK();
  ++launches_;
  if (n) B200_CHECK(cudaMemcpyAsync(so.z.data(), obj_t_.get(), n * sizeof(double), cudaMemcpyDeviceToHost, st_));
  double obj = 0;
  B200_CHECK(cudaMemcpyAsync(&obj, obj_out_.get(), sizeof obj, cudaMemcpyDeviceToHost, st_));
  B200_CHECK(cudaStreamSynchronize(st_));
  so.objective = obj;
  so.dual_objective = B_.sense * kk.dual_obj + B_.offset;
  so.primal_residual = kk.rel_primal();
  so.dual_residual = kk.rel_dual();
  so.gap = kk.rel_gap();
  so.iterations = it;
  so.seconds = elapsed();
  so.setup_seconds = setup_s_;
}

void BatchEngine::run(std::vector<BatchOutcome>& out) {
  setup();
  const int K = static_cast<int>(out.size());
  std::vector<double> omega(K, 1.0), best_omega(K, 1.0), best_balance(K, 1e300), pid_int(K, 0.0), pid_last(K, 0.0);
  std::vector<double> r0(K, -1.0), r_last(K, std::numeric_limits<double>::infinity());
  std::vector<double> pol_best(K, 1e300);
  std::vector<int> pol_since(K, 0);
  std::vector<long long> inner(K, 0), fast_it(K, -1);
  std::vector<double> fast_s(K, -1.0);
  const int Kc = o_.check_every;
  long long it = 0;
  auto resid_of = [&](const double* r, int k, int base) {
    const double om = omega[k];
    return std::sqrt(std::max(om * r[base] + r[base + 1] / om + 2.0 * eta_ * r[base + 2], 0.0));
  };
  while (W_ > 0) {
    // per-slot step data for this epoch: τ = η/ω, σ = ηω, the Halpern counters
    bool any_new = false;
    for (int t = 0; t < W_; ++t) {
      const int k = sid_[t];
      h_par_[t] = eta_ / omega[k];
      h_par_[W_ + t] = eta_ * omega[k];
      h_inner_[t] = inner[k];
      any_new = any_new || inner[k] == 0;
    }
    B200_CHECK(cudaMemcpyAsync(tau_.get(), h_par_.get(), W_ * sizeof(double), cudaMemcpyHostToDevice, st_));
    B200_CHECK(cudaMemcpyAsync(sigma_.get(), h_par_.get() + W_, W_ * sizeof(double), cudaMemcpyHostToDevice, st_));
    B200_CHECK(cudaMemcpyAsync(inner0_.get(), h_inner_.get(), W_ * sizeof(long long), cudaMemcpyHostToDevice, st_));
    launch_epoch(any_new);
    for (int t = 0; t < W_; ++t) inner[sid_[t]] += Kc;
    it += Kc;
    // ---- check: residual + restart distances, KKT of every slot, one download
    launch_residual(true);
    launch_kkt();
    {
      ISegs g{};
      g.s[0] = {nv_[TPX].get(), n_, nullptr, 0, 0.0, kBPx};
      g.s[1] = {mv_[TPY].get(), m_, nullptr, 0, 0.0, kBPy};
      g.s[2] = {mv_[TCR].get(), m_, nullptr, 0, 0.0, kBCr};
      g.s[3] = {mv_[TRP2].get(), m_, nullptr, 0, 0.0, kBRp2};
      g.s[4] = {mv_[TDR].get(), m_, nv_[TDC].get(), n_, 0.0, kBD};
      g.s[5] = {mv_[TRDR].get(), m_, nv_[TRDC].get(), n_, 0.0, kBRd2};
      g.s[6] = {nv_[TP].get(), n_, nullptr, 0, 0.0, kBP};
      g.n = 7;
      launch_sums(g, o_.exact);
      // the restart distances enter each slot's primal weight ω: always the reference's order
      ISegs d{};
      d.s[0] = {nv_[TDXN].get(), n_, nullptr, 0, 0.0, kBDxn};
      d.s[1] = {mv_[TDYN].get(), m_, nullptr, 0, 0.0, kBDyn};
      d.n = 2;
      launch_sums(d, true);
    }
    B200_CHECK(cudaMemcpyAsync(h_res_.get(), res_.get(), static_cast<std::size_t>(W_) * kRes * sizeof(double),
                               cudaMemcpyDeviceToHost, st_));
    B200_CHECK(cudaStreamSynchronize(st_));
    {
      float a = 0, b = 0;
      B200_CHECK(cudaEventElapsedTime(&a, ev_[0], ev_[1]));
      B200_CHECK(cudaEventElapsedTime(&b, ev_[2], ev_[3]));
      spmm_ms_ += a + b;
      spmm_launches_ += 2LL * Kc;
    }
    // r⁰ of the slots that started this epoch, with the ω they ran with
    if (any_new)
      for (int t = 0; t < W_; ++t)
        if (inner[sid_[t]] == Kc) r0[sid_[t]] = resid_of(h_res_.get() + static_cast<std::size_t>(t) * kRes, sid_[t], kBPx0);
    const bool over_iter = it >= o_.iteration_limit, over_time = elapsed() > o_.time_limit;
    auto kkt_at = [&](int t) {
      const double* r = h_res_.get() + static_cast<std::size_t>(t) * kRes;
      BKkt kk;
      kk.primal_residual = std::sqrt(r[kBRp2]);
      kk.dual_residual = std::sqrt(r[kBRd2]);
      kk.primal_obj = r[kBP];
      kk.dual_obj = r[kBD];
      kk.b_norm = std::sqrt(r[kBB2]);
      kk.c_norm = std::sqrt(r[kBC2]);
      double pmax, dmax, cinf;
      std::memcpy(&pmax, r + kBPmax, sizeof pmax);
      std::memcpy(&dmax, r + kBDmax, sizeof dmax);
      std::memcpy(&cinf, r + kBCinf, sizeof cinf);
      kk.primal_max_rel = pmax;
      kk.dual_max_rel = dmax / (1.0 + cinf);
      return kk;
    };
    // Mixed form: each running slot follows PrecisionPolicy::on_check (engine.cpp:61-79) — it asks
    // for fp64 at rel KKT ≤ 1e-6 (when the target is tighter) or after 10 checks without a 10%
    // gain — and the batch, which runs in lockstep in one precision, promotes when every slot
    // that keeps running has asked.
    bool promote_now = false;
    if (mixed_now_) {
      bool all = true, any = false;
      for (int t = 0; t < W_; ++t) {
        const int k = sid_[t];
        const BKkt kk = kkt_at(t);
        if (!kk.finite() || kk.converged(o_.tolerance) || over_iter || over_time) continue;
        const double rk = kk.rel_kkt();
        if (rk < 0.9 * pol_best[k]) pol_best[k] = rk, pol_since[k] = 0;
        else ++pol_since[k];
        const bool want = (rk <= 1e-6 && o_.tolerance < 1e-6) || pol_since[k] >= 10;
        all = all && want;
        any = true;
      }
      promote_now = any && all;
    }
    std::vector<int> keep;
    bool any_restart = false;
    for (int t = 0; t < W_; ++t) h_int_[t] = 0;
    for (int t = 0; t < W_; ++t) {
      const int k = sid_[t];
      const BKkt kk = kkt_at(t);
      auto fin = [&](Status st, const std::string& msg) {
        std::string m2 = msg;
        if (switch_it_ >= 0)
          m2 += std::string(m2.empty() ? "" : "; ") + "fp32 -> fp64 at iteration " + std::to_string(switch_it_);
        finish_slot(t, out[k], st, kk, it, m2);
        out[k].iterations_to_fast = fast_it[k];
        out[k].seconds_to_fast = fast_s[k];
        out[k].primal_weight = omega[k];
      };
      if (!kk.finite()) {
        fin(Status::NumericalError, "non-finite iterate");
        continue;
      }
      if (fast_it[k] < 0 && kk.rel_kkt() <= kFirstOrderFast) fast_it[k] = it, fast_s[k] = elapsed();
      if (kk.converged(o_.tolerance)) {
        fin(Status::Optimal, "");
        continue;
      }
      if (over_iter || over_time) {
        fin(over_iter ? Status::IterationLimit : Status::TimeLimit, "");
        continue;
      }
      keep.push_back(t);
      const double* r = h_res_.get() + static_cast<std::size_t>(t) * kRes;
      const double rr = resid_of(r, k, kBPx);
      const bool ratios_ok = r0[k] > 0 && std::isfinite(r0[k]) && rr > 0;
      const bool restart = promote_now || (ratios_ok && (rr <= o_.restart_sufficient * r0[k] ||
                                          (rr <= o_.restart_necessary * r0[k] && rr > r_last[k]))) ||
                           static_cast<double>(inner[k]) >= o_.restart_artificial * static_cast<double>(it);
      r_last[k] = rr;
      if (!restart) continue;
      // PID primal weight (batch.cpp:393-411)
      const double dxn = std::sqrt(r[kBDxn]), dyn = std::sqrt(r[kBDyn]);
      const bool both_pos = kk.rel_dual() > 0 && kk.rel_primal() > 0;
      const double ratio = both_pos ? kk.rel_dual() / kk.rel_primal() : 1.0;
      if (dxn > 1e-16 && dyn > 1e-16 && dxn < 1e12 && dyn < 1e12 && ratio > 1e-8 && ratio < 1e8) {
        const double e = std::log(dyn) - std::log(dxn) - std::log(omega[k]);
        pid_int[k] = o_.pid_integral_decay * pid_int[k] + e;
        const double stp = o_.pid_kp * e + o_.pid_ki * pid_int[k] + o_.pid_kd * (e - pid_last[k]);
        omega[k] *= std::exp(std::clamp(stp, -o_.pid_max_log_step, o_.pid_max_log_step));
        pid_last[k] = e;
      } else {
        omega[k] = best_omega[k];
        pid_int[k] = pid_last[k] = 0.0;
      }
      if (both_pos && std::fabs(std::log10(ratio)) < best_balance[k]) {
        best_balance[k] = std::fabs(std::log10(ratio));
        best_omega[k] = omega[k];
      }
      h_int_[t] = 1;
      any_restart = true;
      inner[k] = 0;
      r_last[k] = std::numeric_limits<double>::infinity();
    }
    if (any_restart) {
      B200_CHECK(cudaMemcpyAsync(flag_.get(), h_int_.get(), W_ * sizeof(int), cudaMemcpyHostToDevice, st_));
      const long long nw = static_cast<long long>(n_) * W_, mw = static_cast<long long>(m_) * W_;
      if (mixed_now_)
        k_brestart<float><<<grid_for(std::max(nw, mw)), kBlock, 0, st_>>>(nw, mw, W_, flag_.get(), fn_[FXH].get(),
                                                                          fn_[FX].get(), fn_[FX0].get(), fm_[FYH].get(),
                                                                          fm_[FY].get(), fm_[FY0].get());
      else
        k_brestart<double><<<grid_for(std::max(nw, mw)), kBlock, 0, st_>>>(nw, mw, W_, flag_.get(), nv_[XH].get(),
                                                                           nv_[X].get(), nv_[X0].get(), mv_[YH].get(),
                                                                           mv_[Y].get(), mv_[Y0].get());
      B200_LAUNCH_CHECK();
      ++launches_;
      B200_CHECK(cudaStreamSynchronize(st_));  // h_int_ is reused by compact()
    }
    if (static_cast<int>(keep.size()) != W_) compact(keep);
    if (promote_now && W_ > 0) {  // every kept slot restarted above from its x̂, ŷ
      promote();
      switch_it_ = it;
    }
    if (o_.verbosity >= 2)
      std::fprintf(stderr, "batch it %lld  t %.2fs  running %d\n", it, elapsed(), W_);
  }
  for (auto& so : out) {
    so.kernel_launches = launches_;
    so.spmm_kernel_ms = spmm_ms_;
    so.spmm_launches = spmm_launches_;
  }
}

}  // namespace

std::vector<BatchOutcome> run_batch_host(const HostModelView& base, const std::vector<BatchScenarioView>& scenarios,
                                         const std::vector<int>& slots, const EngineOptions& opt,
                                         std::chrono::steady_clock::time_point t0) {
  std::vector<BatchOutcome> out(scenarios.size());
  if (slots.empty()) return out;
  cudaStream_t st = nullptr;
  B200_CHECK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  struct StreamGuard {
    cudaStream_t s;
    ~StreamGuard() { cudaStreamDestroy(s); }
  } guard{st};
  for (std::size_t a = 0; a < slots.size(); a += kMaxSlots) {
    const std::vector<int> group(slots.begin() + static_cast<long>(a),
                                 slots.begin() + static_cast<long>(std::min(slots.size(), a + kMaxSlots)));
    BatchEngine eng(base, scenarios, group, opt, st, t0);
    std::vector<BatchOutcome> part(scenarios.size());
    eng.run(part);
    if (eng.stage_errors()) throw CudaError("a shared-memory staging wait timed out on the device");
    for (int k : group) out[k] = std::move(part[k]);
  }
  return out;
}

}  // namespace b200
