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

#include <cstddef>

#include "common.cuh"

namespace b200 {

constexpr int kSlabRows = 256;
constexpr int kSlabTile = 2048;

template <class T>
struct SlabSmem {
  int rp[kSlabRows + 1];
  int col[kSlabTile];
  T val[kSlabTile];
};

// Row-sequential fp64 accumulation of `rows` CSR rows; calls epi(row, s) for each row.
// epi.active() lets graph-replayed launches exit early (device-side flag).
template <class T, class Epi>
static __global__ void __launch_bounds__(kSlabRows, 6) k_slab(int rows, const int* __restrict__ rp,
                                                     const int* __restrict__ col,
                                                     const T* __restrict__ val,
                                                     const T* __restrict__ x, Epi epi) {
  __shared__ SlabSmem<T> sm;
  if (!epi.active()) return;
  const int r0 = blockIdx.x * kSlabRows;
  const int nr = min(kSlabRows, rows - r0);
  for (int i = threadIdx.x; i <= nr; i += blockDim.x) sm.rp[i] = rp[r0 + i];
  __syncthreads();
  const int k0 = sm.rp[0], k1 = sm.rp[nr];
  const bool mine = threadIdx.x < nr;
  const int beg = mine ? sm.rp[threadIdx.x] : 0, end = mine ? sm.rp[threadIdx.x + 1] : 0;
  double s = 0.0;
  for (int t0 = k0; t0 < k1; t0 += kSlabTile) {
    const int t1 = min(t0 + kSlabTile, k1);
    if (t0 != k0) __syncthreads();  // previous tile fully consumed
    for (int k = t0 + threadIdx.x; k < t1; k += blockDim.x) {
      sm.col[k - t0] = __ldg(col + k);
      sm.val[k - t0] = __ldg(val + k);
    }
    __syncthreads();
    const int a = max(beg, t0) - t0, b = min(end, t1) - t0;
    int k = a;
    for (; k + 4 <= b; k += 4) {
      const double p0 = static_cast<double>(sm.val[k]) * static_cast<double>(x[sm.col[k]]);
      const double p1 = static_cast<double>(sm.val[k + 1]) * static_cast<double>(x[sm.col[k + 1]]);
      const double p2 = static_cast<double>(sm.val[k + 2]) * static_cast<double>(x[sm.col[k + 2]]);
      const double p3 = static_cast<double>(sm.val[k + 3]) * static_cast<double>(x[sm.col[k + 3]]);
      s += p0;
      s += p1;
      s += p2;
      s += p3;
    }
    for (; k < b; ++k) s += static_cast<double>(sm.val[k]) * static_cast<double>(x[sm.col[k]]);
  }
  if (mine) epi(r0 + threadIdx.x, s);
}

template <class T, class Epi>
inline void launch_slab(int rows, const int* rp, const int* col, const T* val, const T* x, const Epi& epi,
                        cudaStream_t st) {
  if (rows <= 0) return;
  const int grid = (rows + kSlabRows - 1) / kSlabRows;
  k_slab<T, Epi><<<grid, kSlabRows, 0, st>>>(rows, rp, col, val, x, epi);
  B200_LAUNCH_CHECK();
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
  __device__ bool active() const { return P == nullptr || !P->done; }
  __device__ void operator()(int j, double s) const {
    double tau_d = tau, w_d = w, rho_d = rho;
    if (P) tau_d = P->tau, w_d = halpern_weight(P, step), rho_d = P->rho;
    const T aty = static_cast<T>(s);
    const T t = static_cast<T>(tau_d), tw = static_cast<T>(w_d);
    const T a = static_cast<T>(2 * rho_d), b = static_cast<T>(1 - 2 * rho_d);
    const T xj = x[j];
    const T h = ref_clamp<T>(xj - t * (c[j] - aty), l[j], u[j]);
    xh[j] = h;
    xb[j] = static_cast<T>(2) * h - xj;
    x[j] = tw * (a * h + b * xj) + (static_cast<T>(1) - tw) * x0[j];
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
  __device__ bool active() const { return P == nullptr || !P->done; }
  __device__ void operator()(int i, double s) const {
    double sig_d = sigma, w_d = w, rho_d = rho;
    bool wb = write_yb != 0;
    if (P) {
      sig_d = P->sigma, w_d = halpern_weight(P, step), rho_d = P->rho;
      wb = (step == P->K - 1) || (P->inner0 + step == 0);
    }
    const T ax = static_cast<T>(s);
    const T sg = static_cast<T>(sig_d), tw = static_cast<T>(w_d);
    const T a = static_cast<T>(2 * rho_d), b = static_cast<T>(1 - 2 * rho_d);
    const T yi = y[i];
    const T v = ax - yi / sg;
    const T h = yi - sg * ax + sg * ref_clamp<T>(v, rl[i], ru[i]);
    yh[i] = h;
    if (wb) yb[i] = static_cast<T>(2) * h - yi;
    y[i] = tw * (a * h + b * yi) + (static_cast<T>(1) - tw) * y0[i];
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
