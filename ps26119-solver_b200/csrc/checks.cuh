// checks.cuh — the every-K-iterations work of r²HPDHG on the device: fixed-point residual,
// KKT statistics on the ORIGINAL problem, infeasibility ray tests, and the final unscaling.
//
// Each kernel writes per-element TERMS of the reference's sums into term arrays (reduced by a
// SumPlan in the reference's order or a fixed tree) and folds maxima into atomic slots.
// References:
//   residual  r2hpdhg.cpp:50-59 (Δ = x̄ − x̂ etc., dots via la::parallel_sum)
//   KKT       cpu_backend.cpp:226-284 (kkt_general) with unscaling scaling.cpp:144-155
//   ray test  engine.cpp:82-155
//   finish    engine.cpp:268-307 (z = c − Aᵀy, objective)
//   check     core/solution_checker.cpp:61-133 (in-process verification)
#pragma once

#include "spmv.cuh"

namespace b200 {

// Result slots (doubles; maxima stored as the bit pattern of a non-negative double).
enum Slot : int {
  kPx0 = 0, kPy0, kCross0,                  // fixed-point residual at the epoch's first step
  kPx, kPy, kCross, kDxn2, kDyn2,           // residual at the check + restart distances
  kRp2, kD, kRd2, kP,                       // KKT sums
  kRayObj, kRayMag, kRayCd, kRayCmag,       // ray test on T(z) − z
  kRayObj2, kRayMag2, kRayCd2, kRayCmag2,   // ray test on the drift z − z0
  kObjective, kChkDual, kChkPrimal,         // finish: objective; check sums
  kNumSums,
  kMaxPmax = 32, kMaxDmax, kMaxRmax, kMaxDviol, kMaxDabs, kMaxPviol,
  kMaxRmax2, kMaxDviol2, kMaxDabs2, kMaxPviol2,
  kMaxChkPrimal, kMaxChkDual,
  kNumSlots = 48
};

__device__ __forceinline__ unsigned long long* max_slot(double* res, int s) {
  return reinterpret_cast<unsigned long long*>(res + s);
}

// ---------------------------------------------------------------------- residual
// dx = x̄ − x̂ written as the reference's axpby(−1, x̂, 1, dx) with dx = x̄; terms Δx², and the
// restart distance (x̂ − x0)² (diff_norm2, evaluated in fp64 of the working values).
template <class T>
static __global__ void k_res_x(int n, const T* __restrict__ xb, const T* __restrict__ xh, const T* __restrict__ x0,
                        T* __restrict__ dx, double* t_px, double* t_dxn, const int* skip) {
  if (skip && *skip) return;
  B200_FOR(j, n) {
    const T d = static_cast<T>(-1.0) * xh[j] + static_cast<T>(1.0) * xb[j];
    dx[j] = d;
    t_px[j] = static_cast<double>(d) * static_cast<double>(d);
    if (t_dxn) {
      const double e = static_cast<double>(xh[j]) - static_cast<double>(x0[j]);
      t_dxn[j] = e * e;
    }
  }
}
// Epilogue after adx = Ã·dx: dy = ȳ − ŷ, terms Δy², Δyᵀ(AΔx), (ŷ − y0)².
template <class T>
struct EpiResY {
  const T *yb, *yh, *y0;
  T *dy, *adx;
  double *t_py, *t_cross, *t_dyn;
  const int* skip;
  __device__ bool active() const { return !(skip && *skip); }
  __device__ void operator()(int i, double s) const {
    const T ax = static_cast<T>(s);
    adx[i] = ax;
    const T d = static_cast<T>(-1.0) * yh[i] + static_cast<T>(1.0) * yb[i];
    dy[i] = d;
    t_py[i] = static_cast<double>(d) * static_cast<double>(d);
    t_cross[i] = static_cast<double>(d) * static_cast<double>(ax);
    if (t_dyn) {
      const double e = static_cast<double>(yh[i]) - static_cast<double>(y0[i]);
      t_dyn[i] = e * e;
    }
  }
};

// ---------------------------------------------------------------------- unscale
// x = clamp(C x̃ / bs, l, u), y_min = R ỹ / os (scaling.cpp:144-155)
template <class T>
static __global__ void k_unscale_x(int n, const T* xs, const double* col_scale, double bound_scale, const double* cl,
                            const double* cu, double* xo) {
  B200_FOR(j, n) xo[j] = std_min(std_max(col_scale[j] * static_cast<double>(xs[j]) / bound_scale, cl[j]), cu[j]);
}
template <class T>
static __global__ void k_unscale_y(int m, const T* ys, const double* row_scale, double obj_scale, double* yo) {
  B200_FOR(i, m) yo[i] = row_scale[i] * static_cast<double>(ys[i]) / obj_scale;
}

__device__ __forceinline__ double elem_viol(double v, double lo, double up) {
  if (v < lo) return (lo - v) / (1.0 + fabs(lo));
  if (v > up) return (v - up) / (1.0 + fabs(up));
  return 0.0;
}

// ---------------------------------------------------------------------- KKT
// Row part of kkt_general after ax = A_orig·x (row-sequential). Term arrays have m+n entries:
// rows at [0, m), columns at [m, m+n) so that sums continuing over both loops are one chain.
struct EpiKktRows : AlwaysActive {
  const double *y, *rl, *ru;
  double *t_rp2, *t_d, *t_rd2;
  double* res;
  struct Acc {
    double pmax = 0.0, dmax = 0.0;
  };
  __device__ void operator()(int i, double ax, Acc& acc) const {
    const double lo = rl[i], up = ru[i];
    const double viol = ax < lo ? lo - ax : (ax > up ? ax - up : 0.0);
    t_rp2[i] = viol * viol;
    acc.pmax = elem_viol(ax, lo, up);
    const double yi = y[i];
    double d = 0.0, rd = 0.0;
    if (yi > 0) {
      if (isfinite(lo)) d = yi * lo;
      else rd = yi * yi, acc.dmax = yi;
    } else if (yi < 0) {
      if (isfinite(up)) d = yi * up;
      else rd = yi * yi, acc.dmax = -yi;
    }
    t_d[i] = d;
    t_rd2[i] = rd;
  }
  __device__ void flush(const Acc& a) const {
    warp_max_atomic(max_slot(res, kMaxPmax), a.pmax);
    warp_max_atomic(max_slot(res, kMaxDmax), a.dmax);
  }
};
// Column part after aty = Aᵀ_orig·y (the caller's CSC order).
struct EpiKktCols : AlwaysActive {
  const double *x, *c, *cl, *cu;
  double sense;
  int m;
  double *t_p, *t_d, *t_rd2;
  double* res;
  struct Acc {
    double pmax = 0.0, dmax = 0.0;
  };
  __device__ void operator()(int j, double aty, Acc& acc) const {
    const double cj = sense * c[j];
    t_p[m + j] = cj * x[j];
    const double lo = cl[j], up = cu[j];
    acc.pmax = elem_viol(x[j], lo, up);
    const double lam = cj - aty;
    double z;
    if (isfinite(lo) && isfinite(up)) z = lam;
    else if (isfinite(lo)) z = std_max(lam, 0.0);
    else if (isfinite(up)) z = std_min(lam, 0.0);
    else z = 0.0;
    t_rd2[m + j] = (lam - z) * (lam - z);
    acc.dmax = fabs(lam - z);
    t_d[m + j] = z > 0 ? z * lo : (z < 0 ? z * up : 0.0);
  }
  __device__ void flush(const Acc& a) const {
    warp_max_atomic(max_slot(res, kMaxPmax), a.pmax);
    warp_max_atomic(max_slot(res, kMaxDmax), a.dmax);
  }
};

// ---------------------------------------------------------------------- ray test
// Dual ray r from Δy (rows), primal ray d from Δx (columns), engine.cpp:88-96 / 130-137.
template <class T>
static __global__ void k_ray_r(int m, const T* dy, const double* row_scale, double obj_scale, const double* rl,
                        const double* ru, double* r, double* res, int slot_rmax) {
  double mx = 0.0;
  B200_FOR(i, m) {
    double v = row_scale[i] * static_cast<double>(dy[i]) / obj_scale;
    if (!isfinite(rl[i])) v = std_min(v, 0.0);
    if (!isfinite(ru[i])) v = std_max(v, 0.0);
    r[i] = v;
    mx = std_max(mx, fabs(v));
  }
  warp_max_atomic(max_slot(res, slot_rmax), mx);
}
template <class T>
static __global__ void k_ray_d(int n, const T* dx, const double* col_scale, double bound_scale, const double* cl,
                        const double* cu, double* d, double* res, int slot_dabs) {
  double mx = 0.0;
  B200_FOR(j, n) {
    double v = col_scale[j] * static_cast<double>(dx[j]) / bound_scale;
    if (isfinite(cl[j])) v = std_max(v, 0.0);
    if (isfinite(cu[j])) v = std_min(v, 0.0);
    d[j] = v;
    mx = std_max(mx, fabs(v));
  }
  warp_max_atomic(max_slot(res, slot_dabs), mx);
}
// Columns: g = Aᵀr and gabs = Σ|a r| (CSC order), λ = −g; objective/magnitude terms and the
// dual-ray violation; plus the primal-ray terms cᵀd and Σ|c d| (engine.cpp:97-116, 138-139).
static __global__ void k_ray_cols(int n, int m, const int* cp, const int* ri, const double* v, const double* r,
                           const double* d, const double* c, double sense, const double* cl, const double* cu,
                           double* t_obj, double* t_mag, double* t_cd, double* t_cmag, double* res, int slot_dviol) {
  double dviol = 0.0;
  B200_FOR(j, n) {
    double g = 0.0, gabs = 0.0;
    for (int k = cp[j]; k < cp[j + 1]; ++k) {
      g += v[k] * r[ri[k]];
      gabs += fabs(v[k] * r[ri[k]]);
    }
    const double lam = -g, lo = cl[j], up = cu[j];
    double ob = 0.0, mg = 0.0;
    if (lam > 0) {
      if (isfinite(lo)) ob = lo * lam, mg = gabs * fabs(lo);
      else dviol = std_max(dviol, lam);
    } else if (lam < 0) {
      if (isfinite(up)) ob = up * lam, mg = gabs * fabs(up);
      else dviol = std_max(dviol, -lam);
    }
    t_obj[m + j] = ob;
    t_mag[m + j] = mg;
    t_cd[j] = sense * c[j] * d[j];
    t_cmag[j] = fabs(c[j] * d[j]);
  }
  warp_max_atomic(max_slot(res, slot_dviol), dviol);
}
// Rows after ad = A_orig·d: primal-ray violation; dual-ray objective/magnitude row terms.
struct EpiRayRows : AlwaysActive {
  const double *r, *rl, *ru;
  double *t_obj, *t_mag;
  double* res;
  int slot_pviol;
  struct Acc {
    double pviol = 0.0;
  };
  __device__ void operator()(int i, double ad, Acc& acc) const {
    double v = 0.0;
    if (isfinite(rl[i])) v = std_max(v, -ad);
    if (isfinite(ru[i])) v = std_max(v, ad);
    acc.pviol = v;
    const double ri = r[i];
    const double term = ri > 0 ? rl[i] * ri : (ri < 0 ? ru[i] * ri : 0.0);
    t_obj[i] = term;
    t_mag[i] = fabs(term);
  }
  __device__ void flush(const Acc& a) const { warp_max_atomic(max_slot(res, slot_pviol), a.pviol); }
};

// ---------------------------------------------------------------------- finish
// y = sense · y_min; z_j = c_j − Σ a_ij y_i with the subtractions in CSC order (engine.cpp:283-286)
static __global__ void k_dual_out(int m, double sense, const double* ymin, double* y) {
  B200_FOR(i, m) y[i] = sense * ymin[i];
}
static __global__ void k_reduced_costs(int n, const int* cp, const int* ri, const double* v, const double* c,
                                const double* y, double* z) {
  B200_FOR(j, n) {
    double zz = c[j];
    for (int k = cp[j]; k < cp[j + 1]; ++k) zz -= v[k] * y[ri[k]];
    z[j] = zz;
  }
}
static __global__ void k_obj_terms(int n, const double* c, const double* x, double* t) {
  B200_FOR(j, n) t[j] = c[j] * x[j];
}

// In-process check (solution_checker.cpp:61-133) on the device, for the device-resident path.
__device__ __forceinline__ double bound_violation(double val, double lo, double up) {
  double v = 0.0;
  if (lo != -INFINITY) v = std_max(v, (lo - val) / (1.0 + fabs(lo)));
  if (up != INFINITY) v = std_max(v, (val - up) / (1.0 + fabs(up)));
  return v;
}
__device__ __forceinline__ void multiplier(double mult, double lo, double up, double& viol, double& contrib) {
  viol = 0.0, contrib = 0.0;
  if (mult > 0.0) {
    if (lo == -INFINITY) viol = mult;
    else contrib = mult * lo;
  } else if (mult < 0.0) {
    if (up == INFINITY) viol = -mult;
    else contrib = mult * up;
  }
}
struct EpiCheckRows : AlwaysActive {  // after ax = A·x; y = min-form duals (sense · reported y)
  const double *y, *rl, *ru;
  double c_scale;
  double* t_dual;  // [0, m) rows, [m, m+n) cols
  double* res;
  struct Acc {
    double primal = 0.0, dual = 0.0;
  };
  __device__ void operator()(int i, double ax, Acc& acc) const {
    acc.primal = bound_violation(ax, rl[i], ru[i]);
    double viol, contrib;
    multiplier(y[i], rl[i], ru[i], viol, contrib);
    acc.dual = viol / c_scale;
    t_dual[i] = contrib;
  }
  __device__ void flush(const Acc& a) const {
    warp_max_atomic(max_slot(res, kMaxChkPrimal), a.primal);
    warp_max_atomic(max_slot(res, kMaxChkDual), a.dual);
  }
};
struct EpiCheckCols : AlwaysActive {  // after aty = Aᵀ·y_min (CSC order)
  const double *x, *c, *cl, *cu;
  double sense, c_scale;
  int m;
  double *t_dual, *t_primal;
  double* res;
  struct Acc {
    double primal = 0.0, dual = 0.0;
  };
  __device__ void operator()(int j, double aty, Acc& acc) const {
    acc.primal = bound_violation(x[j], cl[j], cu[j]);
    const double cj = sense * c[j];
    const double d = cj - aty;
    double viol, contrib;
    multiplier(d, cl[j], cu[j], viol, contrib);
    acc.dual = viol / c_scale;
    t_dual[m + j] = contrib;
    t_primal[j] = cj * x[j];
  }
  __device__ void flush(const Acc& a) const {
    warp_max_atomic(max_slot(res, kMaxChkPrimal), a.primal);
    warp_max_atomic(max_slot(res, kMaxChkDual), a.dual);
  }
};
static __global__ void k_scale_copy(long long n, const double* src, double s, double* dst) {
  B200_FOR(i, n) dst[i] = s * src[i];
}

// ---------------------------------------------------------------------- vector helpers
template <class T>
static __global__ void k_fill(long long n, T* v, T a) {
  B200_FOR(i, n) v[i] = a;
}
template <class T>
static __global__ void k_axpby(long long n, T a, const T* x, T b, T* y) {
  B200_FOR(i, n) y[i] = a * x[i] + b * y[i];
}
// x = proj_[l,u](0 − 0·(c − 0)), the reference's primal_step(dx=0, aty=0, τ=0) start point
template <class T>
static __global__ void k_init_x(int n, const T* c, const T* l, const T* u, T* x) {
  B200_FOR(j, n) {
    const T zero = static_cast<T>(0.0);
    x[j] = ref_clamp<T>(zero - zero * (c[j] - zero), l[j], u[j]);
  }
}
// restart at T(z): x = x0 = x̂, y = y0 = ŷ (r2hpdhg.cpp:155-158)
template <class T>
static __global__ void k_restart(int n, int m, const T* xh, T* x, T* x0, const T* yh, T* y, T* y0) {
  B200_FOR(i, (n > m ? n : m)) {
    if (i < n) x[i] = xh[i], x0[i] = xh[i];
    if (i < m) y[i] = yh[i], y0[i] = yh[i];
  }
}

}  // namespace b200
