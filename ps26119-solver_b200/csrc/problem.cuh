// problem.cuh — the scaled problem resident on the device (≙ pdhg::ScaledProblem,
// reference src/pdhg/scaling.h:48-67) and the ‖Ã‖₂ estimate (la::estimate_norm2,
// src/la/csr.cpp:86-132), both computed on the device.
//
// HBM layout (m rows, n cols, nnz nonzeros; int32 indices):
//   A_orig  CSR  a_rp[m+1] a_col[nnz] a_v0[nnz]          (original values, rows sorted by col)
//   Aᵀ_orig CSC  the caller's col_start/row_index/value  (borrowed; original order)
//   Ãᵀ      CSR  col_start[n+1] t_ri[nnz] sat[nnz]       (CSC of Ã, rows sorted inside columns)
//   Ã       CSR  a_rp a_col sa[nnz]                      (shares A_orig's structure)
//   fp32 copies saf / satf and of the scaled vectors for mixed precision.
#pragma once

#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "engine.hpp"
#include "reduce.cuh"
#include "setup.cuh"
#include "spmv.cuh"

namespace b200 {

static __global__ void k_fill_d(long long n, double* v, double a) {
  B200_FOR(i, n) v[i] = a;
}
static __global__ void k_absmax(long long n, const double* v, unsigned long long* key) {
  double mx = 0.0;
  B200_FOR(i, n) mx = std_max(mx, fabs(v[i]));
  warp_max_atomic(key, mx);
}
static __global__ void k_prod_terms(int n, const double* a, const double* b, double* t) {
  B200_FOR(i, n) t[i] = a[i] * b[i];
}
// w[j] -= al*v[j] + bprev*vprev[j]; t[j] = w[j]² (csr.cpp:108-112)
static __global__ void k_lanczos_update(int n, double* w, const double* v, const double* vprev, double al, double bprev,
                                 double* t) {
  B200_FOR(j, n) {
    w[j] -= al * v[j] + bprev * vprev[j];
    t[j] = w[j] * w[j];
  }
}
static __global__ void k_lanczos_next(int n, const double* w, double* v, double* vprev, double bn) {
  B200_FOR(j, n) {
    vprev[j] = v[j];
    v[j] = w[j] / bn;
  }
}
// The same two steps with α and β read from the device, where the sums left them: α = *al,
// β_prev = sqrt(*bsq_prev) (0 without one), β = sqrt(*bsq) — sqrt correctly rounded, as the
// host's std::sqrt. `hist` receives (α, β²) of step k for the host's later replay.
static __global__ void k_lanczos_update_dev(int n, double* w, const double* v, const double* vprev, const double* al,
                                            const double* bsq_prev, double* t) {
  const double a = *al, bp = bsq_prev ? sqrt(*bsq_prev) : 0.0;
  B200_FOR(j, n) {
    w[j] -= a * v[j] + bp * vprev[j];
    t[j] = w[j] * w[j];
  }
}
static __global__ void k_lanczos_next_dev(int n, const double* w, double* v, double* vprev, const double* ab,
                                          double* hist) {
  const double bn = sqrt(ab[1]);
  if (blockIdx.x == 0 && threadIdx.x == 0) hist[0] = ab[0], hist[1] = ab[1];
  B200_FOR(j, n) {
    vprev[j] = v[j];
    v[j] = w[j] / bn;
  }
}


struct ScaledDevice {
  int m = 0, n = 0, sense = 1;
  long long nnz = 0;
  DeviceModel M;
  DevBuf<int> a_rp, a_col, t_ri;
  DevBuf<int> t_rp;  // this library's copy of the caller's col_start (Ãᵀ row pointers, TMA-staged)
  DevBuf<double> a_v0, t_v0, sa, sat;
  DevBuf<float> saf, satf;
  DevBuf<double> row_scale, col_scale;
  DevBuf<double> sc, scl, scu, srl, sru;
  DevBuf<float> scf, sclf, scuf, srlf, sruf;
  double bound_scale = 1.0, obj_scale = 1.0, log10_range = 0.0;
  bool gm_applied = false, have_f32 = false, exact = false;
  // original-space constants of kkt_general (cpu_backend.cpp:233-262): ‖b‖₂, ‖c‖₂, ‖c‖∞
  double b_norm = 0, c_norm = 0, c_inf = 0;
  long long kernels = 0;
  int lanczos_launched = 0;  // Lanczos steps launched by the last lanczos() (counted or not)

  // Scratch for the setup reductions.
  DevBuf<double> tmp_m, tmp_n, fac_m, fac_n, sums;
  DevBuf<unsigned long long> keys;

  void build(const DeviceModel& dm, const ScalingOptions& so, bool exact_order, cudaStream_t st) {
    M = dm;
    m = dm.m, n = dm.n, sense = dm.sense, nnz = dm.nnz;
    exact = exact_order;
    const std::size_t mm = static_cast<std::size_t>(m), nn = static_cast<std::size_t>(n);
    const std::size_t nz = static_cast<std::size_t>(nnz);
    a_rp.alloc(mm + 1);
    t_rp.alloc(nn + 1);
    B200_CHECK(cudaMemcpyAsync(t_rp.get(), dm.col_start, (nn + 1) * sizeof(int), cudaMemcpyDeviceToDevice, st));
    a_col.alloc(nz);
    a_v0.alloc(nz);
    t_ri.alloc(nz);
    t_v0.alloc(nz);
    sa.alloc(nz);
    sat.alloc(nz);
    row_scale.alloc(mm);
    col_scale.alloc(nn);
    tmp_m.alloc(mm + 1);
    tmp_n.alloc(nn + 1);
    fac_m.alloc(mm + 1);
    fac_n.alloc(nn + 1);
    sums.alloc(16);
    keys.alloc(4);

    // ---- CSR of A (la::transpose of the CSC, csr.cpp:19-36)
    {
      DevBuf<int> counts(mm + 1), cursor(mm + 1), long_rows(std::max(mm, nn) + 1), n_long(1);
      B200_CHECK(cudaMemsetAsync(counts.get(), 0, (mm + 1) * sizeof(int), st));
      if (nnz > 0) k_count<<<grid_for(nnz), kBlock, 0, st>>>(nnz, dm.row_index, counts.get());
      B200_LAUNCH_CHECK();
      exclusive_scan(counts.get(), a_rp.get(), static_cast<long long>(mm) + 1, st);
      B200_CHECK(cudaMemcpyAsync(cursor.get(), a_rp.get(), (mm + 1) * sizeof(int), cudaMemcpyDeviceToDevice, st));
      if (n > 0)
        k_scatter<<<grid_for(n), kBlock, 0, st>>>(n, dm.col_start, dm.row_index, dm.value, cursor.get(), a_col.get(),
                                                  a_v0.get());
      B200_LAUNCH_CHECK();
      sort_segments(m, a_rp.get(), a_col.get(), a_v0.get(), long_rows.get(), n_long.get(), st);
      // canonical CSC of A (rows sorted inside each column) = CSR of Aᵀ as la::transpose makes it
      if (nnz > 0) {
        B200_CHECK(cudaMemcpyAsync(t_ri.get(), dm.row_index, nz * sizeof(int), cudaMemcpyDeviceToDevice, st));
        B200_CHECK(cudaMemcpyAsync(t_v0.get(), dm.value, nz * sizeof(double), cudaMemcpyDeviceToDevice, st));
      }
      sort_segments(n, dm.col_start, t_ri.get(), t_v0.get(), long_rows.get(), n_long.get(), st);
      B200_CHECK(cudaStreamSynchronize(st));
    }
    if (nnz > 0) {
      B200_CHECK(cudaMemcpyAsync(sa.get(), a_v0.get(), nz * sizeof(double), cudaMemcpyDeviceToDevice, st));
      B200_CHECK(cudaMemcpyAsync(sat.get(), t_v0.get(), nz * sizeof(double), cudaMemcpyDeviceToDevice, st));
    }
    k_fill_d<<<grid_for(mm), kBlock, 0, st>>>(static_cast<long long>(mm), row_scale.get(), 1.0);
    k_fill_d<<<grid_for(nn), kBlock, 0, st>>>(static_cast<long long>(nn), col_scale.get(), 1.0);
    B200_LAUNCH_CHECK();

    // ---- log10 range of |a| (scaling.cpp:51-56)
    {
      unsigned long long init[2] = {0x7ff0000000000000ULL /* +inf */, 0ULL};
      B200_CHECK(cudaMemcpyAsync(keys.get(), init, sizeof init, cudaMemcpyHostToDevice, st));
      if (nnz > 0) k_abs_range<<<grid_for(nnz), kBlock, 0, st>>>(nnz, a_v0.get(), keys.get(), keys.get() + 1);
      B200_LAUNCH_CHECK();
      unsigned long long got[2];
      B200_CHECK(cudaMemcpyAsync(got, keys.get(), sizeof got, cudaMemcpyDeviceToHost, st));
      B200_CHECK(cudaStreamSynchronize(st));
      double amin, amax;
      std::memcpy(&amin, &got[0], sizeof amin);
      std::memcpy(&amax, &got[1], sizeof amax);
      log10_range = amax > 0 ? std::log10(amax / amin) : 0.0;
    }
    gm_applied = so.geometric_mean_iterations > 0 && log10_range >= so.geometric_mean_min_log10_range;
    if (gm_applied) {  // scaling.cpp:57-80: factors from the ORIGINAL entries, applied once
      for (int it = 0; it < so.geometric_mean_iterations; ++it) {
        k_gm_pass<<<grid_for(mm), kBlock, 0, st>>>(m, a_rp.get(), a_col.get(), a_v0.get(), col_scale.get(),
                                                   row_scale.get());
        k_gm_pass<<<grid_for(nn), kBlock, 0, st>>>(n, dm.col_start, dm.row_index, dm.value, row_scale.get(),
                                                   col_scale.get());
        B200_LAUNCH_CHECK();
      }
      apply(row_scale.get(), col_scale.get(), st);
    }
    for (int it = 0; it < so.ruiz_iterations; ++it) norm_step(true, st);  // scaling.cpp:81-88
    if (so.pock_chambolle) norm_step(false, st);                          // scaling.cpp:89-96

    sc.alloc(nn), scl.alloc(nn), scu.alloc(nn), srl.alloc(mm), sru.alloc(mm);
    k_scaled_cols<<<grid_for(nn), kBlock, 0, st>>>(n, sense, dm.c, dm.col_lower, dm.col_upper, col_scale.get(),
                                                   sc.get(), scl.get(), scu.get());
    k_scaled_rows<<<grid_for(mm), kBlock, 0, st>>>(m, dm.row_lower, dm.row_upper, row_scale.get(), srl.get(),
                                                   sru.get());
    B200_LAUNCH_CHECK();
    if (so.bound_objective_rescaling) {  // scaling.cpp:126-141
      double b2 = 0, c2 = 0;
      seq_sums(st, [&](double* tm, double* tn) {
        k_b2_terms<<<grid_for(mm), kBlock, 0, st>>>(m, srl.get(), sru.get(), tm);
        k_sq_terms<<<grid_for(nn), kBlock, 0, st>>>(static_cast<long long>(nn), sc.get(), tn);
      }, b2, c2);
      bound_scale = 1.0 / (std::sqrt(b2) + 1.0);
      obj_scale = 1.0 / (std::sqrt(c2) + 1.0);
      k_scale_vec<<<grid_for(mm), kBlock, 0, st>>>(static_cast<long long>(mm), srl.get(), bound_scale);
      k_scale_vec<<<grid_for(mm), kBlock, 0, st>>>(static_cast<long long>(mm), sru.get(), bound_scale);
      k_scale_vec<<<grid_for(nn), kBlock, 0, st>>>(static_cast<long long>(nn), scl.get(), bound_scale);
      k_scale_vec<<<grid_for(nn), kBlock, 0, st>>>(static_cast<long long>(nn), scu.get(), bound_scale);
      k_scale_vec<<<grid_for(nn), kBlock, 0, st>>>(static_cast<long long>(nn), sc.get(), obj_scale);
      B200_LAUNCH_CHECK();
    }
    // ---- original-space constants of kkt_general
    {
      double b2 = 0, c2 = 0;
      seq_sums(st, [&](double* tm, double* tn) {
        k_b2_terms<<<grid_for(mm), kBlock, 0, st>>>(m, dm.row_lower, dm.row_upper, tm);
        k_sq_terms<<<grid_for(nn), kBlock, 0, st>>>(static_cast<long long>(nn), dm.c, tn);
      }, b2, c2);
      b_norm = std::sqrt(b2);
      c_norm = std::sqrt(c2);
      B200_CHECK(cudaMemsetAsync(keys.get(), 0, sizeof(unsigned long long), st));
      k_absmax<<<grid_for(nn), kBlock, 0, st>>>(static_cast<long long>(nn), dm.c, keys.get());
      B200_LAUNCH_CHECK();
      unsigned long long key = 0;
      B200_CHECK(cudaMemcpyAsync(&key, keys.get(), sizeof key, cudaMemcpyDeviceToHost, st));
      B200_CHECK(cudaStreamSynchronize(st));
      std::memcpy(&c_inf, &key, sizeof c_inf);
    }
  }

  void make_f32(cudaStream_t st) {
    if (have_f32) return;
    const long long nz = nnz, nn = n, mm = m;
    saf.alloc(static_cast<std::size_t>(nz)), satf.alloc(static_cast<std::size_t>(nz));
    scf.alloc(n), sclf.alloc(n), scuf.alloc(n), srlf.alloc(m), sruf.alloc(m);
    k_convert<float, double><<<grid_for(nz), kBlock, 0, st>>>(nz, sa.get(), saf.get());
    k_convert<float, double><<<grid_for(nz), kBlock, 0, st>>>(nz, sat.get(), satf.get());
    k_convert<float, double><<<grid_for(nn), kBlock, 0, st>>>(nn, sc.get(), scf.get());
    k_convert<float, double><<<grid_for(nn), kBlock, 0, st>>>(nn, scl.get(), sclf.get());
    k_convert<float, double><<<grid_for(nn), kBlock, 0, st>>>(nn, scu.get(), scuf.get());
    k_convert<float, double><<<grid_for(mm), kBlock, 0, st>>>(mm, srl.get(), srlf.get());
    k_convert<float, double><<<grid_for(mm), kBlock, 0, st>>>(mm, sru.get(), sruf.get());
    B200_LAUNCH_CHECK();
    have_f32 = true;
  }

  // Scaled matrix views for SpMV in precision T.
  template <class T> const T* A_val() const;
  template <class T> const T* At_val() const;
  template <class T> const T* c() const;
  template <class T> const T* l() const;
  template <class T> const T* u() const;
  template <class T> const T* rl() const;
  template <class T> const T* ru() const;

  // ‖Ã‖₂ by Lanczos on ÃᵀÃ (csr.cpp:86-132). The start vector is the reference's xorshift64*
  // stream, generated and normalised on the host in the reference's order; the products run
  // on the device; α and β are reduced in the selected order and stay on the device, where the
  // next step's update reads them. The host reads them back once per batch of steps (21, then
  // 8 at a time) and replays the reference's per-step decisions on them (Sturm bisection,
  // breakdown and stagnation tests) in step order: the result and the number of steps that
  // count are the sequential loop's; steps run past the stopping one are discarded.
  double lanczos(cudaStream_t st, unsigned* err = nullptr) {
    if (n == 0 || nnz == 0) return 0.0;
    const int K = 400;
    const double rel_tol = 1e-12;
    std::vector<double> hv(static_cast<std::size_t>(n));
    std::uint64_t state = 0x9E3779B97F4A7C15ULL;
    double nv = 0;
    for (int j = 0; j < n; ++j) {
      state ^= state >> 12, state ^= state << 25, state ^= state >> 27;
      hv[j] = static_cast<double>((state * 0x2545F4914F6CDD1DULL) >> 11) / 9007199254740992.0 * 2.0 - 1.0;
      nv += hv[j] * hv[j];
    }
    nv = std::sqrt(nv);
    for (double& e : hv) e /= nv;
    lanczos_launched = 0;
    DevBuf<double> v(n), vprev(n), w(n), t(m), terms(n);
    B200_CHECK(cudaMemcpyAsync(v.get(), hv.data(), hv.size() * sizeof(double), cudaMemcpyHostToDevice, st));
    B200_CHECK(cudaMemsetAsync(vprev.get(), 0, static_cast<std::size_t>(n) * sizeof(double), st));
    DevBuf<double> out(2), hist(2 * static_cast<std::size_t>(K));
    SumPlan pal, pbn;
    pal.add(terms.get(), 0, n, 0.0, SumOrder::kSeq, out.get());
    pbn.add(terms.get(), 0, n, 0.0, SumOrder::kSeq, out.get() + 1);
    pal.build(true, nullptr, st);  // α and β enter η = 0.998/‖Ã‖₂: always the reference's order
    pbn.build(true, nullptr, st);
    std::vector<double> alpha, beta, h(2 * static_cast<std::size_t>(K));
    double theta = 0, theta_old = -1;
    int stagnant = 0;
    int done = 0;  // steps launched
    for (;;) {
      const int batch = std::min(K - done, done == 0 ? 21 : 8);
      for (int k = done; k < done + batch; ++k) {
        launch_slab_tma<double>(m, a_rp.get(), a_col.get(), sa.get(), v.get(), EpiStore<double>{{}, t.get()}, st,
                                nullptr, err);
        launch_slab_tma<double>(n, M.col_start, t_ri.get(), sat.get(), t.get(), EpiStore<double>{{}, w.get()}, st,
                                nullptr, err);
        k_prod_terms<<<grid_for(n), kBlock, 0, st>>>(n, w.get(), v.get(), terms.get());
        B200_LAUNCH_CHECK();
        pal.launch(st);
        // β of the previous step is still in out[1]: this step's β² overwrites it only below
        k_lanczos_update_dev<<<grid_for(n), kBlock, 0, st>>>(n, w.get(), v.get(), vprev.get(), out.get(),
                                                              k > 0 ? out.get() + 1 : nullptr, terms.get());
        B200_LAUNCH_CHECK();
        pbn.launch(st);
        k_lanczos_next_dev<<<grid_for(n), kBlock, 0, st>>>(n, w.get(), v.get(), vprev.get(), out.get(),
                                                            hist.get() + 2 * k);
        B200_LAUNCH_CHECK();
        kernels += 5 + pal.kernel_count() + pbn.kernel_count();
      }
      lanczos_launched = done + batch;
      B200_CHECK(cudaMemcpyAsync(h.data() + 2 * done, hist.get() + 2 * done, 2 * batch * sizeof(double),
                                 cudaMemcpyDeviceToHost, st));
      B200_CHECK(cudaStreamSynchronize(st));
      for (int k = done; k < done + batch; ++k) {  // the reference's loop body, step by step
        const double al = h[2 * k], bn = std::sqrt(h[2 * k + 1]);
        alpha.push_back(al);
        theta = tridiag_max_eig(alpha, beta, static_cast<int>(alpha.size()));
        if (bn <= 1e-14 * std_max(1.0, theta)) return std::sqrt(std_max(theta, 0.0)) * (1.0 + 1e-4);
        beta.push_back(bn);
        if (theta - theta_old <= rel_tol * theta) {
          if (++stagnant >= 5 && k >= 20) return std::sqrt(std_max(theta, 0.0)) * (1.0 + 1e-4);
        } else {
          stagnant = 0;
        }
        theta_old = theta;
      }
      done += batch;
      if (done >= K) return std::sqrt(std_max(theta, 0.0)) * (1.0 + 1e-4);
    }
  }

  // Largest eigenvalue of the Lanczos tridiagonal by Sturm bisection (csr.cpp:54-84).
  static double tridiag_max_eig(const std::vector<double>& a, const std::vector<double>& b, int k) {
    double lo = 1e300, hi = -1e300;
    for (int i = 0; i < k; ++i) {
      const double r = (i > 0 ? std::fabs(b[i - 1]) : 0.0) + (i + 1 < k ? std::fabs(b[i]) : 0.0);
      lo = std_min(lo, a[i] - r);
      hi = std_max(hi, a[i] + r);
    }
    for (int it = 0; it < 200 && hi - lo > 1e-15 * std_max(1.0, std::fabs(hi)); ++it) {
      const double mid = 0.5 * (lo + hi);
      int c = 0;
      double d = 1.0;
      for (int i = 0; i < k; ++i) {
        const double bb = i > 0 ? b[i - 1] * b[i - 1] : 0.0;
        d = (a[i] - mid) - (i > 0 ? bb / d : 0.0);
        if (d == 0.0) d = -1e-300;
        if (d < 0) ++c;
      }
      if (c == k) hi = mid;
      else lo = mid;
    }
    return hi;
  }

 private:
  static void sort_segments(int rows, const int* rp, int* key, double* val, int* long_rows, int* n_long,
                                     cudaStream_t st) {
    if (rows <= 0) return;
    B200_CHECK(cudaMemsetAsync(n_long, 0, sizeof(int), st));
    k_sort_short<<<grid_for(rows), kBlock, 0, st>>>(rows, rp, key, val, long_rows, n_long);
    B200_LAUNCH_CHECK();
    k_sort_long<<<148, 512, 0, st>>>(rp, long_rows, n_long, key, val);
    B200_LAUNCH_CHECK();
  }

  void apply(const double* rf, const double* cf, cudaStream_t st) {
    k_apply_csr<<<grid_for(m), kBlock, 0, st>>>(m, a_rp.get(), a_col.get(), sa.get(), rf, cf);
    k_apply_csc<<<grid_for(n), kBlock, 0, st>>>(n, M.col_start, t_ri.get(), sat.get(), rf, cf);
    B200_LAUNCH_CHECK();
  }

  // One Ruiz (∞-norm) or Pock–Chambolle (1-norm, α = 1) step: factors 1/sqrt(norm), applied to
  // Ã and Ãᵀ, accumulated into the scales.
  void norm_step(bool inf_norm, cudaStream_t st) {
    DevBuf<double>& rf = fac_m;
    DevBuf<double>& cf = fac_n;
    k_row_norm<<<grid_for(m), kBlock, 0, st>>>(m, a_rp.get(), sa.get(), inf_norm ? 1 : 0, tmp_m.get());
    k_row_norm<<<grid_for(n), kBlock, 0, st>>>(n, M.col_start, sat.get(), inf_norm ? 1 : 0, tmp_n.get());
    k_inv_sqrt_factor<<<grid_for(m), kBlock, 0, st>>>(m, tmp_m.get(), rf.get(), row_scale.get());
    k_inv_sqrt_factor<<<grid_for(n), kBlock, 0, st>>>(n, tmp_n.get(), cf.get(), col_scale.get());
    B200_LAUNCH_CHECK();
    apply(rf.get(), cf.get(), st);
  }

  // Two sequential-order sums: terms over m (into tmp_m) and over n (into tmp_n).
  template <class F>
  void seq_sums(cudaStream_t st, F&& fill_terms, double& sm, double& sn) {
    fill_terms(tmp_m.get(), tmp_n.get());
    B200_LAUNCH_CHECK();
    SumPlan p;
    p.add(tmp_m.get(), 0, m, 0.0, SumOrder::kSeq, sums.get());
    p.add(tmp_n.get(), 0, n, 0.0, SumOrder::kSeq, sums.get() + 1);
    p.build(true, nullptr, st);  // norms that enter the scaled data: always the reference's order
    p.launch(st);
    double h[2];
    B200_CHECK(cudaMemcpyAsync(h, sums.get(), sizeof h, cudaMemcpyDeviceToHost, st));
    B200_CHECK(cudaStreamSynchronize(st));
    sm = h[0], sn = h[1];
  }

};

template <> inline const double* ScaledDevice::A_val<double>() const { return sa.get(); }
template <> inline const float* ScaledDevice::A_val<float>() const { return saf.get(); }
template <> inline const double* ScaledDevice::At_val<double>() const { return sat.get(); }
template <> inline const float* ScaledDevice::At_val<float>() const { return satf.get(); }
template <> inline const double* ScaledDevice::c<double>() const { return sc.get(); }
template <> inline const float* ScaledDevice::c<float>() const { return scf.get(); }
template <> inline const double* ScaledDevice::l<double>() const { return scl.get(); }
template <> inline const float* ScaledDevice::l<float>() const { return sclf.get(); }
template <> inline const double* ScaledDevice::u<double>() const { return scu.get(); }
template <> inline const float* ScaledDevice::u<float>() const { return scuf.get(); }
template <> inline const double* ScaledDevice::rl<double>() const { return srl.get(); }
template <> inline const float* ScaledDevice::rl<float>() const { return srlf.get(); }
template <> inline const double* ScaledDevice::ru<double>() const { return sru.get(); }
template <> inline const float* ScaledDevice::ru<float>() const { return sruf.get(); }

}  // namespace b200
