// backend.cu — the reference's pdhg::Backend plugin interface (src/pdhg/backend.h:36-69)
// on the GPU: vectors addressed by handles, working precision fp64 or fp32, every O(n)/O(nnz)
// op a kernel. It shares the engine's kernels and epilogue functors, so an op-by-op comparison
// against the reference CpuBackend (the check of tests/unit/test_gpu.cpp:33-95) exercises the
// exact arithmetic the engine uses, fused forms included.
#include <cmath>
#include <memory>
#include <string>
#include <vector>

#include "../../include/ps26119.h"
#include "../../include/ps26119_backend.h"
#include "checks.cuh"
#include "engine.hpp"
#include "problem.cuh"

namespace b200 {
namespace {

template <class T>
__global__ void k_pair_terms(long long n, const T* a, const T* b, bool diff, double* t) {
  B200_FOR(i, n) {
    const double x = static_cast<double>(a[i]), y = static_cast<double>(b[i]);
    if (diff) {
      const double d = x - y;
      t[i] = d * d;
    } else {
      t[i] = x * y;
    }
  }
}

class GpuBackendImpl final : public GpuBackend {
 public:
  GpuBackendImpl(const HostModelView& H, const ScalingOptions& so, bool exact) : exact_(exact) {
    B200_CHECK(cudaStreamCreateWithFlags(&st_, cudaStreamNonBlocking));
    m_ = H.m, n_ = H.n;
    const long long nnz = H.col_start[n_];
    c_.upload(H.c, n_, st_), cl_.upload(H.col_lower, n_, st_), cu_.upload(H.col_upper, n_, st_);
    rl_.upload(H.row_lower, m_, st_), ru_.upload(H.row_upper, m_, st_);
    cs_.upload(H.col_start, static_cast<std::size_t>(n_) + 1, st_);
    ri_.upload(H.row_index, static_cast<std::size_t>(nnz), st_);
    v_.upload(H.value, static_cast<std::size_t>(nnz), st_);
    M_.m = m_, M_.n = n_, M_.sense = H.sense, M_.offset = H.offset, M_.nnz = nnz;
    M_.c = c_.get(), M_.col_lower = cl_.get(), M_.col_upper = cu_.get(), M_.row_lower = rl_.get();
    M_.row_upper = ru_.get(), M_.col_start = cs_.get(), M_.row_index = ri_.get(), M_.value = v_.get();
    sp_.build(M_, so, exact, st_);
    sp_.make_f32(st_);
    xo_.alloc(n_), yo_.alloc(m_), terms_.alloc(4 * (static_cast<std::size_t>(m_) + n_)), res_.alloc(kNumSlots);
    out_.alloc(4);
    B200_CHECK(cudaStreamSynchronize(st_));
  }
  ~GpuBackendImpl() override { cudaStreamDestroy(st_); }

  void set_precision(bool mixed) override {
    if (mixed == mixed_) return;
    for (std::size_t k = 0; k < sizes_.size(); ++k) {
      const long long len = sizes_[k];
      if (mixed) k_convert<float, double><<<grid_for(len), kBlock, 0, st_>>>(len, d_[k].get(), f_[k].get());
      else k_convert<double, float><<<grid_for(len), kBlock, 0, st_>>>(len, f_[k].get(), d_[k].get());
    }
    B200_LAUNCH_CHECK();
    mixed_ = mixed;
  }
  bool mixed() const override { return mixed_; }
  int create_vector(bool dual) override {
    const long long len = dual ? m_ : n_;
    d_.emplace_back(static_cast<std::size_t>(len));
    f_.emplace_back(static_cast<std::size_t>(len));
    B200_CHECK(cudaMemsetAsync(d_.back().get(), 0, len * sizeof(double), st_));
    B200_CHECK(cudaMemsetAsync(f_.back().get(), 0, len * sizeof(float), st_));
    sizes_.push_back(len);
    return static_cast<int>(sizes_.size()) - 1;
  }
  void upload(int v, const double* src) override {
    const long long len = sizes_[v];
    if (!mixed_) {
      B200_CHECK(cudaMemcpyAsync(d_[v].get(), src, len * sizeof(double), cudaMemcpyHostToDevice, st_));
    } else {
      std::vector<float> f(src, src + len);
      B200_CHECK(cudaMemcpyAsync(f_[v].get(), f.data(), len * sizeof(float), cudaMemcpyHostToDevice, st_));
    }
    B200_CHECK(cudaStreamSynchronize(st_));
  }
  void download(int v, double* dst) override {
    const long long len = sizes_[v];
    if (!mixed_) {
      B200_CHECK(cudaMemcpyAsync(dst, d_[v].get(), len * sizeof(double), cudaMemcpyDeviceToHost, st_));
      B200_CHECK(cudaStreamSynchronize(st_));
    } else {
      std::vector<float> f(static_cast<std::size_t>(len));
      B200_CHECK(cudaMemcpyAsync(f.data(), f_[v].get(), len * sizeof(float), cudaMemcpyDeviceToHost, st_));
      B200_CHECK(cudaStreamSynchronize(st_));
      for (long long i = 0; i < len; ++i) dst[i] = f[i];
    }
  }
  void fill(int v, double a) override {
    const long long len = sizes_[v];
    if (mixed_) k_fill<float><<<grid_for(len), kBlock, 0, st_>>>(len, f_[v].get(), static_cast<float>(a));
    else k_fill<double><<<grid_for(len), kBlock, 0, st_>>>(len, d_[v].get(), a);
    B200_LAUNCH_CHECK();
  }
  void copy(int dst, int src) override {
    const long long len = sizes_[dst];
    if (mixed_) B200_CHECK(cudaMemcpyAsync(f_[dst].get(), f_[src].get(), len * sizeof(float), cudaMemcpyDeviceToDevice, st_));
    else B200_CHECK(cudaMemcpyAsync(d_[dst].get(), d_[src].get(), len * sizeof(double), cudaMemcpyDeviceToDevice, st_));
  }
  void axpby(double a, int x, double b, int y) override {  // y ← a·x + b·y in the working type
    const long long len = sizes_[y];
    if (mixed_)
      k_axpby<float><<<grid_for(len), kBlock, 0, st_>>>(len, static_cast<float>(a), f_[x].get(), static_cast<float>(b),
                                                        f_[y].get());
    else k_axpby<double><<<grid_for(len), kBlock, 0, st_>>>(len, a, d_[x].get(), b, d_[y].get());
    B200_LAUNCH_CHECK();
  }
  void spmv(int x, int out) override {
    if (mixed_) launch_slab_tma<float>(m_, sp_.a_rp.get(), sp_.a_col.get(), sp_.saf.get(), f_[x].get(), EpiStore<float>{{}, f_[out].get()}, st_);
    else launch_slab_tma<double>(m_, sp_.a_rp.get(), sp_.a_col.get(), sp_.sa.get(), d_[x].get(), EpiStore<double>{{}, d_[out].get()}, st_);
  }
  void spmv_t(int y, int out) override {
    if (mixed_) launch_slab_tma<float>(n_, cs_.get(), sp_.t_ri.get(), sp_.satf.get(), f_[y].get(), EpiStore<float>{{}, f_[out].get()}, st_);
    else launch_slab_tma<double>(n_, cs_.get(), sp_.t_ri.get(), sp_.sat.get(), d_[y].get(), EpiStore<double>{{}, d_[out].get()}, st_);
  }
  double dot(int a, int b) override { return pair_sum(a, b, false); }
  double norm2(int a) override { return std::sqrt(pair_sum(a, a, false)); }
  double diff_norm2(int a, int b) override { return std::sqrt(pair_sum(a, b, true)); }

  void primal_step(int x, int aty, double tau, int xh) override {
    if (mixed_) k_elementwise<float><<<grid_for(n_), kBlock, 0, st_>>>(n_, f_[aty].get(), EpiPrimalStep<float>{{}, f_[x].get(), sp_.scf.get(), sp_.sclf.get(), sp_.scuf.get(), f_[xh].get(), tau});
    else k_elementwise<double><<<grid_for(n_), kBlock, 0, st_>>>(n_, d_[aty].get(), EpiPrimalStep<double>{{}, d_[x].get(), sp_.sc.get(), sp_.scl.get(), sp_.scu.get(), d_[xh].get(), tau});
    B200_LAUNCH_CHECK();
  }
  void dual_step(int y, int ax, double sigma, int yh) override {
    if (mixed_) k_elementwise<float><<<grid_for(m_), kBlock, 0, st_>>>(m_, f_[ax].get(), EpiDualStep<float>{{}, f_[y].get(), sp_.srlf.get(), sp_.sruf.get(), f_[yh].get(), sigma});
    else k_elementwise<double><<<grid_for(m_), kBlock, 0, st_>>>(m_, d_[ax].get(), EpiDualStep<double>{{}, d_[y].get(), sp_.srl.get(), sp_.sru.get(), d_[yh].get(), sigma});
    B200_LAUNCH_CHECK();
  }
  template <class T>
  EpiPrimal<T> epi_primal(int x, int x0, double tau, double w, double rho, int xh, int xb) {
    auto& V = vec<T>();
    return EpiPrimal<T>{V[x].get(), V[xh].get(), V[xb].get(), V[x0].get(), sp_.c<T>(), sp_.l<T>(), sp_.u<T>(), nullptr, 0, tau, w, rho};
  }
  template <class T>
  EpiDual<T> epi_dual(int y, int y0, double sigma, double w, double rho, int yh, int yb) {
    auto& V = vec<T>();
    return EpiDual<T>{V[y].get(), V[yh].get(), yb >= 0 ? V[yb].get() : nullptr, V[y0].get(), sp_.rl<T>(), sp_.ru<T>(),
                      nullptr, 0, sigma, w, rho, yb >= 0 ? 1 : 0};
  }
  void r2h_primal(int x, int x0, int aty, double tau, double w, double rho, int xh, int xb) override {
    if (mixed_) k_elementwise<float><<<grid_for(n_), kBlock, 0, st_>>>(n_, f_[aty].get(), epi_primal<float>(x, x0, tau, w, rho, xh, xb));
    else k_elementwise<double><<<grid_for(n_), kBlock, 0, st_>>>(n_, d_[aty].get(), epi_primal<double>(x, x0, tau, w, rho, xh, xb));
    B200_LAUNCH_CHECK();
  }
  void r2h_dual(int y, int y0, int ax, double sigma, double w, double rho, int yh, int yb) override {
    if (mixed_) k_elementwise<float><<<grid_for(m_), kBlock, 0, st_>>>(m_, f_[ax].get(), epi_dual<float>(y, y0, sigma, w, rho, yh, yb));
    else k_elementwise<double><<<grid_for(m_), kBlock, 0, st_>>>(m_, d_[ax].get(), epi_dual<double>(y, y0, sigma, w, rho, yh, yb));
    B200_LAUNCH_CHECK();
  }
  void fused_primal(int y, int x, int x0, double tau, double w, double rho, int xh, int xb) override {
    if (mixed_) launch_slab_tma<float>(n_, cs_.get(), sp_.t_ri.get(), sp_.satf.get(), f_[y].get(), epi_primal<float>(x, x0, tau, w, rho, xh, xb), st_);
    else launch_slab_tma<double>(n_, cs_.get(), sp_.t_ri.get(), sp_.sat.get(), d_[y].get(), epi_primal<double>(x, x0, tau, w, rho, xh, xb), st_);
  }
  void fused_dual(int xb, int y, int y0, double sigma, double w, double rho, int yh, int yb) override {
    if (mixed_) launch_slab_tma<float>(m_, sp_.a_rp.get(), sp_.a_col.get(), sp_.saf.get(), f_[xb].get(), epi_dual<float>(y, y0, sigma, w, rho, yh, yb), st_);
    else launch_slab_tma<double>(m_, sp_.a_rp.get(), sp_.a_col.get(), sp_.sa.get(), d_[xb].get(), epi_dual<double>(y, y0, sigma, w, rho, yh, yb), st_);
  }

  // Backend::kkt (cpu_backend.cpp:269-276 + 226-284) on the device.
  void kkt(int xs, int ys, double* out) override {
    if (mixed_) kkt_t<float>(xs, ys, out);
    else kkt_t<double>(xs, ys, out);
  }
  template <class T>
  void kkt_t(int xs, int ys, double* out) {
    auto& V = vec<T>();
    const long long L = static_cast<long long>(m_) + n_;
    B200_CHECK(cudaMemsetAsync(res_.get(), 0, kNumSlots * sizeof(double), st_));
    k_unscale_x<T><<<grid_for(n_), kBlock, 0, st_>>>(n_, V[xs].get(), sp_.col_scale.get(), sp_.bound_scale, M_.col_lower, M_.col_upper, xo_.get());
    k_unscale_y<T><<<grid_for(m_), kBlock, 0, st_>>>(m_, V[ys].get(), sp_.row_scale.get(), sp_.obj_scale, yo_.get());
    B200_LAUNCH_CHECK();
    double* K0 = terms_.get();
    EpiKktRows er{{}, yo_.get(), M_.row_lower, M_.row_upper, K0, K0 + L, K0 + 2 * L, res_.get()};
    launch_slab_tma<double>(m_, sp_.a_rp.get(), sp_.a_col.get(), sp_.a_v0.get(), xo_.get(), er, st_);
    EpiKktCols ec{{}, xo_.get(), M_.c, M_.col_lower, M_.col_upper, static_cast<double>(M_.sense), m_, K0 + 3 * L, K0 + L, K0 + 2 * L, res_.get()};
    launch_slab<double>(n_, M_.col_start, M_.row_index, M_.value, yo_.get(), ec, st_);
    SumPlan p;
    double* R = res_.get();
    p.add(K0, 0, m_, 0.0, SumOrder::kSeq, R + kRp2);
    p.add(K0 + L, 0, L, 0.0, SumOrder::kSeq, R + kD);
    p.add(K0 + 2 * L, 0, L, 0.0, SumOrder::kSeq, R + kRd2);
    p.add(K0 + 3 * L, m_, L, 0.0, SumOrder::kSeq, R + kP);
    p.build(exact_, nullptr, st_);
    p.launch(st_);
    double h[kNumSlots];
    B200_CHECK(cudaMemcpyAsync(h, res_.get(), sizeof h, cudaMemcpyDeviceToHost, st_));
    B200_CHECK(cudaStreamSynchronize(st_));
    out[0] = std::sqrt(h[kRp2]);
    out[1] = std::sqrt(h[kRd2]);
    out[2] = h[kP];
    out[3] = h[kD];
    out[4] = sp_.b_norm;
    out[5] = sp_.c_norm;
    out[6] = h[kMaxPmax];
    out[7] = h[kMaxDmax] / (1.0 + sp_.c_inf);
  }

  long long scaled_get(int which, double* dst) override {
    const double* src = nullptr;
    long long len = 0;
    switch (which) {
      case 0: src = sp_.sa.get(), len = sp_.nnz; break;
      case 1: src = sp_.sat.get(), len = sp_.nnz; break;
      case 2: src = sp_.sc.get(), len = n_; break;
      case 3: src = sp_.scl.get(), len = n_; break;
      case 4: src = sp_.scu.get(), len = n_; break;
      case 5: src = sp_.srl.get(), len = m_; break;
      case 6: src = sp_.sru.get(), len = m_; break;
      case 7: src = sp_.row_scale.get(), len = m_; break;
      case 8: src = sp_.col_scale.get(), len = n_; break;
      default: return -1;
    }
    if (dst && len > 0) {
      B200_CHECK(cudaMemcpyAsync(dst, src, len * sizeof(double), cudaMemcpyDeviceToHost, st_));
      B200_CHECK(cudaStreamSynchronize(st_));
    }
    return len;
  }
  long long scaled_structure(int which, int* row_ptr, int* col) override {
    const int rows = which == 0 ? m_ : n_;
    const int* rp = which == 0 ? sp_.a_rp.get() : cs_.get();
    const int* cc = which == 0 ? sp_.a_col.get() : sp_.t_ri.get();
    if (row_ptr) B200_CHECK(cudaMemcpyAsync(row_ptr, rp, (rows + 1) * sizeof(int), cudaMemcpyDeviceToHost, st_));
    if (col && sp_.nnz > 0) B200_CHECK(cudaMemcpyAsync(col, cc, sp_.nnz * sizeof(int), cudaMemcpyDeviceToHost, st_));
    B200_CHECK(cudaStreamSynchronize(st_));
    return sp_.nnz;
  }
  void scalars(double* out) override {
    out[0] = sp_.bound_scale;
    out[1] = sp_.obj_scale;
    out[2] = sp_.log10_range;
    out[3] = sp_.gm_applied ? 1.0 : 0.0;
  }
  double norm2_estimate() override { return sp_.lanczos(st_); }
  void sync() override { B200_CHECK(cudaStreamSynchronize(st_)); }

 private:
  template <class T> std::vector<DevBuf<T>>& vec();

  // la::parallel_sum over (a·b) or (a − b)² in fp64 of the working values (exact: 64 chunks).
  double pair_sum(int a, int b, bool diff) {
    const long long len = sizes_[a];
    if (mixed_) k_pair_terms<float><<<grid_for(len), kBlock, 0, st_>>>(len, f_[a].get(), f_[b].get(), diff, terms_.get());
    else k_pair_terms<double><<<grid_for(len), kBlock, 0, st_>>>(len, d_[a].get(), d_[b].get(), diff, terms_.get());
    B200_LAUNCH_CHECK();
    SumPlan p;
    p.add(terms_.get(), 0, len, 0.0, SumOrder::kChunk64, out_.get());
    p.build(exact_, nullptr, st_);
    p.launch(st_);
    double r = 0;
    B200_CHECK(cudaMemcpyAsync(&r, out_.get(), sizeof r, cudaMemcpyDeviceToHost, st_));
    B200_CHECK(cudaStreamSynchronize(st_));
    return r;
  }
  cudaStream_t st_ = nullptr;
  bool exact_ = false, mixed_ = false;
  int m_ = 0, n_ = 0;
  DevBuf<double> c_, cl_, cu_, rl_, ru_, v_, xo_, yo_, terms_, res_, out_;
  DevBuf<int> cs_, ri_;
  DeviceModel M_;
  ScaledDevice sp_;
  std::vector<DevBuf<double>> d_;
  std::vector<DevBuf<float>> f_;
  std::vector<long long> sizes_;
};

template <> std::vector<DevBuf<double>>& GpuBackendImpl::vec<double>() { return d_; }
template <> std::vector<DevBuf<float>>& GpuBackendImpl::vec<float>() { return f_; }

}  // namespace

std::unique_ptr<GpuBackend> GpuBackend::create(const HostModelView& M, const ScalingOptions& so, bool exact) {
  require_device();
  return std::make_unique<GpuBackendImpl>(M, so, exact);
}

}  // namespace b200

namespace b200 {
void set_backend_error(const std::string& text);  // c_api.cpp: the thread's last-error text
}

// Σ of a device vector in one of the reference's two summation orders (see the header).
extern "C" int ps26119_ordered_sum(long long n, const double* t, double init, int order, int exact, double* out,
                                   void* stream) {
  using namespace b200;
  if (n < 0 || !out || (n > 0 && !t) || (order != 0 && order != 1)) {
    set_backend_error("invalid arguments: n >= 0, t and out non-NULL, order 0 or 1");
    return PS26119_INVALID_ARGUMENT;
  }
  try {
    require_device();
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    DevBuf<double> d(1);
    SumPlan p;
    p.add(t, 0, n, init, order == 1 ? SumOrder::kChunk64 : SumOrder::kSeq, d.get());
    p.build(exact != 0, nullptr, st);
    p.launch(st);
    B200_CHECK(cudaMemcpyAsync(out, d.get(), sizeof(double), cudaMemcpyDeviceToHost, st));
    B200_CHECK(cudaStreamSynchronize(st));
    return 0;
  } catch (const std::bad_alloc&) {
    set_backend_error("out of memory");
    return PS26119_NOT_SOLVED;
  } catch (const std::exception& e) {
    set_backend_error(e.what());
    return PS26119_NUMERICAL_ERROR;
  }
}
