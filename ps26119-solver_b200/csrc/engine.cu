// engine.cu — the r²HPDHG solve on the device (≙ pdhg::solve_r2hpdhg, reference
// src/pdhg/r2hpdhg.cpp:11-162, with EngineContext src/pdhg/engine.cpp:195-307).
//
// Execution model:
//   * One CUDA stream per solve. Setup (structure, scaling, ‖Ã‖₂) runs on the device.
//   * An EPOCH = K iterations, captured once per precision as a CUDA graph: 2K fused kernels
//     (Ãᵀy + primal update, Ãx̄ + dual update) plus the epoch-start residual section, which
//     returns at once unless the epoch starts a Halpern cycle (inner = 0). The step scalars
//     (τ, σ, the Halpern counter) live in device memory and are refreshed by one small copy
//     before each replay, so the graph is never rebuilt.
//   * A CHECK after each epoch is a second graph (three variants: without ray test, with it,
//     with the drift test as well). It ends by copying one small status block to pinned host
//     memory; the host then takes exactly the reference's decisions (termination, ray test,
//     precision promotion, restart, PID primal weight) in fp64 with the same libm calls.
//   * In exact mode every sum uses the reference's order, so the whole trajectory is
//     bit-identical to the reference CPU engine; in fast mode only the reductions differ
//     (fixed-order trees), by rounding.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <exception>
#include <limits>
#include <map>
#include <memory>
#include <mutex>
#include <utility>
#include <string>
#include <thread>
#include <vector>

#include "checks.cuh"
#include "engine.hpp"
#include "parallel.hpp"
#include "problem.cuh"
#include "tune.hpp"

namespace b200 {

const char* status_name(Status s) {
  switch (s) {
    case Status::Optimal: return "Optimal";
    case Status::Infeasible: return "Infeasible";
    case Status::Unbounded: return "Unbounded";
    case Status::IterationLimit: return "IterationLimit";
    case Status::TimeLimit: return "TimeLimit";
    case Status::NumericalError: return "NumericalError";
    default: return "NotSolved";
  }
}

void require_device() {
  int count = 0;
  const cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess) {
    (void)cudaGetLastError();
    throw std::runtime_error(std::string("no CUDA device: ") + cudaGetErrorString(e));
  }
  if (count == 0) throw std::runtime_error("no CUDA device");
}

namespace {

constexpr double kFirstOrderFast = 1e-4, kFirstOrderInfeasible = 1e-8, kMixedPrecisionSwitch = 1e-6;
constexpr double kVerifyPrimal = 1e-6, kVerifyDual = 1e-6, kVerifyGap = 1e-6;

// termination.h:35-60
struct Kkt {
  double primal_residual = 0, dual_residual = 0, primal_obj = 0, dual_obj = 0, b_norm = 0, c_norm = 0;
  double primal_max_rel = 0, dual_max_rel = 0, obj_shift = 0;
  double rel_primal() const { return primal_residual / (1.0 + b_norm); }
  double rel_dual() const { return dual_residual / (1.0 + c_norm); }
  double rel_gap() const {
    return std::fabs(primal_obj - dual_obj) / (1.0 + std::fabs(primal_obj + obj_shift) + std::fabs(dual_obj + obj_shift));
  }
  double rel_kkt() const {
    double mx = rel_primal();
    if (mx < rel_dual()) mx = rel_dual();
    if (mx < rel_gap()) mx = rel_gap();
    return mx;
  }
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

double slot_max(const double* h, int s) { return h[s]; }  // bit pattern of a non-negative double

template <class T>
struct IterVecs {
  DevBuf<T> x, x0, xh, xb, dx, ddx, y, y0, yh, yb, dy, adx, ddy;
  void alloc(int n, int m) {
    for (DevBuf<T>* v : {&x, &x0, &xh, &xb, &dx, &ddx}) v->alloc(static_cast<std::size_t>(n));
    for (DevBuf<T>* v : {&y, &y0, &yh, &yb, &dy, &adx, &ddy}) v->alloc(static_cast<std::size_t>(m));
  }
};

template <class T>
__global__ void k_diff(long long n, const T* a, const T* b, T* out) {  // out = a − b as axpby(−1, b, 1, out=a)
  B200_FOR(i, n) out[i] = static_cast<T>(-1.0) * b[i] + static_cast<T>(1.0) * a[i];
}

class Engine {
 public:
  Engine(const DeviceModel& M, const EngineOptions& o, cudaStream_t st) : M_(M), o_(o), st_(st) {
    for (auto& e : ev_) B200_CHECK(cudaEventCreate(&e));
  }
  ~Engine() {
#ifdef B200_TEARDOWN_TRACE
    const auto tt0 = std::chrono::steady_clock::now();
#endif
    for (auto& g : g_epoch_)
      if (g) cudaGraphExecDestroy(g);
    for (auto& row : g_check_)
      for (auto& g : row)
        if (g) cudaGraphExecDestroy(g);
    for (auto& row : g_pdlp_)
      for (auto& g : row)
        if (g) cudaGraphExecDestroy(g);
    for (auto& a : g_pdlp_chk_)
      for (auto& row : a)
        for (auto& g : row)
          if (g) cudaGraphExecDestroy(g);
    for (auto& e : ev_)
      if (e) cudaEventDestroy(e);
    for (auto& e : fork_)
      if (e) cudaEventDestroy(e);
    for (auto& q : side_)
      if (q) cudaStreamDestroy(q);
#ifdef B200_TEARDOWN_TRACE
    std::fprintf(stderr, "teardown: graphs+events %.1f ms\n",
                 std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - tt0).count());
#endif
  }

  EngineResult run(const DeviceOutputs& out);
  EngineResult run_pdlp(const DeviceOutputs& out);
  // run() as steps, for a scheduler that interleaves several engines on one stream:
  // start() once (true: finished already); then per epoch begin_epoch(), the epoch's iteration
  // kernels (launch_epoch(), or a scheduler's grouped kernels followed by launch_r0()),
  // launch_check(), a synchronisation of the stream, end_epoch() (true: finished). result()
  // holds the outcome once finished.
  bool start(const DeviceOutputs& out);
  void begin_epoch();
  void launch_epoch();
  void launch_r0(cudaStream_t on);
  void launch_check();
  bool end_epoch();
  const EngineResult& result() const { return R_; }
  int check_every() const { return o_.check_every; }
  cudaStream_t stream() const { return st_; }
  bool mixed_now() const { return mixed_now_; }
  // the operands of this engine's iteration kernels at step s of the current epoch
  template <class T> EpiPrimal<T> primal_epi(int s);
  template <class T> EpiDual<T> dual_epi(int s);
  struct SlabOperands {
    int rows, cap;
    const int *rp, *col;
    const void *val, *x;
    const int2* slab;
    unsigned* err;
  };
  template <class T> SlabOperands primal_operands();
  template <class T> SlabOperands dual_operands();
  // Bulk-copy waits of this solve's kernels that ran out (synchronises the stream).
  unsigned stage_errors() {
    unsigned v = 0;
    if (stage_err_.get()) {
      B200_CHECK(cudaMemcpyAsync(&v, stage_err_.get(), sizeof v, cudaMemcpyDeviceToHost, st_));
      B200_CHECK(cudaStreamSynchronize(st_));
    }
    return v;
  }

 private:
  using clock = std::chrono::steady_clock;
  unsigned* err() { return stage_err_.get(); }
  void finish_run(Status s, bool hat, const std::string& m, int ray);
  struct LoopState {  // the r²HPDHG loop's scalars (r2hpdhg.cpp:41-160)
    double omega = 1.0, pid_integral = 0.0, pid_last = 0.0, best_omega = 1.0, best_balance = 1e300;
    long long it = 0, inner = 0;
    double r0 = -1.0, r_last = std::numeric_limits<double>::infinity();
    std::string msg;
    bool fresh = false, finished = false;
    int variant = 0;
  };
  LoopState L_;
  EngineResult R_;
  const DeviceOutputs* out_ = nullptr;
  double elapsed() const { return std::chrono::duration<double>(clock::now() - t0_).count(); }

  template <class T> IterVecs<T>& vecs();
  template <class T> void capture_epoch();
  template <class T> void capture_check(int variant);
  template <class T> void launch_residual(bool with_restart_terms, const int* skip, SumPlan& plan,
                                          cudaStream_t sums_on = nullptr);
  template <class T> void launch_kkt_scaled(const T* xs, const T* ys, cudaStream_t on = nullptr);
  void launch_kkt_original(cudaStream_t on = nullptr);
  void make_side_streams();
  template <class T> void launch_ray(const T* dx, const T* dy, double* r, double* d, int drift);
  Kkt read_kkt(const double* h) const;
  Status ray_verdict(const double* h, int which, const Kkt& k, std::string& why) const;
  void setup();
  void build_plans();
  template <class T> void tune_slab();
  template <class T> void init_iterates();
  bool apply_warm_start();
  template <class T> void restart();
  void promote();
  double initial_primal_weight();
  void finish(EngineResult& R, Status st, bool use_hat, long long it, const std::string& msg,
              const DeviceOutputs& out, int ray_test);
  template <class T> void finish_t(EngineResult& R, Status st, bool use_hat, long long it, const std::string& msg,
                                   const DeviceOutputs& out, int ray_test);
  template <class T> void finish_p(EngineResult& R, Status st, const T* xs, const T* ys, long long it,
                                   const std::string& msg, const DeviceOutputs& out, int ray_test);
  // PDLP-style restarted averaged PDHG on the same kernels (pdlp.cpp:9-126)
  template <class T> void capture_pdlp_epoch(int phase);
  template <class T> void capture_pdlp_check(int phase, int variant);
  template <class T> void pdlp_restart(int cur, bool use_avg);
  template <class T> void pdlp_distances(int cur, bool use_avg, double& dx, double& dy);
  void promote_pdlp();
  void sync_results() {
    B200_CHECK(cudaMemcpyAsync(hres_.get(), res_.get(), kNumSlots * sizeof(double), cudaMemcpyDeviceToHost, st_));
    B200_CHECK(cudaStreamSynchronize(st_));
  }
  void clear_maxima() { B200_CHECK(cudaMemsetAsync(res_.get() + 32, 0, 16 * sizeof(double), st_)); }

  DeviceModel M_;
  const EngineOptions& o_;
  cudaStream_t st_;
  DevBuf<unsigned> stage_err_;  // this solve's bulk-copy timeouts (see count_stage_timeout)
  clock::time_point t0_;
  ScaledDevice sp_;
  IterVecs<double> vd_;
  IterVecs<float> vf_;
  bool mixed_now_ = false;
  double eta_ = 1.0;
  DevBuf<StepParams> params_;
  PinnedBuf<StepParams> hparams_;
  DevBuf<double> res_;
  PinnedBuf<double> hres_;
  DevBuf<double> rt_, kt_, rayt_, xo_, yo_, r1_, d1_, r2_, d2_, objt_;
  SumPlan plan_r0_, plan_res_, plan_pid_, plan_kkt_, plan_ray1_, plan_ray2_, plan_obj_, plan_chk_;
  cudaGraphExec_t g_epoch_[2] = {nullptr, nullptr};
  cudaGraphExec_t g_check_[2][3] = {{nullptr, nullptr, nullptr}, {nullptr, nullptr, nullptr}};
  cudaGraphExec_t g_pdlp_[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};         // [precision][phase]
  cudaGraphExec_t g_pdlp_chk_[2][2][3] = {};                                        // [precision][phase][variant]
  long long pdlp_kernels_[2][2] = {}, pdlp_chk_kernels_[2][2][3] = {};
  DevBuf<double> res2_;
  DevBuf<int2> slab_a_, slab_t_;
  int cap_a_ = kSlabTile, cap_t_ = kSlabTile;  // k_slab_fed tile capacities (largest slab, rounded up)
  int var_a_ = 0, var_t_ = 0;                  // k_slab_fed launch variants (dual, primal), tuned
  bool tuned_now_ = false;                     // this solve measured the variants itself
  PinnedBuf<double> hres2_;
  SumPlan plan_dist_;
  long long epoch_kernels_[2] = {0, 0}, check_kernels_[2][3] = {{0, 0, 0}, {0, 0, 0}};
  cudaEvent_t ev_[4] = {nullptr, nullptr, nullptr, nullptr};
  // The check graph's side branches: side_[0] runs the KKT statistics, side_[1] the residual's
  // and restart distances' sums, while the engine's stream runs the ray tests (fork_[0..3]: the
  // forks and joins that order them).
  cudaStream_t side_[2] = {nullptr, nullptr};
  cudaEvent_t fork_[4] = {nullptr, nullptr, nullptr, nullptr};
  long long kernels_ = 0;  // counted launches (graph kernel nodes per replay)
  long long capture_count_ = 0;
  bool capturing_ = false;
  double iter_ms_ = 0;
  long long iter_launches_ = 0;
  long long fast_it_ = -1, switch_it_ = -1;
  double primal_weight_ = std::numeric_limits<double>::quiet_NaN();
  // precision policy (engine.cpp:56-79)
  double pol_best_ = 1e300;
  int pol_since_best_ = 0;
};

template <> IterVecs<double>& Engine::vecs<double>() { return vd_; }
template <> IterVecs<float>& Engine::vecs<float>() { return vf_; }

#define B200_COUNT(k) (capturing_ ? capture_count_ += (k) : kernels_ += (k))

void Engine::setup() {
  // verbosity >= 2: the setup's phases on the host clock, the stream synchronised at each mark
  std::vector<std::pair<const char*, double>> marks;
  auto mark = [&](const char* name) {
    if (o_.verbosity < 2) return;
    B200_CHECK(cudaStreamSynchronize(st_));
    marks.emplace_back(name, elapsed());
  };
  mark("start");
  stage_err_.alloc(1);
  B200_CHECK(cudaMemsetAsync(stage_err_.get(), 0, sizeof(unsigned), st_));
  sp_.build(M_, o_.scaling, o_.exact, st_);
  mark("structure+scaling");
  if (o_.mixed) sp_.make_f32(st_);
  const double norm = sp_.lanczos(st_, err());
  mark("lanczos");
  eta_ = norm > 0 ? 0.998 / norm : 1.0;  // engine.cpp:203-204
  kernels_ += sp_.kernels;
  const int m = M_.m, n = M_.n;
  // each slab's nonzero range for the iteration kernels (Ã rows; Ãᵀ rows = the columns)
  slab_a_.alloc(static_cast<std::size_t>(std::max(1, slab_count(m))));
  slab_t_.alloc(static_cast<std::size_t>(std::max(1, slab_count(n))));
  if (m > 0) k_slab_table<<<grid_for(slab_count(m)), kBlock, 0, st_>>>(m, sp_.a_rp.get(), slab_a_.get());
  if (n > 0) k_slab_table<<<grid_for(slab_count(n)), kBlock, 0, st_>>>(n, M_.col_start, slab_t_.get());
  B200_LAUNCH_CHECK();
  kernels_ += 2;
  cap_a_ = fed_tile_capacity(slab_max_nnz(slab_a_.get(), slab_count(m), st_));
  cap_t_ = fed_tile_capacity(slab_max_nnz(slab_t_.get(), slab_count(n), st_));
  vd_.alloc(n, m);
  if (o_.mixed) vf_.alloc(n, m);
  params_.alloc(1);
  hparams_.alloc(1);
  res_.alloc(kNumSlots);
  hres_.alloc(kNumSlots);
  B200_CHECK(cudaMemsetAsync(res_.get(), 0, kNumSlots * sizeof(double), st_));
  const std::size_t mm = static_cast<std::size_t>(m), nn = static_cast<std::size_t>(n);
  rt_.alloc(2 * nn + 3 * mm);
  kt_.alloc(4 * (mm + nn));
  rayt_.alloc(2 * (mm + nn) + 2 * nn);
  xo_.alloc(nn), yo_.alloc(mm), r1_.alloc(mm), d1_.alloc(nn), r2_.alloc(mm), d2_.alloc(nn);
  objt_.alloc(mm + 2 * nn);
  build_plans();
  mark("tables+buffers+plans");
  if (o_.mixed) tune_slab<float>();
  else tune_slab<double>();
  mark("tuner");
  if (o_.verbosity >= 2) {
    std::string line = "setup phases:";
    char buf[96];
    for (std::size_t k = 1; k < marks.size(); ++k) {
      std::snprintf(buf, sizeof buf, " %s %.2f ms", marks[k].first, 1e3 * (marks[k].second - marks[k - 1].second));
      line += buf;
    }
    std::snprintf(buf, sizeof buf, " (Lanczos steps launched: %d)", sp_.lanczos_launched);
    std::fprintf(stderr, "%s%s\n", line.c_str(), buf);
  }
}

// The autotuner (tune.hpp): times the k_slab_fed variants on this matrix, for both iteration
// kernels, unless the shape class was measured before in this process. A variant is timed the
// way an epoch runs it: primal and dual kernels alternating on the stream with programmatic
// dependent launch (one warm-up pair, then kTunePairs timed pairs), so that what overlaps across
// kernel boundaries counts. The primal kernel's variant is picked first, with the dual kernel on
// the default; then the dual kernel's, with the primal kernel on its pick. The iterates are not
// initialised yet, so the timed launches (real operands, step parameters of an idle step) disturb
// nothing; every variant computes the same values.
template <class T>
void Engine::tune_slab() {
  const int forced = tune_forced();
  if (forced >= 0) {
    var_a_ = var_t_ = forced < kNumSlabVariants ? forced : 0;
    return;
  }
  if (!tune_enabled()) return;
  const int prec = std::is_same<T, float>::value ? 1 : 0;
  const int m = M_.m, n = M_.n;
  const TuneKey kt = tune_key(0, prec, n, M_.nnz), ka = tune_key(1, prec, m, M_.nnz);
  TuneCache& cache = TuneCache::instance();
  if (cache.get(kt, var_t_) && cache.get(ka, var_a_)) return;
  IterVecs<T>& v = vecs<T>();
  StepParams hp{};
  hp.tau = 0.0, hp.sigma = 0.0, hp.rho = o_.reflection, hp.inner0 = 0, hp.K = o_.check_every, hp.done = 0;
  hp.skip_r0 = 1;
  B200_CHECK(cudaMemcpyAsync(params_.get(), &hp, sizeof hp, cudaMemcpyHostToDevice, st_));
  const StepParams* P = params_.get();
  auto pair = [&](int vt, int va, bool pdl) {  // one iteration: Ãᵀy + primal update, Ãx̄ + dual update
    EpiPrimal<T> ep{v.x.get(), v.xh.get(), v.xb.get(), v.x0.get(), sp_.c<T>(), sp_.l<T>(), sp_.u<T>(), P, 1, 0, 0, 0};
    launch_slab_fed<T>(n, sp_.t_rp.get(), sp_.t_ri.get(), sp_.At_val<T>(), v.y.get(), ep, st_, slab_t_.get(), cap_t_,
                       err(), pdl, vt);
    EpiDual<T> ed{v.y.get(), v.yh.get(), v.yb.get(), v.y0.get(), sp_.rl<T>(), sp_.ru<T>(), P, 1, 0, 0, 0, 0};
    launch_slab_fed<T>(m, sp_.a_rp.get(), sp_.a_col.get(), sp_.A_val<T>(), v.xb.get(), ed, st_, slab_a_.get(), cap_a_,
                       err(), true, va);
    kernels_ += 2;
  };
  constexpr int kTunePairs = 6;
  auto measure = [&](auto&& variant_pair) {
    double ms[kNumSlabVariants];
    for (int k = 0; k < kNumSlabVariants; ++k) {
      const auto vv = variant_pair(k);
      pair(vv.first, vv.second, false);  // warm-up (first use of the instantiation, caches)
      B200_CHECK(cudaEventRecord(ev_[0], st_));
      for (int r = 0; r < kTunePairs; ++r) pair(vv.first, vv.second, r > 0);
      B200_CHECK(cudaEventRecord(ev_[1], st_));
      B200_CHECK(cudaEventSynchronize(ev_[1]));
      float t = 0;
      B200_CHECK(cudaEventElapsedTime(&t, ev_[0], ev_[1]));
      ms[k] = t / kTunePairs;
    }
    return pick_variant(ms, kNumSlabVariants);
  };
  var_t_ = measure([](int k) { return std::make_pair(k, 0); });
  const int vt = var_t_;
  var_a_ = measure([vt](int k) { return std::make_pair(vt, k); });
  cache.put(kt, var_t_);
  cache.put(ka, var_a_);
  tuned_now_ = true;
}

void Engine::build_plans() {
  const long long m = M_.m, n = M_.n;
  double* R = res_.get();
  double* px = rt_.get();
  double* dxn = px + n;
  double* py = dxn + n;
  double* cross = py + m;
  double* dyn = cross + m;
  // fixed-point residual dots: la::parallel_sum order (64 chunks)
  plan_r0_.add(px, 0, n, 0.0, SumOrder::kChunk64, R + kPx0);
  plan_r0_.add(py, 0, m, 0.0, SumOrder::kChunk64, R + kPy0);
  plan_r0_.add(cross, 0, m, 0.0, SumOrder::kChunk64, R + kCross0);
  plan_res_.add(px, 0, n, 0.0, SumOrder::kChunk64, R + kPx);
  plan_res_.add(py, 0, m, 0.0, SumOrder::kChunk64, R + kPy);
  plan_res_.add(cross, 0, m, 0.0, SumOrder::kChunk64, R + kCross);
  // the restart distances enter the PID primal weight ω (and so every later step): always the
  // reference's order, whatever the mode (positive terms: the exact chains are cheap on them)
  plan_pid_.add(dxn, 0, n, 0.0, SumOrder::kChunk64, R + kDxn2);
  plan_pid_.add(dyn, 0, m, 0.0, SumOrder::kChunk64, R + kDyn2);
  // KKT: host loops of kkt_general (rows, then columns for the continuing sums)
  double* K0 = kt_.get();
  const long long L = m + n;
  plan_kkt_.add(K0, 0, m, 0.0, SumOrder::kSeq, R + kRp2);
  plan_kkt_.add(K0 + L, 0, L, 0.0, SumOrder::kSeq, R + kD);
  plan_kkt_.add(K0 + 2 * L, 0, L, 0.0, SumOrder::kSeq, R + kRd2);
  plan_kkt_.add(K0 + 3 * L, m, L, 0.0, SumOrder::kSeq, R + kP);
  double* T0 = rayt_.get();
  plan_ray1_.add(T0, 0, L, 0.0, SumOrder::kSeq, R + kRayObj);
  plan_ray1_.add(T0 + L, 0, L, 0.0, SumOrder::kSeq, R + kRayMag);
  plan_ray1_.add(T0 + 2 * L, 0, n, 0.0, SumOrder::kSeq, R + kRayCd);
  plan_ray1_.add(T0 + 2 * L + n, 0, n, 0.0, SumOrder::kSeq, R + kRayCmag);
  plan_ray2_.add(T0, 0, L, 0.0, SumOrder::kSeq, R + kRayObj2);
  plan_ray2_.add(T0 + L, 0, L, 0.0, SumOrder::kSeq, R + kRayMag2);
  plan_ray2_.add(T0 + 2 * L, 0, n, 0.0, SumOrder::kSeq, R + kRayCd2);
  plan_ray2_.add(T0 + 2 * L + n, 0, n, 0.0, SumOrder::kSeq, R + kRayCmag2);
  // finish: objective = offset + Σ c x (Model::objective_value), check sums (solution_checker)
  double* O = objt_.get();
  plan_obj_.add(O, 0, n, M_.offset, SumOrder::kSeq, R + kObjective);
  plan_chk_.add(O + n, 0, L, 0.0, SumOrder::kSeq, R + kChkDual);
  plan_chk_.add(O, 0, n, 0.0, SumOrder::kSeq, R + kChkPrimal);
  plan_r0_.build(o_.exact, skip_r0_flag(params_.get()), st_);
  plan_res_.build(o_.exact, nullptr, st_);
  plan_pid_.build(true, nullptr, st_);
  plan_kkt_.build(o_.exact, nullptr, st_);
  plan_ray1_.build(o_.exact, nullptr, st_);
  plan_ray2_.build(o_.exact, nullptr, st_);
  plan_obj_.build(o_.exact, nullptr, st_);
  plan_chk_.build(o_.exact, nullptr, st_);
}

// The residual: dx = x̄ − x̂, adx = Ã dx, dy = ȳ − ŷ and the terms of the five dots.
// sums_on: the stream of the dots' sums (nullptr: the engine's; another stream must already wait for
// the engine's stream, and the caller joins it back).
template <class T>
void Engine::launch_residual(bool with_restart_terms, const int* skip, SumPlan& plan, cudaStream_t sums_on) {
  IterVecs<T>& v = vecs<T>();
  const int m = M_.m, n = M_.n;
  double* px = rt_.get();
  double* dxn = px + n;
  double* py = dxn + n;
  double* cross = py + m;
  double* dyn = cross + m;
  k_res_x<T><<<grid_for(n), kBlock, 0, st_>>>(n, v.xb.get(), v.xh.get(), v.x0.get(), v.dx.get(), px,
                                              with_restart_terms ? dxn : nullptr, skip);
  B200_LAUNCH_CHECK();
  EpiResY<T> e{v.yb.get(), v.yh.get(), v.y0.get(), v.dy.get(), v.adx.get(), py, cross,
               with_restart_terms ? dyn : nullptr, skip};
  launch_slab_tma<T>(m, sp_.a_rp.get(), sp_.a_col.get(), sp_.A_val<T>(), v.dx.get(), e, st_, nullptr, err());
  cudaStream_t ss = st_;
  if (sums_on) {
    B200_CHECK(cudaEventRecord(fork_[2], st_));
    B200_CHECK(cudaStreamWaitEvent(sums_on, fork_[2], 0));
    ss = sums_on;
  }
  plan.launch(ss);
  B200_COUNT(2 + plan.kernel_count());
  if (with_restart_terms) {
    plan_pid_.launch(ss);
    B200_COUNT(plan_pid_.kernel_count());
  }
}

void Engine::launch_kkt_original(cudaStream_t on) {
  const cudaStream_t s = on ? on : st_;
  const int m = M_.m, n = M_.n;
  const long long L = static_cast<long long>(m) + n;
  double* K0 = kt_.get();
  EpiKktRows er{{}, yo_.get(), M_.row_lower, M_.row_upper, K0, K0 + L, K0 + 2 * L, res_.get()};
  launch_slab_tma<double>(m, sp_.a_rp.get(), sp_.a_col.get(), sp_.a_v0.get(), xo_.get(), er, s, nullptr, err());
  EpiKktCols ec{{}, xo_.get(), M_.c, M_.col_lower, M_.col_upper, static_cast<double>(M_.sense), m,
                K0 + 3 * L, K0 + L, K0 + 2 * L, res_.get()};
  launch_slab<double>(n, M_.col_start, M_.row_index, M_.value, yo_.get(), ec, s, nullptr, err());
  plan_kkt_.launch(s);
  B200_COUNT(2 + plan_kkt_.kernel_count());
}

template <class T>
void Engine::launch_kkt_scaled(const T* xs, const T* ys, cudaStream_t on) {
  const cudaStream_t s = on ? on : st_;
  const int m = M_.m, n = M_.n;
  k_unscale_x<T><<<grid_for(n), kBlock, 0, s>>>(n, xs, sp_.col_scale.get(), sp_.bound_scale, M_.col_lower,
                                                M_.col_upper, xo_.get());
  k_unscale_y<T><<<grid_for(m), kBlock, 0, s>>>(m, ys, sp_.row_scale.get(), sp_.obj_scale, yo_.get());
  B200_LAUNCH_CHECK();
  B200_COUNT(2);
  launch_kkt_original(s);
}

// The check graph's two side streams and its fork / join events, made once per engine outside
// any capture.
void Engine::make_side_streams() {
  if (side_[0]) return;
  for (auto& q : side_) B200_CHECK(cudaStreamCreateWithFlags(&q, cudaStreamNonBlocking));
  for (auto& e : fork_) B200_CHECK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
}

template <class T>
void Engine::launch_ray(const T* dx, const T* dy, double* r, double* d, int drift) {
  const int m = M_.m, n = M_.n;
  const long long L = static_cast<long long>(m) + n;
  double* T0 = rayt_.get();
  const int s_rmax = drift ? kMaxRmax2 : kMaxRmax, s_dabs = drift ? kMaxDabs2 : kMaxDabs;
  const int s_dviol = drift ? kMaxDviol2 : kMaxDviol, s_pviol = drift ? kMaxPviol2 : kMaxPviol;
  k_ray_r<T><<<grid_for(m), kBlock, 0, st_>>>(m, dy, sp_.row_scale.get(), sp_.obj_scale, M_.row_lower,
                                              M_.row_upper, r, res_.get(), s_rmax);
  k_ray_d<T><<<grid_for(n), kBlock, 0, st_>>>(n, dx, sp_.col_scale.get(), sp_.bound_scale, M_.col_lower,
                                              M_.col_upper, d, res_.get(), s_dabs);
  k_ray_cols<<<grid_for(n), kBlock, 0, st_>>>(n, m, M_.col_start, M_.row_index, M_.value, r, d, M_.c,
                                              static_cast<double>(M_.sense), M_.col_lower, M_.col_upper, T0,
                                              T0 + L, T0 + 2 * L, T0 + 2 * L + n, res_.get(), s_dviol);
  B200_LAUNCH_CHECK();
  EpiRayRows er{{}, r, M_.row_lower, M_.row_upper, T0, T0 + L, res_.get(), s_pviol};
  launch_slab_tma<double>(m, sp_.a_rp.get(), sp_.a_col.get(), sp_.a_v0.get(), d, er, st_, nullptr, err());
  SumPlan& p = drift ? plan_ray2_ : plan_ray1_;
  p.launch(st_);
  B200_COUNT(4 + p.kernel_count());
}

template <class T>
EpiPrimal<T> Engine::primal_epi(int s) {
  IterVecs<T>& v = vecs<T>();
  return EpiPrimal<T>{v.x.get(), v.xh.get(), v.xb.get(), v.x0.get(), sp_.c<T>(), sp_.l<T>(), sp_.u<T>(), params_.get(),
                      s, 0, 0, 0};
}
template <class T>
EpiDual<T> Engine::dual_epi(int s) {
  IterVecs<T>& v = vecs<T>();
  return EpiDual<T>{v.y.get(), v.yh.get(), v.yb.get(), v.y0.get(), sp_.rl<T>(), sp_.ru<T>(), params_.get(), s, 0, 0, 0,
                    0};
}
template <class T>
Engine::SlabOperands Engine::primal_operands() {  // Ãᵀy: rows of Ãᵀ (the columns), gathers y
  return SlabOperands{M_.n, cap_t_, sp_.t_rp.get(), sp_.t_ri.get(), sp_.At_val<T>(), vecs<T>().y.get(), slab_t_.get(),
                      err()};
}
template <class T>
Engine::SlabOperands Engine::dual_operands() {  // Ãx̄: rows of Ã, gathers x̄
  return SlabOperands{M_.m, cap_a_, sp_.a_rp.get(), sp_.a_col.get(), sp_.A_val<T>(), vecs<T>().xb.get(),
                      slab_a_.get(), err()};
}

template <class T>
void Engine::capture_epoch() {
  const int idx = std::is_same<T, float>::value ? 1 : 0;
  if (g_epoch_[idx]) return;
  IterVecs<T>& v = vecs<T>();
  const int m = M_.m, n = M_.n, K = o_.check_every;
  const StepParams* P = params_.get();
  const int* r0_skip = skip_r0_flag(P);
  cudaGraph_t g;
  slab_prepare<T, EpiPrimal<T>, B200_STAGE_TMA != 0>();
  slab_prepare<T, EpiDual<T>, B200_STAGE_TMA != 0>();
  slab_prepare<T, EpiResY<T>, B200_STAGE_TMA != 0>();
  capturing_ = true;
  capture_count_ = 0;
  auto capture_scope = std::make_unique<CaptureScope>();  // no device-wide syncs elsewhere meanwhile
  B200_CHECK(cudaStreamBeginCapture(st_, cudaStreamCaptureModeThreadLocal));
  // Programmatic dependent launch for every iteration kernel whose predecessor in the stream is
  // another iteration kernel (not the first kernel of the epoch, nor the one after the residual).
  auto step = [&](int s) {
    EpiPrimal<T> ep{v.x.get(), v.xh.get(), v.xb.get(), v.x0.get(), sp_.c<T>(), sp_.l<T>(), sp_.u<T>(), P, s, 0, 0, 0};
    launch_slab_fed<T>(n, sp_.t_rp.get(), sp_.t_ri.get(), sp_.At_val<T>(), v.y.get(), ep, st_, slab_t_.get(), cap_t_,
                       err(), s >= 2, var_t_);
    EpiDual<T> ed{v.y.get(), v.yh.get(), v.yb.get(), v.y0.get(), sp_.rl<T>(), sp_.ru<T>(), P, s, 0, 0, 0, 0};
    launch_slab_fed<T>(m, sp_.a_rp.get(), sp_.a_col.get(), sp_.A_val<T>(), v.xb.get(), ed, st_, slab_a_.get(), cap_a_,
                       err(), true, var_a_);
    capture_count_ += 2;
  };
  B200_CHECK(cudaEventRecordWithFlags(ev_[0], st_, cudaEventRecordExternal));
  step(0);
  B200_CHECK(cudaEventRecordWithFlags(ev_[1], st_, cudaEventRecordExternal));
  launch_residual<T>(false, r0_skip, plan_r0_);  // r⁰ after the first step of a Halpern cycle
  B200_CHECK(cudaEventRecordWithFlags(ev_[2], st_, cudaEventRecordExternal));
  for (int s = 1; s < K; ++s) step(s);
  B200_CHECK(cudaEventRecordWithFlags(ev_[3], st_, cudaEventRecordExternal));
  const cudaError_t e = cudaStreamEndCapture(st_, &g);
  capture_scope.reset();
  capturing_ = false;
  B200_CHECK(e);
  B200_CHECK(cudaGraphInstantiate(&g_epoch_[idx], g, 0));
  cudaGraphDestroy(g);
  epoch_kernels_[idx] = capture_count_;
}

template <class T>
void Engine::capture_check(int variant) {
  const int idx = std::is_same<T, float>::value ? 1 : 0;
  if (g_check_[idx][variant]) return;
  IterVecs<T>& v = vecs<T>();
  cudaGraph_t g;
  slab_prepare<T, EpiResY<T>, B200_STAGE_TMA != 0>();
  slab_prepare<double, EpiKktRows, B200_STAGE_TMA != 0>();
  slab_prepare<double, EpiKktCols, false>();
  slab_prepare<double, EpiRayRows, B200_STAGE_TMA != 0>();
  make_side_streams();
  capturing_ = true;
  capture_count_ = 0;
  auto capture_scope = std::make_unique<CaptureScope>();  // no device-wide syncs elsewhere meanwhile
  B200_CHECK(cudaStreamBeginCapture(st_, cudaStreamCaptureModeThreadLocal));
  clear_maxima();
  // Three branches that share no buffer and write disjoint result slots: the KKT statistics of
  // (x̂, ŷ) on side_[0]; the residual's kernels on the engine's stream, then their sums and the
  // restart distances on side_[1] while the ray tests (which read dx, dy) run on the engine's
  // stream. Each branch's order is the serial one, so every value is the same; the short sum
  // kernels of one branch overlap the matrix products of another.
  B200_CHECK(cudaEventRecord(fork_[0], st_));
  B200_CHECK(cudaStreamWaitEvent(side_[0], fork_[0], 0));
  launch_kkt_scaled<T>(v.xh.get(), v.yh.get(), side_[0]);
  B200_CHECK(cudaEventRecord(fork_[1], side_[0]));
  launch_residual<T>(true, nullptr, plan_res_, side_[1]);
  B200_CHECK(cudaEventRecord(fork_[3], side_[1]));
  if (variant >= 1) launch_ray<T>(v.dx.get(), v.dy.get(), r1_.get(), d1_.get(), 0);
  if (variant == 2) {
    k_diff<T><<<grid_for(M_.n), kBlock, 0, st_>>>(M_.n, v.xh.get(), v.x0.get(), v.ddx.get());
    k_diff<T><<<grid_for(M_.m), kBlock, 0, st_>>>(M_.m, v.yh.get(), v.y0.get(), v.ddy.get());
    B200_LAUNCH_CHECK();
    capture_count_ += 2;
    launch_ray<T>(v.ddx.get(), v.ddy.get(), r2_.get(), d2_.get(), 1);
  }
  B200_CHECK(cudaStreamWaitEvent(st_, fork_[1], 0));  // join the KKT branch
  B200_CHECK(cudaStreamWaitEvent(st_, fork_[3], 0));  // join the sums branch
  B200_CHECK(cudaMemcpyAsync(hres_.get(), res_.get(), kNumSlots * sizeof(double), cudaMemcpyDeviceToHost, st_));
  const cudaError_t e = cudaStreamEndCapture(st_, &g);
  capture_scope.reset();
  capturing_ = false;
  B200_CHECK(e);
  B200_CHECK(cudaGraphInstantiate(&g_check_[idx][variant], g, 0));
  cudaGraphDestroy(g);
  check_kernels_[idx][variant] = capture_count_;
}

Kkt Engine::read_kkt(const double* h) const {
  Kkt k;
  k.primal_residual = std::sqrt(h[kRp2]);
  k.dual_residual = std::sqrt(h[kRd2]);
  k.primal_obj = h[kP];
  k.dual_obj = h[kD];
  k.b_norm = sp_.b_norm;
  k.c_norm = sp_.c_norm;
  k.primal_max_rel = slot_max(h, kMaxPmax);
  k.dual_max_rel = slot_max(h, kMaxDmax) / (1.0 + sp_.c_inf);
  // EngineContext::adjust (engine.h:121-126)
  if (o_.kkt_b_norm >= 0) k.b_norm = o_.kkt_b_norm;
  if (o_.kkt_c_norm >= 0) k.c_norm = o_.kkt_c_norm;
  k.obj_shift = o_.kkt_obj_shift;
  return k;
}

template <class T>
void Engine::init_iterates() {
  IterVecs<T>& v = vecs<T>();
  const int m = M_.m, n = M_.n;
  k_init_x<T><<<grid_for(n), kBlock, 0, st_>>>(n, sp_.c<T>(), sp_.l<T>(), sp_.u<T>(), v.x.get());
  k_fill<T><<<grid_for(m), kBlock, 0, st_>>>(m, v.y.get(), static_cast<T>(0.0));
  B200_LAUNCH_CHECK();
  kernels_ += 2;
}

template <class T>
void Engine::restart() {
  IterVecs<T>& v = vecs<T>();
  const int m = M_.m, n = M_.n;
  k_restart<T><<<grid_for(std::max(m, n)), kBlock, 0, st_>>>(n, m, v.xh.get(), v.x.get(), v.x0.get(), v.yh.get(),
                                                               v.y.get(), v.y0.get());
  B200_LAUNCH_CHECK();
  ++kernels_;
}

// set_precision(Fp64): every iterate converted float -> double (cuda_backend.cu:474-483)
void Engine::promote() {
  const long long m = M_.m, n = M_.n;
  DevBuf<float>* fs[] = {&vf_.x, &vf_.x0, &vf_.xh, &vf_.xb, &vf_.y, &vf_.y0, &vf_.yh, &vf_.yb};
  DevBuf<double>* ds[] = {&vd_.x, &vd_.x0, &vd_.xh, &vd_.xb, &vd_.y, &vd_.y0, &vd_.yh, &vd_.yb};
  for (int q = 0; q < 8; ++q) {
    const long long len = q < 4 ? n : m;
    k_convert<double, float><<<grid_for(len), kBlock, 0, st_>>>(len, fs[q]->get(), ds[q]->get());
  }
  B200_LAUNCH_CHECK();
  kernels_ += 8;
  mixed_now_ = false;
}

double Engine::initial_primal_weight() {  // engine.cpp:207-218
  if (o_.warm_primal_weight > 0) return o_.warm_primal_weight;
  if (o_.scaling.bound_objective_rescaling) return 1.0;
  const int m = M_.m, n = M_.n;
  DevBuf<double> tm(m), tn(n), s(2);
  k_b2_terms<<<grid_for(m), kBlock, 0, st_>>>(m, sp_.srl.get(), sp_.sru.get(), tm.get());
  k_sq_terms<<<grid_for(n), kBlock, 0, st_>>>(n, sp_.sc.get(), tn.get());
  B200_LAUNCH_CHECK();
  SumPlan p;
  p.add(tm.get(), 0, m, 0.0, SumOrder::kSeq, s.get());
  p.add(tn.get(), 0, n, 0.0, SumOrder::kSeq, s.get() + 1);
  p.build(true, nullptr, st_);  // ω0 enters every step: always the reference's order
  p.launch(st_);
  double h[2];
  B200_CHECK(cudaMemcpyAsync(h, s.get(), sizeof h, cudaMemcpyDeviceToHost, st_));
  B200_CHECK(cudaStreamSynchronize(st_));
  return (std::sqrt(h[1]) + 1.0) / (std::sqrt(h[0]) + 1.0);
}

// EngineContext::apply_warm_start (engine.cpp:237-266). Returns true if applied.
bool Engine::apply_warm_start() {
  if (o_.warm_x.empty() && o_.warm_y.empty()) return false;
  const int m = M_.m, n = M_.n;
  std::vector<double> lo(n), up(n), rl(m), ru(m), cs(n), rs(m);
  B200_CHECK(cudaMemcpyAsync(lo.data(), M_.col_lower, n * sizeof(double), cudaMemcpyDeviceToHost, st_));
  B200_CHECK(cudaMemcpyAsync(up.data(), M_.col_upper, n * sizeof(double), cudaMemcpyDeviceToHost, st_));
  B200_CHECK(cudaMemcpyAsync(rl.data(), M_.row_lower, m * sizeof(double), cudaMemcpyDeviceToHost, st_));
  B200_CHECK(cudaMemcpyAsync(ru.data(), M_.row_upper, m * sizeof(double), cudaMemcpyDeviceToHost, st_));
  B200_CHECK(cudaMemcpyAsync(cs.data(), sp_.col_scale.get(), n * sizeof(double), cudaMemcpyDeviceToHost, st_));
  B200_CHECK(cudaMemcpyAsync(rs.data(), sp_.row_scale.get(), m * sizeof(double), cudaMemcpyDeviceToHost, st_));
  std::vector<double> xo(n), yo(m, 0.0);
  if (!o_.warm_x.empty()) {
    B200_CHECK(cudaStreamSynchronize(st_));
    for (int j = 0; j < n; ++j) xo[j] = std_min(std_max(o_.warm_x[j], lo[j]), up[j]);
  } else {  // the engine's cold x, unscaled
    std::vector<double> xs(n);
    if (mixed_now_) {
      std::vector<float> xf(n);
      B200_CHECK(cudaMemcpyAsync(xf.data(), vf_.x.get(), n * sizeof(float), cudaMemcpyDeviceToHost, st_));
      B200_CHECK(cudaStreamSynchronize(st_));
      for (int j = 0; j < n; ++j) xs[j] = xf[j];
    } else {
      B200_CHECK(cudaMemcpyAsync(xs.data(), vd_.x.get(), n * sizeof(double), cudaMemcpyDeviceToHost, st_));
      B200_CHECK(cudaStreamSynchronize(st_));
    }
    for (int j = 0; j < n; ++j) xo[j] = std_min(std_max(cs[j] * xs[j] / sp_.bound_scale, lo[j]), up[j]);
  }
  if (!o_.warm_y.empty()) {
    for (int i = 0; i < m; ++i) {
      double v = static_cast<double>(M_.sense) * o_.warm_y[i];
      if (!std::isfinite(rl[i])) v = std_min(v, 0.0);
      if (!std::isfinite(ru[i])) v = std_max(v, 0.0);
      yo[i] = v;
    }
  }
  // decide the working precision before uploading (PrecisionPolicy::on_warm_start)
  B200_CHECK(cudaMemcpyAsync(xo_.get(), xo.data(), n * sizeof(double), cudaMemcpyHostToDevice, st_));
  B200_CHECK(cudaMemcpyAsync(yo_.get(), yo.data(), m * sizeof(double), cudaMemcpyHostToDevice, st_));
  clear_maxima();
  launch_kkt_original();
  sync_results();
  const double wr = read_kkt(hres_.get()).rel_kkt();
  if (o_.mixed && mixed_now_ && wr <= kMixedPrecisionSwitch && o_.tolerance < kMixedPrecisionSwitch) {
    mixed_now_ = false;
    switch_it_ = 0;
  }
  std::vector<double> xs(n), ys(m);
  for (int j = 0; j < n; ++j) xs[j] = sp_.bound_scale * xo[j] / cs[j];
  for (int i = 0; i < m; ++i) ys[i] = sp_.obj_scale * yo[i] / rs[i];
  if (mixed_now_) {
    std::vector<float> xf(xs.begin(), xs.end()), yf(ys.begin(), ys.end());
    B200_CHECK(cudaMemcpyAsync(vf_.x.get(), xf.data(), n * sizeof(float), cudaMemcpyHostToDevice, st_));
    B200_CHECK(cudaMemcpyAsync(vf_.y.get(), yf.data(), m * sizeof(float), cudaMemcpyHostToDevice, st_));
    B200_CHECK(cudaStreamSynchronize(st_));
  } else {
    B200_CHECK(cudaMemcpyAsync(vd_.x.get(), xs.data(), n * sizeof(double), cudaMemcpyHostToDevice, st_));
    B200_CHECK(cudaMemcpyAsync(vd_.y.get(), ys.data(), m * sizeof(double), cudaMemcpyHostToDevice, st_));
    B200_CHECK(cudaStreamSynchronize(st_));
  }
  return true;
}

void Engine::finish(EngineResult& R, Status st, bool use_hat, long long it, const std::string& msg,
                    const DeviceOutputs& out, int ray_test) {
  if (mixed_now_) finish_t<float>(R, st, use_hat, it, msg, out, ray_test);
  else finish_t<double>(R, st, use_hat, it, msg, out, ray_test);
}

// EngineContext::finish (engine.cpp:268-307) plus the device-side in-process check.
template <class T>
void Engine::finish_t(EngineResult& R, Status status, bool use_hat, long long it, const std::string& msg,
                      const DeviceOutputs& out, int ray_test) {
  IterVecs<T>& v = vecs<T>();
  finish_p<T>(R, status, use_hat ? v.xh.get() : v.x.get(), use_hat ? v.yh.get() : v.y.get(), it, msg, out, ray_test);
}

template <class T>
void Engine::finish_p(EngineResult& R, Status status, const T* xs, const T* ys, long long it, const std::string& msg,
                      const DeviceOutputs& out, int ray_test) {
  const auto tf = clock::now();
  const int m = M_.m, n = M_.n;
  clear_maxima();
  launch_kkt_scaled<T>(xs, ys);
  // objective = offset + Σ c_j x_j (Model::objective_value)
  k_obj_terms<<<grid_for(n), kBlock, 0, st_>>>(n, M_.c, xo_.get(), objt_.get());
  B200_LAUNCH_CHECK();
  plan_obj_.launch(st_);
  // in-process check (solution_checker.cpp:61-133) on xo and y_min = yo
  double c_scale = std_max(1.0, sp_.c_inf);
  EpiCheckRows cr{{}, yo_.get(), M_.row_lower, M_.row_upper, c_scale, objt_.get() + n, res_.get()};
  launch_slab_tma<double>(m, sp_.a_rp.get(), sp_.a_col.get(), sp_.a_v0.get(), xo_.get(), cr, st_, nullptr, err());
  // t_primal lands in objt_[0, n): the objective terms were consumed by plan_obj_ above
  EpiCheckCols cc{{}, xo_.get(), M_.c, M_.col_lower, M_.col_upper, static_cast<double>(M_.sense), c_scale, m,
                  objt_.get() + n, objt_.get(), res_.get()};
  launch_slab<double>(n, M_.col_start, M_.row_index, M_.value, yo_.get(), cc, st_, nullptr, err());
  plan_chk_.launch(st_);
  kernels_ += 3 + plan_obj_.kernel_count() + plan_chk_.kernel_count();
  // outputs
  if (out.x) B200_CHECK(cudaMemcpyAsync(out.x, xo_.get(), n * sizeof(double), cudaMemcpyDeviceToDevice, st_));
  if (out.y || out.z) {
    DevBuf<double> ytmp;
    double* y = out.y;
    if (!y) {
      ytmp.alloc(m);
      y = ytmp.get();
    }
    k_dual_out<<<grid_for(m), kBlock, 0, st_>>>(m, static_cast<double>(M_.sense), yo_.get(), y);
    if (out.z) k_reduced_costs<<<grid_for(n), kBlock, 0, st_>>>(n, M_.col_start, M_.row_index, M_.value, M_.c, y, out.z);
    B200_LAUNCH_CHECK();
    kernels_ += 2;
    if (ytmp.get()) B200_CHECK(cudaStreamSynchronize(st_));
  }
  if (status == Status::Infeasible && out.dual_ray)
    B200_CHECK(cudaMemcpyAsync(out.dual_ray, ray_test == 2 ? r2_.get() : r1_.get(), m * sizeof(double),
                               cudaMemcpyDeviceToDevice, st_));
  if (status == Status::Unbounded && out.primal_ray)
    B200_CHECK(cudaMemcpyAsync(out.primal_ray, ray_test == 2 ? d2_.get() : d1_.get(), n * sizeof(double),
                               cudaMemcpyDeviceToDevice, st_));
  sync_results();
  const double* h = hres_.get();
  const Kkt k = read_kkt(h);
  if (!k.finite()) status = Status::NumericalError;
  if (status == Status::Optimal && !k.converged(o_.tolerance)) status = Status::NumericalError;  // never over-claim
  const double sense = M_.sense;
  R.status = status;
  R.iterations = it;
  R.message = msg;
  R.objective = h[kObjective];
  R.dual_objective = sense * k.dual_obj + M_.offset;
  R.primal_residual = k.rel_primal();
  R.dual_residual = k.rel_dual();
  R.gap = k.rel_gap();
  R.iterations_to_fast = fast_it_;
  R.switch_iteration = switch_it_;
  R.primal_weight = primal_weight_;
  R.eta = eta_;
  R.have_dual_ray = status == Status::Infeasible;
  R.have_primal_ray = status == Status::Unbounded;
  if (status == Status::Infeasible || status == Status::Unbounded)
    R.objective = R.dual_objective = std::numeric_limits<double>::quiet_NaN();
  // check report (solution_checker.cpp:111-131)
  const double pobj = sense * h[kChkPrimal] + M_.offset, dobj = sense * h[kChkDual] + M_.offset;
  R.check_primal = slot_max(h, kMaxChkPrimal);
  R.check_dual = slot_max(h, kMaxChkDual);
  R.check_gap = std::fabs(pobj - dobj) / (1.0 + std::fabs(pobj) + std::fabs(dobj));
  const bool finite_pt = std::isfinite(pobj) && std::isfinite(dobj) && std::isfinite(R.check_primal);
  R.check = finite_pt && R.check_primal <= kVerifyPrimal && R.check_dual <= kVerifyDual && R.check_gap <= kVerifyGap;
  R.finish_seconds = std::chrono::duration<double>(clock::now() - tf).count();
}

// EngineContext::ray_test on the device sums of one candidate direction (engine.cpp:82-155):
// which = 1 the last step's Δ, 2 the drift since the restart anchor; k = the current KKT.
Status Engine::ray_verdict(const double* h, int which, const Kkt& k, std::string& why) const {
  const int s_rmax = which == 2 ? kMaxRmax2 : kMaxRmax, s_dabs = which == 2 ? kMaxDabs2 : kMaxDabs;
  const int s_dviol = which == 2 ? kMaxDviol2 : kMaxDviol, s_pviol = which == 2 ? kMaxPviol2 : kMaxPviol;
  const double obj = h[which == 2 ? kRayObj2 : kRayObj], mag = h[which == 2 ? kRayMag2 : kRayMag];
  const double cd = h[which == 2 ? kRayCd2 : kRayCd], cmag = h[which == 2 ? kRayCmag2 : kRayCmag];
  const double rmax = slot_max(h, s_rmax), dmax = slot_max(h, s_dabs);
  bool pinf = false, dinf = false;
  double dro = 0, drv = 0, pro = 0, prv = 0;
  if (rmax > 0) {
    const double viol = slot_max(h, s_dviol), scale = std_max(rmax, viol);
    dro = obj / scale, drv = viol / scale;
    pinf = dro > 0 && obj > kFirstOrderInfeasible * mag && drv <= kFirstOrderInfeasible * dro;
  }
  if (dmax > 0) {
    const double viol = slot_max(h, s_pviol), scale = std_max(dmax, viol);
    pro = cd / scale, prv = viol / scale;
    dinf = pro < 0 && -cd > kFirstOrderInfeasible * cmag && prv <= kFirstOrderInfeasible * -pro;
  }
  char buf[200];
  if (pinf) {
    std::snprintf(buf, sizeof buf, "primal infeasible: dual ray certificate (objective %f, violation %f)", dro, drv);
    why = buf;
    return Status::Infeasible;
  }
  if (dinf) {
    const bool feasible = k.rel_primal() <= kVerifyPrimal && k.primal_max_rel <= kVerifyPrimal;
    std::snprintf(buf, sizeof buf, "unbounded: primal ray certificate (c'd %f, violation %f)%s", pro, prv,
                  feasible ? " at a primal-feasible iterate" : "; iterate not primal-feasible yet");
    why = buf;
    return Status::Unbounded;
  }
  return Status::NotSolved;
}

// The r²HPDHG solve as steps. run() chains them on this engine's stream; the group scheduler
// (group.cu) interleaves the steps of several engines on one stream, launching their iteration
// kernels together. Either way each engine takes the same values and decisions.

void Engine::finish_run(Status s, bool hat, const std::string& m, int ray) {
  R_.loop_seconds = elapsed() - R_.setup_seconds;
  finish(R_, s, hat, L_.it, m, *out_, ray);
  R_.kernel_launches = kernels_;
  R_.iter_kernel_ms = iter_ms_;
  R_.iter_kernel_launches = iter_launches_;
  R_.slab_variant_primal = var_t_, R_.slab_variant_dual = var_a_, R_.tuned = tuned_now_ ? 1 : 0;
  R_.seconds = elapsed();
  L_.finished = true;
}

bool Engine::start(const DeviceOutputs& out) {
  t0_ = clock::now();
  out_ = &out;
  R_ = EngineResult{};
  L_ = LoopState{};
  setup();
  mixed_now_ = o_.mixed;
  L_.omega = initial_primal_weight();
  if (mixed_now_) init_iterates<float>();
  else init_iterates<double>();
  const bool warm = apply_warm_start();
  primal_weight_ = L_.omega;
  L_.best_omega = L_.omega;
  L_.msg = warm ? "warm start" : "";
  R_.setup_seconds = elapsed();
  if (warm) {  // the warm point may already be good enough (r2hpdhg.cpp:37-40)
    clear_maxima();
    if (mixed_now_) launch_kkt_scaled<float>(vf_.x.get(), vf_.y.get());
    else launch_kkt_scaled<double>(vd_.x.get(), vd_.y.get());
    sync_results();
    const Kkt kw = read_kkt(hres_.get());
    if (fast_it_ < 0 && kw.rel_kkt() <= kFirstOrderFast) fast_it_ = 0;
    if (kw.finite() && kw.converged(o_.tolerance)) {
      finish_run(Status::Optimal, false, "warm start already optimal", 0);
      return true;
    }
  }
  const long long m = M_.m, n = M_.n;
  if (mixed_now_) {
    B200_CHECK(cudaMemcpyAsync(vf_.x0.get(), vf_.x.get(), n * sizeof(float), cudaMemcpyDeviceToDevice, st_));
    B200_CHECK(cudaMemcpyAsync(vf_.xh.get(), vf_.x.get(), n * sizeof(float), cudaMemcpyDeviceToDevice, st_));
    B200_CHECK(cudaMemcpyAsync(vf_.y0.get(), vf_.y.get(), m * sizeof(float), cudaMemcpyDeviceToDevice, st_));
    B200_CHECK(cudaMemcpyAsync(vf_.yh.get(), vf_.y.get(), m * sizeof(float), cudaMemcpyDeviceToDevice, st_));
  } else {
    B200_CHECK(cudaMemcpyAsync(vd_.x0.get(), vd_.x.get(), n * sizeof(double), cudaMemcpyDeviceToDevice, st_));
    B200_CHECK(cudaMemcpyAsync(vd_.xh.get(), vd_.x.get(), n * sizeof(double), cudaMemcpyDeviceToDevice, st_));
    B200_CHECK(cudaMemcpyAsync(vd_.y0.get(), vd_.y.get(), m * sizeof(double), cudaMemcpyDeviceToDevice, st_));
    B200_CHECK(cudaMemcpyAsync(vd_.yh.get(), vd_.y.get(), m * sizeof(double), cudaMemcpyDeviceToDevice, st_));
  }
  return false;
}

// The step scalars of the next epoch: τ = η/ω, σ = ηω (r2hpdhg.cpp:67), the Halpern counter.
void Engine::begin_epoch() {
  StepParams& hp = *hparams_.get();
  hp.tau = eta_ / L_.omega;
  hp.sigma = eta_ * L_.omega;
  hp.rho = o_.reflection;
  hp.inner0 = L_.inner;
  hp.K = o_.check_every;
  hp.done = 0;
  hp.skip_r0 = L_.inner != 0 ? 1 : 0;
  B200_CHECK(cudaMemcpyAsync(params_.get(), &hp, sizeof(StepParams), cudaMemcpyHostToDevice, st_));
  L_.fresh = L_.inner == 0;
}

void Engine::launch_epoch() {
  const int pidx = mixed_now_ ? 1 : 0;
  if (mixed_now_) capture_epoch<float>();
  else capture_epoch<double>();
  B200_CHECK(cudaGraphLaunch(g_epoch_[pidx], st_));
  kernels_ += epoch_kernels_[pidx];
}

// The r⁰ residual after the first step of an epoch that starts a Halpern cycle (the section the
// epoch graph holds), for epochs whose steps the group scheduler launches.
void Engine::launch_r0(cudaStream_t on) {
  if (!L_.fresh) return;
  const cudaStream_t own = st_;
  st_ = on;  // launched on the group's stream, between the group's step 0 and step 1
  if (mixed_now_) launch_residual<float>(false, nullptr, plan_r0_);
  else launch_residual<double>(false, nullptr, plan_r0_);
  st_ = own;
}

void Engine::launch_check() {
  const int K = o_.check_every;
  L_.it += K;
  L_.inner += K;
  L_.variant = L_.it >= 4LL * K ? (((L_.it / K) % 4 == 0) ? 2 : 1) : 0;
  const int pidx = mixed_now_ ? 1 : 0;
  if (mixed_now_) capture_check<float>(L_.variant);
  else capture_check<double>(L_.variant);
  B200_CHECK(cudaGraphLaunch(g_check_[pidx][L_.variant], st_));
  kernels_ += check_kernels_[pidx][L_.variant];
}

// The reference's decisions on the check's results (r2hpdhg.cpp:93-160, engine.cpp:56-192),
// once the stream has synchronised. Returns true when the solve has ended (result in R_).
bool Engine::end_epoch() {
  LoopState& S = L_;
  ++R_.checks;
  const double* h = hres_.get();
  const double omega = S.omega;
  if (S.fresh) S.r0 = std::sqrt(std_max(omega * h[kPx0] + h[kPy0] / omega + 2.0 * eta_ * h[kCross0], 0.0));
  const double r = std::sqrt(std_max(omega * h[kPx] + h[kPy] / omega + 2.0 * eta_ * h[kCross], 0.0));
  const Kkt k = read_kkt(h);
  if (o_.verbosity >= 2)
    std::fprintf(stderr, "r2hpdhg-b200 it %8lld  t %7.2fs  pobj %+.10e  dobj %+.10e  rp %.2e  rd %.2e  gap %.2e  %s\n",
                 S.it, elapsed(), k.primal_obj, k.dual_obj, k.rel_primal(), k.rel_dual(), k.rel_gap(),
                 mixed_now_ ? "fp32" : "fp64");
  auto done = [&](Status st, bool hat, const std::string& m, int ray) {
    finish_run(st, hat, m, ray);
    return true;
  };
  if (!k.finite() || !std::isfinite(r)) return done(Status::NumericalError, true, "non-finite iterate", 0);
  if (fast_it_ < 0 && k.rel_kkt() <= kFirstOrderFast) fast_it_ = S.it;
  if (k.converged(o_.tolerance)) return done(Status::Optimal, true, S.msg, 0);
  if (S.it >= o_.iteration_limit) return done(Status::IterationLimit, true, S.msg, 0);
  if (elapsed() > o_.time_limit) return done(Status::TimeLimit, true, S.msg, 0);
  if (S.variant >= 1) {  // EngineContext::check_infeasibility + ray_test (engine.cpp:82-184)
    auto test = [&](int which, std::string& why) { return ray_verdict(h, which, k, why); };
    std::string why;
    int which = 1;
    Status st = test(1, why);
    if (st == Status::NotSolved && S.variant == 2) {
      which = 2;
      st = test(2, why);
      if (st != Status::NotSolved) why += " (drift since the restart anchor)";
    }
    if (st != Status::NotSolved) return done(st, true, why, which);
  }
  // PrecisionPolicy::on_check (engine.cpp:61-79)
  bool promoted = false;
  if (o_.mixed && mixed_now_) {
    const double rk = k.rel_kkt();
    if (rk < 0.9 * pol_best_) pol_best_ = rk, pol_since_best_ = 0;
    else ++pol_since_best_;
    const bool reached = rk <= kMixedPrecisionSwitch && o_.tolerance < kMixedPrecisionSwitch;
    if (reached || pol_since_best_ >= o_.mixed_stall_checks) {
      promote();
      switch_it_ = S.it;
      promoted = true;
      S.msg += std::string(S.msg.empty() ? "" : "; ") + "fp32 -> fp64 at iteration " + std::to_string(S.it);
    }
  }
  const bool ratios_ok = S.r0 > 0 && std::isfinite(S.r0) && r > 0;
  const bool restart_now = promoted ||
                           (ratios_ok && (r <= o_.restart_sufficient * S.r0 ||
                                          (r <= o_.restart_necessary * S.r0 && r > S.r_last))) ||
                           static_cast<double>(S.inner) >= o_.restart_artificial * static_cast<double>(S.it);
  S.r_last = r;
  if (!restart_now) return false;
  // PID primal weight (r2hpdhg.cpp:126-148)
  const double dxn = std::sqrt(h[kDxn2]), dyn = std::sqrt(h[kDyn2]);
  const bool both_pos = k.rel_dual() > 0 && k.rel_primal() > 0;
  const double ratio = both_pos ? k.rel_dual() / k.rel_primal() : 1.0;
  if (dxn > 1e-16 && dyn > 1e-16 && dxn < 1e12 && dyn < 1e12 && ratio > 1e-8 && ratio < 1e8) {
    const double e = std::log(dyn) - std::log(dxn) - std::log(S.omega);
    S.pid_integral = o_.pid_integral_decay * S.pid_integral + e;
    const double step = o_.pid_kp * e + o_.pid_ki * S.pid_integral + o_.pid_kd * (e - S.pid_last);
    S.omega *= std::exp(std::clamp(step, -o_.pid_max_log_step, o_.pid_max_log_step));
    S.pid_last = e;
  } else {
    S.omega = S.best_omega;
    S.pid_integral = S.pid_last = 0.0;
  }
  const double balance = std::fabs(std::log10(ratio));
  if (both_pos && balance < S.best_balance) {
    S.best_balance = balance;
    S.best_omega = S.omega;
  }
  primal_weight_ = S.omega;
  ++R_.restarts;
  if (o_.verbosity >= 2)
    std::fprintf(stderr, "  restart at %lld: r/r0 %.3f  omega %.4e  dx %.3e dy %.3e\n", S.it, r / S.r0, S.omega, dxn,
                 dyn);
  if (mixed_now_) restart<float>();
  else restart<double>();
  S.inner = 0;
  S.r_last = std::numeric_limits<double>::infinity();
  return false;
}

EngineResult Engine::run(const DeviceOutputs& out) {
  if (start(out)) return R_;
  const int K = o_.check_every;
  for (;;) {
    begin_epoch();
    launch_epoch();
    launch_check();
    B200_CHECK(cudaStreamSynchronize(st_));
    {  // the iteration kernels' time, from the events inside the epoch graph
      float a = 0, b = 0;
      B200_CHECK(cudaEventElapsedTime(&a, ev_[0], ev_[1]));
      B200_CHECK(cudaEventElapsedTime(&b, ev_[2], ev_[3]));
      iter_ms_ += a + b;
      iter_launches_ += 2LL * K;
    }
    if (end_epoch()) return R_;
  }
}

// ============================================================================ PDLP
// Restarted averaged PDHG (reference src/pdhg/pdlp.cpp:9-126) on the same fused kernels. The
// current and next iterates alternate between two buffers (x / x̂ storage, y / ŷ storage): an
// epoch graph is captured per starting phase. xa / ya (the running averages) live in the Δx / Δy
// buffers, x̄ in x̄'s. A check evaluates the KKT statistics of the current point and of the
// average and, after 4K iterations, the ray tests on z_k − z_{k−1} (and the drift z − z0).
template <class T>
__global__ void k_dist_terms(long long n, const T* a, const T* b, double* t) {  // (a − b)² in fp64
  B200_FOR(i, n) {
    const double d = static_cast<double>(a[i]) - static_cast<double>(b[i]);
    t[i] = d * d;
  }
}

template <class T>
void Engine::capture_pdlp_epoch(int phase) {
  const int idx = std::is_same<T, float>::value ? 1 : 0;
  if (g_pdlp_[idx][phase]) return;
  IterVecs<T>& v = vecs<T>();
  const int m = M_.m, n = M_.n, K = o_.check_every;
  const StepParams* P = params_.get();
  cudaGraph_t g;
  slab_prepare<T, EpiPdlpPrimal<T>, B200_STAGE_TMA != 0>();
  slab_prepare<T, EpiPdlpDual<T>, B200_STAGE_TMA != 0>();
  capturing_ = true;
  capture_count_ = 0;
  auto capture_scope = std::make_unique<CaptureScope>();  // no device-wide syncs elsewhere meanwhile
  B200_CHECK(cudaStreamBeginCapture(st_, cudaStreamCaptureModeThreadLocal));
  B200_CHECK(cudaEventRecordWithFlags(ev_[0], st_, cudaEventRecordExternal));
  for (int s = 0; s < K; ++s) {
    const bool odd = ((phase + s) & 1) != 0;
    T* xc = odd ? v.xh.get() : v.x.get();
    T* xn = odd ? v.x.get() : v.xh.get();
    T* yc = odd ? v.yh.get() : v.y.get();
    T* yn = odd ? v.y.get() : v.yh.get();
    EpiPdlpPrimal<T> ep{xc, sp_.c<T>(), sp_.l<T>(), sp_.u<T>(), xn, v.xb.get(), v.dx.get(), P, s};
    launch_slab_fed<T>(n, sp_.t_rp.get(), sp_.t_ri.get(), sp_.At_val<T>(), yc, ep, st_, slab_t_.get(), cap_t_, err(),
                       s >= 1, var_t_);
    EpiPdlpDual<T> ed{yc, sp_.rl<T>(), sp_.ru<T>(), yn, v.dy.get(), P, s};
    launch_slab_fed<T>(m, sp_.a_rp.get(), sp_.a_col.get(), sp_.A_val<T>(), v.xb.get(), ed, st_, slab_a_.get(), cap_a_,
                       err(), true, var_a_);
    capture_count_ += 2;
  }
  B200_CHECK(cudaEventRecordWithFlags(ev_[1], st_, cudaEventRecordExternal));
  B200_CHECK(cudaEventRecordWithFlags(ev_[2], st_, cudaEventRecordExternal));
  B200_CHECK(cudaEventRecordWithFlags(ev_[3], st_, cudaEventRecordExternal));
  const cudaError_t e = cudaStreamEndCapture(st_, &g);
  capture_scope.reset();
  capturing_ = false;
  B200_CHECK(e);
  B200_CHECK(cudaGraphInstantiate(&g_pdlp_[idx][phase], g, 0));
  cudaGraphDestroy(g);
  pdlp_kernels_[idx][phase] = capture_count_;
}

template <class T>
void Engine::capture_pdlp_check(int phase, int variant) {
  const int idx = std::is_same<T, float>::value ? 1 : 0;
  if (g_pdlp_chk_[idx][phase][variant]) return;
  IterVecs<T>& v = vecs<T>();
  const long long m = M_.m, n = M_.n;
  T* xc = phase ? v.xh.get() : v.x.get();
  T* xp = phase ? v.x.get() : v.xh.get();  // z_{k−1}, scratch for the ray directions
  T* yc = phase ? v.yh.get() : v.y.get();
  T* yp = phase ? v.y.get() : v.yh.get();
  cudaGraph_t g;
  slab_prepare<double, EpiKktRows, B200_STAGE_TMA != 0>();
  slab_prepare<double, EpiKktCols, false>();
  slab_prepare<double, EpiRayRows, B200_STAGE_TMA != 0>();
  capturing_ = true;
  capture_count_ = 0;
  auto capture_scope = std::make_unique<CaptureScope>();  // no device-wide syncs elsewhere meanwhile
  B200_CHECK(cudaStreamBeginCapture(st_, cudaStreamCaptureModeThreadLocal));
  clear_maxima();
  launch_kkt_scaled<T>(xc, yc);  // KKT of the current point -> res2_
  B200_CHECK(cudaMemcpyAsync(res2_.get(), res_.get(), kNumSlots * sizeof(double), cudaMemcpyDeviceToDevice, st_));
  clear_maxima();
  launch_kkt_scaled<T>(v.dx.get(), v.dy.get());  // KKT of the average -> res_
  if (variant >= 1) {  // Δ = z_k − z_{k−1}: axpby(1, x, −1, x_prev) (pdlp.cpp:83-85)
    k_axpby<T><<<grid_for(n), kBlock, 0, st_>>>(n, static_cast<T>(1.0), xc, static_cast<T>(-1.0), xp);
    k_axpby<T><<<grid_for(m), kBlock, 0, st_>>>(m, static_cast<T>(1.0), yc, static_cast<T>(-1.0), yp);
    B200_LAUNCH_CHECK();
    capture_count_ += 2;
    launch_ray<T>(xp, yp, r1_.get(), d1_.get(), 0);
  }
  if (variant == 2) {  // the drift z − z0: copy + axpby(−1, x0, 1, ·) (pdlp.cpp:89-93)
    k_diff<T><<<grid_for(n), kBlock, 0, st_>>>(n, xc, v.x0.get(), xp);
    k_diff<T><<<grid_for(m), kBlock, 0, st_>>>(m, yc, v.y0.get(), yp);
    B200_LAUNCH_CHECK();
    capture_count_ += 2;
    launch_ray<T>(xp, yp, r2_.get(), d2_.get(), 1);
  }
  B200_CHECK(cudaMemcpyAsync(hres_.get(), res_.get(), kNumSlots * sizeof(double), cudaMemcpyDeviceToHost, st_));
  B200_CHECK(cudaMemcpyAsync(hres2_.get(), res2_.get(), kNumSlots * sizeof(double), cudaMemcpyDeviceToHost, st_));
  const cudaError_t e = cudaStreamEndCapture(st_, &g);
  capture_scope.reset();
  capturing_ = false;
  B200_CHECK(e);
  B200_CHECK(cudaGraphInstantiate(&g_pdlp_chk_[idx][phase][variant], g, 0));
  cudaGraphDestroy(g);
  pdlp_chk_kernels_[idx][phase][variant] = capture_count_;
}

// ‖c_x − x0‖, ‖c_y − y0‖ (Backend::diff_norm2: la::parallel_sum order) for the chosen point.
template <class T>
void Engine::pdlp_distances(int cur, bool use_avg, double& dx, double& dy) {
  IterVecs<T>& v = vecs<T>();
  const long long m = M_.m, n = M_.n;
  const T* cx = use_avg ? v.dx.get() : (cur ? v.xh.get() : v.x.get());
  const T* cy = use_avg ? v.dy.get() : (cur ? v.yh.get() : v.y.get());
  k_dist_terms<T><<<grid_for(n), kBlock, 0, st_>>>(n, cx, v.x0.get(), rt_.get());
  k_dist_terms<T><<<grid_for(m), kBlock, 0, st_>>>(m, cy, v.y0.get(), rt_.get() + 2 * n);
  B200_LAUNCH_CHECK();
  plan_dist_.launch(st_);
  kernels_ += 2 + plan_dist_.kernel_count();
  sync_results();
  dx = std::sqrt(hres_[kPx]);
  dy = std::sqrt(hres_[kPy]);
}

// Restart from the chosen point: x ← c_x, y ← c_y, then x0 = xa = x, y0 = ya = y (pdlp.cpp:113-120).
template <class T>
void Engine::pdlp_restart(int cur, bool use_avg) {
  IterVecs<T>& v = vecs<T>();
  const std::size_t nb = static_cast<std::size_t>(M_.n) * sizeof(T), mb = static_cast<std::size_t>(M_.m) * sizeof(T);
  T* xc = cur ? v.xh.get() : v.x.get();
  T* yc = cur ? v.yh.get() : v.y.get();
  if (use_avg) {
    B200_CHECK(cudaMemcpyAsync(xc, v.dx.get(), nb, cudaMemcpyDeviceToDevice, st_));
    B200_CHECK(cudaMemcpyAsync(yc, v.dy.get(), mb, cudaMemcpyDeviceToDevice, st_));
  }
  B200_CHECK(cudaMemcpyAsync(v.x0.get(), xc, nb, cudaMemcpyDeviceToDevice, st_));
  B200_CHECK(cudaMemcpyAsync(v.y0.get(), yc, mb, cudaMemcpyDeviceToDevice, st_));
  B200_CHECK(cudaMemcpyAsync(v.dx.get(), xc, nb, cudaMemcpyDeviceToDevice, st_));
  B200_CHECK(cudaMemcpyAsync(v.dy.get(), yc, mb, cudaMemcpyDeviceToDevice, st_));
}

// set_precision(Fp64) for PDLP: every vector that carries state is converted.
void Engine::promote_pdlp() {
  const long long m = M_.m, n = M_.n;
  DevBuf<float>* fs[] = {&vf_.x, &vf_.x0, &vf_.xh, &vf_.xb, &vf_.dx, &vf_.y, &vf_.y0, &vf_.yh, &vf_.yb, &vf_.dy};
  DevBuf<double>* ds[] = {&vd_.x, &vd_.x0, &vd_.xh, &vd_.xb, &vd_.dx, &vd_.y, &vd_.y0, &vd_.yh, &vd_.yb, &vd_.dy};
  for (int q = 0; q < 10; ++q) {
    const long long len = q < 5 ? n : m;
    k_convert<double, float><<<grid_for(len), kBlock, 0, st_>>>(len, fs[q]->get(), ds[q]->get());
  }
  B200_LAUNCH_CHECK();
  kernels_ += 10;
  mixed_now_ = false;
}

EngineResult Engine::run_pdlp(const DeviceOutputs& out) {
  t0_ = clock::now();
  EngineResult R;
  setup();
  const long long mm = M_.m, nn = M_.n;
  res2_.alloc(kNumSlots);
  hres2_.alloc(kNumSlots);
  plan_dist_.add(rt_.get(), 0, nn, 0.0, SumOrder::kChunk64, res_.get() + kPx);
  plan_dist_.add(rt_.get() + 2 * nn, 0, mm, 0.0, SumOrder::kChunk64, res_.get() + kPy);
  plan_dist_.build(true, nullptr, st_);  // the distances enter ω: always the reference's order
  mixed_now_ = o_.mixed;
  double omega = initial_primal_weight();
  if (mixed_now_) init_iterates<float>();
  else init_iterates<double>();
  const bool warm = apply_warm_start();
  primal_weight_ = omega;
  std::string msg = warm ? "warm start" : "";
  const int K = o_.check_every;
  R.setup_seconds = elapsed();
  int cur = 0;  // 0: the current point is in the x / y buffers, 1: in the x̂ / ŷ buffers
  auto point = [&](bool avg, auto tag) {
    using T = decltype(tag);
    IterVecs<T>& v = vecs<T>();
    return std::make_pair<const T*, const T*>(avg ? v.dx.get() : (cur ? v.xh.get() : v.x.get()),
                                             avg ? v.dy.get() : (cur ? v.yh.get() : v.y.get()));
  };
  auto done = [&](Status s, bool avg, long long it, const std::string& m, int ray) {
    R.loop_seconds = elapsed() - R.setup_seconds;
    if (mixed_now_) {
      const auto p = point(avg, 0.0f);
      finish_p<float>(R, s, p.first, p.second, it, m, out, ray);
    } else {
      const auto p = point(avg, 0.0);
      finish_p<double>(R, s, p.first, p.second, it, m, out, ray);
    }
    R.kernel_launches = kernels_;
    R.iter_kernel_ms = iter_ms_;
    R.iter_kernel_launches = iter_launches_;
    R.slab_variant_primal = var_t_, R.slab_variant_dual = var_a_, R.tuned = tuned_now_ ? 1 : 0;
    R.seconds = elapsed();
    return R;
  };
  auto kkt_now = [&](bool avg) {
    clear_maxima();
    if (mixed_now_) {
      const auto p = point(avg, 0.0f);
      launch_kkt_scaled<float>(p.first, p.second);
    } else {
      const auto p = point(avg, 0.0);
      launch_kkt_scaled<double>(p.first, p.second);
    }
    sync_results();
    return read_kkt(hres_.get());
  };
  if (warm) {  // the warm point may already be good enough (pdlp.cpp:37-40)
    const Kkt kw = kkt_now(false);
    if (fast_it_ < 0 && kw.rel_kkt() <= kFirstOrderFast) fast_it_ = 0;
    if (kw.finite() && kw.converged(o_.tolerance)) return done(Status::Optimal, false, 0, "warm start already optimal", 0);
  }
  if (mixed_now_) pdlp_restart<float>(cur, false);  // x0 = xa = x, y0 = ya = y
  else pdlp_restart<double>(cur, false);
  const Kkt k0 = kkt_now(false);
  if (fast_it_ < 0 && k0.rel_kkt() <= kFirstOrderFast) fast_it_ = 0;
  double restart_kkt = k0.rel_kkt(), last_candidate = 1e300;
  long long it = 0, inner = 0;
  StepParams& hp = *hparams_.get();
  for (;;) {
    hp.tau = eta_ / omega;
    hp.sigma = eta_ * omega;
    hp.rho = 1.0;
    hp.inner0 = inner;
    hp.K = K;
    hp.done = 0;
    hp.skip_r0 = 1;
    B200_CHECK(cudaMemcpyAsync(params_.get(), &hp, sizeof(StepParams), cudaMemcpyHostToDevice, st_));
    const int pidx = mixed_now_ ? 1 : 0;
    if (mixed_now_) capture_pdlp_epoch<float>(cur);
    else capture_pdlp_epoch<double>(cur);
    B200_CHECK(cudaGraphLaunch(g_pdlp_[pidx][cur], st_));
    kernels_ += pdlp_kernels_[pidx][cur];
    it += K;
    inner += K;
    cur = (cur + K) & 1;
    const int variant = it >= 4LL * K ? (((it / K) % 4 == 0) ? 2 : 1) : 0;
    if (mixed_now_) capture_pdlp_check<float>(cur, variant);
    else capture_pdlp_check<double>(cur, variant);
    B200_CHECK(cudaGraphLaunch(g_pdlp_chk_[pidx][cur][variant], st_));
    kernels_ += pdlp_chk_kernels_[pidx][cur][variant];
    B200_CHECK(cudaStreamSynchronize(st_));
    ++R.checks;
    {
      float a = 0;
      B200_CHECK(cudaEventElapsedTime(&a, ev_[0], ev_[1]));
      iter_ms_ += a;
      iter_launches_ += 2LL * K;
    }
    const Kkt kc = read_kkt(hres2_.get()), ka = read_kkt(hres_.get());
    const bool use_avg = ka.finite() && ka.rel_kkt() < kc.rel_kkt();
    const Kkt& kk = use_avg ? ka : kc;
    if (o_.verbosity >= 2)
      std::fprintf(stderr, "pdlp-b200 it %8lld  t %7.2fs  pobj %+.10e  dobj %+.10e  rp %.2e  rd %.2e  gap %.2e  %s%s\n",
                   it, elapsed(), kk.primal_obj, kk.dual_obj, kk.rel_primal(), kk.rel_dual(), kk.rel_gap(),
                   mixed_now_ ? "fp32" : "fp64", use_avg ? " avg" : "");
    if (!kk.finite()) return done(Status::NumericalError, false, it, "non-finite KKT statistics", 0);
    if (fast_it_ < 0 && kk.rel_kkt() <= kFirstOrderFast) fast_it_ = it;
    if (kk.converged(o_.tolerance)) return done(Status::Optimal, use_avg, it, msg, 0);
    if (it >= o_.iteration_limit) return done(Status::IterationLimit, use_avg, it, msg, 0);
    if (elapsed() > o_.time_limit) return done(Status::TimeLimit, use_avg, it, msg, 0);
    if (variant >= 1) {  // check_infeasibility on Δ, then the drift (pdlp.cpp:82-98)
      const double* h = hres_.get();
      std::string why;
      int which = 1;
      Status st = ray_verdict(h, 1, kc, why);
      if (st == Status::NotSolved && inner >= K && variant == 2) {
        which = 2;
        st = ray_verdict(h, 2, kc, why);
        if (st != Status::NotSolved) why += " (drift since the restart anchor)";
      }
      if (st != Status::NotSolved) return done(st, false, it, why, which);
    }
    const double e = kk.rel_kkt();
    bool promoted = false;  // PrecisionPolicy::on_check (engine.cpp:61-79)
    if (o_.mixed && mixed_now_) {
      if (e < 0.9 * pol_best_) pol_best_ = e, pol_since_best_ = 0;
      else ++pol_since_best_;
      const bool reached = e <= kMixedPrecisionSwitch && o_.tolerance < kMixedPrecisionSwitch;
      if (reached || pol_since_best_ >= o_.mixed_stall_checks) {
        promote_pdlp();
        switch_it_ = it;
        promoted = true;
        msg += std::string(msg.empty() ? "" : "; ") + "fp32 -> fp64 at iteration " + std::to_string(it);
      }
    }
    const bool restart_now = promoted || e <= 0.2 * restart_kkt ||
                             (e <= o_.pdlp_restart_necessary * restart_kkt && e > last_candidate) ||
                             static_cast<double>(inner) >= 0.36 * static_cast<double>(it);
    last_candidate = e;
    if (!restart_now) continue;
    double dx = 0, dy = 0;
    if (mixed_now_) pdlp_distances<float>(cur, use_avg, dx, dy);
    else pdlp_distances<double>(cur, use_avg, dx, dy);
    if (dx > 1e-10 && dy > 1e-10) {
      const double th = o_.pdlp_primal_weight_smoothing;
      omega = std::exp(th * std::log(dy / dx) + (1.0 - th) * std::log(omega));
      primal_weight_ = omega;
    }
    if (mixed_now_) pdlp_restart<float>(cur, use_avg);
    else pdlp_restart<double>(cur, use_avg);
    ++R.restarts;
    inner = 0;
    restart_kkt = e;
    last_candidate = 1e300;
  }
}
// ================================================================ continuous batching
// The group scheduler: one host thread and one stream per device run the r²HPDHG epochs of every
// solve in flight together. Per epoch, each half-step is ONE launch of k_group_fed over the slabs
// of all the solves in that working precision (instead of one launch per solve), each solve with
// its own step scalars, iterates and epilogue; then every solve's own residual section (when its
// epoch starts a Halpern cycle) and check graph follow on the same stream, one synchronisation
// covers them all, and each solve takes its own decisions. A solve joins at the next epoch
// boundary once its setup (on its caller's thread and stream) is done, and leaves when it has
// finished, so requests that arrive while others run are admitted into the running group.
// The grouped kernel runs each row's arithmetic exactly as the solve's own kernel, and the
// checks are the solve's own graphs, so a solve's result does not depend on its company.
class GroupScheduler {
 public:
  struct Job {
    Engine* e = nullptr;
    bool done = false;
    unsigned timeouts = 0;
    std::exception_ptr error;
    cudaEvent_t ready = nullptr;  // the engine's stream has its step scalars (and restart) in place
  };
  // A device has PS26119_GROUPS_PER_DEVICE groups (default 2), each with its own host thread
  // and stream, so that one group's host decisions between epochs overlap another group's
  // kernels; a solve joins the group with the fewest solves.
  static GroupScheduler& for_current_device() {
    static std::mutex mu;
    static std::map<int, std::vector<GroupScheduler*>> all;  // never destroyed: the threads live until exit
    static const int per_device = [] {
      const char* e = std::getenv("PS26119_GROUPS_PER_DEVICE");
      const int k = e && *e ? std::atoi(e) : 2;
      return std::min(64, std::max(1, k));
    }();
    int dev = 0;
    B200_CHECK(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(mu);
    std::vector<GroupScheduler*>& v = all[dev];
    while (static_cast<int>(v.size()) < per_device) v.push_back(new GroupScheduler(dev));
    GroupScheduler* best = v.front();
    for (GroupScheduler* g : v)
      if (g->load_.load() < best->load_.load()) best = g;
    ++best->load_;  // counted from the choice, so that concurrent joiners spread out
    return *best;
  }
  // Runs the engine's epochs in the group until it finishes (the caller's thread waits). The
  // scheduler came from for_current_device(), which counted the solve in.
  void run(Job& job) {
    struct Leave {
      std::atomic<int>& n;
      ~Leave() { --n; }
    } leave{load_};
    std::unique_lock<std::mutex> lk(mu_);
    pending_.push_back(&job);
    cv_.notify_all();
    done_cv_.wait(lk, [&] { return job.done; });
    if (job.error) std::rethrow_exception(job.error);
  }

 private:
  explicit GroupScheduler(int dev) : dev_(dev) {
    B200_CHECK(cudaStreamCreateWithFlags(&st_, cudaStreamNonBlocking));
    B200_CHECK(cudaEventCreateWithFlags(&steps_done_, cudaEventDisableTiming));
    thread_ = std::thread([this] { loop(); });
    thread_.detach();
  }
  template <class T>
  struct Tables {  // the grouped launches' parts in one working precision (pinned and device)
    std::vector<GroupPart<T, EpiPrimal<T>>> hp;
    std::vector<GroupPart<T, EpiDual<T>>> hd;
    PinnedBuf<GroupPart<T, EpiPrimal<T>>> pp;
    PinnedBuf<GroupPart<T, EpiDual<T>>> pd;
    DevBuf<GroupPart<T, EpiPrimal<T>>> dp;
    DevBuf<GroupPart<T, EpiDual<T>>> dd;
    int blocks_p = 0, blocks_d = 0, cap_p = 16, cap_d = 16;
    void clear() { hp.clear(), hd.clear(), blocks_p = blocks_d = 0, cap_p = cap_d = 16; }
  };
  template <class T>
  void add(Tables<T>& tb, Engine& e) {
    const Engine::SlabOperands a = e.primal_operands<T>(), b = e.dual_operands<T>();
    tb.hp.push_back({a.rows, a.cap, tb.blocks_p, a.rp, a.col, static_cast<const T*>(a.val),
                     static_cast<const T*>(a.x), a.slab, a.err, e.primal_epi<T>(0)});
    tb.hd.push_back({b.rows, b.cap, tb.blocks_d, b.rp, b.col, static_cast<const T*>(b.val),
                     static_cast<const T*>(b.x), b.slab, b.err, e.dual_epi<T>(0)});
    tb.blocks_p += slab_count(a.rows), tb.blocks_d += slab_count(b.rows);
    tb.cap_p = std::max(tb.cap_p, a.cap), tb.cap_d = std::max(tb.cap_d, b.cap);
  }
  template <class T>
  void upload(Tables<T>& tb) {
    const std::size_t n = tb.hp.size();
    if (n == 0) return;
    if (tb.pp.size() < n) tb.pp.alloc(2 * n), tb.pd.alloc(2 * n), tb.dp.alloc(2 * n), tb.dd.alloc(2 * n);
    std::copy(tb.hp.begin(), tb.hp.end(), tb.pp.get());
    std::copy(tb.hd.begin(), tb.hd.end(), tb.pd.get());
    B200_CHECK(cudaMemcpyAsync(tb.dp.get(), tb.pp.get(), n * sizeof(tb.hp[0]), cudaMemcpyHostToDevice, st_));
    B200_CHECK(cudaMemcpyAsync(tb.dd.get(), tb.pd.get(), n * sizeof(tb.hd[0]), cudaMemcpyHostToDevice, st_));
  }
  // One half-step of every solve in precision T: the primal (Ãᵀy) or dual (Ãx̄) grouped kernel.
  // pdl: programmatic dependent launch, as in the solo epoch graph (every dual; every primal
  // whose predecessor is a grouped kernel).
  template <class T, class Epi>
  void launch(const DevBuf<GroupPart<T, Epi>>& parts, int nparts, int blocks, int cap, int step, bool pdl) {
    if (nparts == 0 || blocks == 0) return;
    const unsigned smem = fed_layout(Epi::kVecs, static_cast<int>(sizeof(T)), cap).bytes;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(static_cast<unsigned>(blocks));
    cfg.blockDim = dim3(kSlabRows);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st_;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = (B200_PDL && pdl) ? 1 : 0;
    B200_CHECK(cudaLaunchKernelEx(&cfg, k_group_fed<T, Epi>, parts.get(), nparts, step));
  }
  // One epoch of every active solve: each solve's step scalars on its own stream; the grouped
  // iteration kernels on the group's stream once every solve's stream is ready; each solve's
  // residual section (when its epoch starts a Halpern cycle) on the group's stream after step 0;
  // then every solve's check graph on its own stream, so the checks of different solves overlap.
  void epoch(std::vector<Job*>& active) {
    tf_.clear(), td_.clear();
    for (Job* j : active) {
      j->e->begin_epoch();
      if (!j->ready) B200_CHECK(cudaEventCreateWithFlags(&j->ready, cudaEventDisableTiming));
      B200_CHECK(cudaEventRecord(j->ready, j->e->stream()));
      B200_CHECK(cudaStreamWaitEvent(st_, j->ready, 0));
      if (j->e->mixed_now()) add(tf_, *j->e);
      else add(td_, *j->e);
    }
    upload(tf_), upload(td_);
    const int nf = static_cast<int>(tf_.hp.size()), nd = static_cast<int>(td_.hp.size());
    const int K = active.front()->e->check_every();
    for (int s = 0; s < K; ++s) {
      const bool pdl_primal = s >= 2;  // step 1 follows the residual sections
      launch(td_.dp, nd, td_.blocks_p, td_.cap_p, s, pdl_primal && nf == 0);
      launch(tf_.dp, nf, tf_.blocks_p, tf_.cap_p, s, false);
      launch(td_.dd, nd, td_.blocks_d, td_.cap_d, s, nf == 0);
      launch(tf_.dd, nf, tf_.blocks_d, tf_.cap_d, s, false);
      if (s == 0)
        for (Job* j : active) j->e->launch_r0(st_);
    }
    B200_CHECK(cudaEventRecord(steps_done_, st_));
    for (Job* j : active) {
      B200_CHECK(cudaStreamWaitEvent(j->e->stream(), steps_done_, 0));
      j->e->launch_check();
    }
    for (Job* j : active) B200_CHECK(cudaStreamSynchronize(j->e->stream()));
  }
  void loop() {
    (void)cudaSetDevice(dev_);
    std::vector<Job*> active;
    for (;;) {
      {
        std::unique_lock<std::mutex> lk(mu_);
        cv_.wait(lk, [&] { return !pending_.empty() || !active.empty(); });
        for (Job* j : pending_) active.push_back(j);
        pending_.clear();
      }
      std::vector<Job*> finished;
      try {
        epoch(active);
        for (std::size_t k = 0; k < active.size();) {
          Job* j = active[k];
          if (j->e->end_epoch()) {
            j->timeouts = j->e->stage_errors();
            finished.push_back(j);
            active.erase(active.begin() + static_cast<long>(k));
          } else {
            ++k;
          }
        }
      } catch (...) {  // a device error: every solve in the group ends with it
        const std::exception_ptr err = std::current_exception();
        for (Job* j : active) j->error = err, finished.push_back(j);
        active.clear();
        (void)cudaGetLastError();
      }
      if (!finished.empty()) {
        std::lock_guard<std::mutex> lk(mu_);
        for (Job* j : finished) {
          if (j->ready) cudaEventDestroy(j->ready), j->ready = nullptr;
          j->done = true;
        }
        done_cv_.notify_all();
      }
    }
  }
  int dev_ = 0;
  std::atomic<int> load_{0};  // solves joined and not yet finished
  cudaStream_t st_ = nullptr;
  cudaEvent_t steps_done_ = nullptr;
  std::thread thread_;
  std::mutex mu_;
  std::condition_variable cv_, done_cv_;
  std::vector<Job*> pending_;
  Tables<double> td_;
  Tables<float> tf_;
};

}  // namespace

namespace {
thread_local bool t_grouped = false;
}
void set_grouped_engine(bool on) { t_grouped = on; }

EngineResult run_engine(const DeviceModel& M, const EngineOptions& opt, const DeviceOutputs& out, void* stream) {
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  bool own = false;
  if (!st) {
    // The caller's inputs may still be in flight on the legacy default stream: finish them,
    // then run on a stream of our own (capturable, unlike the legacy stream).
    cudaError_t se = cudaSuccess;
    with_device_sync([&se] { se = cudaDeviceSynchronize(); });
    B200_CHECK(se);
    B200_CHECK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    own = true;
  }
  struct StreamGuard {
    cudaStream_t s;
    bool own;
    ~StreamGuard() {
      if (own) cudaStreamDestroy(s);
    }
  } guard{st, own};
  EngineResult R;
  unsigned timeouts = 0;
  {
    auto e = std::make_unique<Engine>(M, opt, st);
    // Large LPs keep their own kernels: they fill the device alone, and in lockstep with a
    // group their epochs would wait for everyone's checks. Small ones (launch-bound alone) join
    // the group. The limit is PS26119_GROUP_MAX_NNZ nonzeros (default 100,000).
    static const long long group_max_nnz = [] {
      const char* e = std::getenv("PS26119_GROUP_MAX_NNZ");
      return e && *e ? std::atoll(e) : 100000LL;
    }();
    if (t_grouped && !opt.pdlp && opt.check_every == 64 && M.nnz <= group_max_nnz) {
      // setup here, on this caller's stream; the epochs in the device's group
      if (e->start(out)) {
        R = e->result();
        timeouts = e->stage_errors();
      } else {
        GroupScheduler& g = GroupScheduler::for_current_device();
        GroupScheduler::Job job;
        job.e = e.get();
        g.run(job);
        R = e->result();
        timeouts = job.timeouts;
      }
    } else {
      R = opt.pdlp ? e->run_pdlp(out) : e->run(out);
      timeouts = e->stage_errors();
    }
    const auto t = std::chrono::steady_clock::now();
    e.reset();
    R.teardown_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t).count();
  }
  if (timeouts) throw CudaError("a shared-memory staging wait timed out on the device");
  return R;
}

namespace {

// Host <-> device copies of pageable host arrays through two page-locked staging blocks: the host
// threads fill (or empty) one block while the copy engine moves the other, so a copy runs at
// the host threads' memcpy rate instead of the single-threaded staging of a pageable
// cudaMemcpyAsync. `jobs` hold device and host addresses and sizes; blocks come from (and go back
// to) the process's pinned-block cache.
struct StagedCopy {
  void* dev;
  void* host;
  std::size_t bytes;
};
constexpr std::size_t kStageBytes = std::size_t{16} << 20;

// The pieces of the concatenated jobs, at most kStageBytes per block: block b takes bytes
// [b·kStageBytes, (b+1)·kStageBytes) of the concatenation.
template <class F>
void for_each_piece(const std::vector<StagedCopy>& jobs, std::size_t block, F&& f) {
  const std::size_t lo = block * kStageBytes, hi = lo + kStageBytes;
  std::size_t off = 0;
  for (const StagedCopy& j : jobs) {
    const std::size_t a = std::max(lo, off), e = std::min(hi, off + j.bytes);
    if (a < e) f(j, a - off, a - lo, e - a);  // job, offset in the job, offset in the block, bytes
    off += j.bytes;
  }
}

class StagingBlocks {
 public:
  explicit StagingBlocks(cudaStream_t st) : st_(st) {
    for (int b = 0; b < 2; ++b) {
      buf_[b] = static_cast<char*>(PinnedBlockCache::instance().acquire(kStageBytes));
      B200_CHECK(cudaEventCreateWithFlags(&ev_[b], cudaEventDisableTiming));
    }
  }
  ~StagingBlocks() {
    for (int b = 0; b < 2; ++b) {  // the copies of both blocks have completed before they go back
      cudaEventSynchronize(ev_[b]);
      cudaEventDestroy(ev_[b]);
      PinnedBlockCache::instance().release(buf_[b], kStageBytes);
    }
  }
  void upload(const std::vector<StagedCopy>& jobs) {
    const std::size_t nb = blocks(jobs);
    for (std::size_t k = 0; k < nb; ++k) {
      const int b = static_cast<int>(k & 1);
      B200_CHECK(cudaEventSynchronize(ev_[b]));  // this block's previous copy has left it
      std::vector<CopyJob> fill;
      for_each_piece(jobs, k, [&](const StagedCopy& j, std::size_t jo, std::size_t bo, std::size_t n) {
        fill.push_back({buf_[b] + bo, static_cast<const char*>(j.host) + jo, n});
      });
      parallel_copy(fill.data(), fill.size());
      for_each_piece(jobs, k, [&](const StagedCopy& j, std::size_t jo, std::size_t bo, std::size_t n) {
        B200_CHECK(cudaMemcpyAsync(static_cast<char*>(j.dev) + jo, buf_[b] + bo, n, cudaMemcpyHostToDevice, st_));
      });
      B200_CHECK(cudaEventRecord(ev_[b], st_));
    }
  }
  void download(const std::vector<StagedCopy>& jobs) {
    const std::size_t nb = blocks(jobs);
    auto issue = [&](std::size_t k) {
      const int b = static_cast<int>(k & 1);
      for_each_piece(jobs, k, [&](const StagedCopy& j, std::size_t jo, std::size_t bo, std::size_t n) {
        B200_CHECK(cudaMemcpyAsync(buf_[b] + bo, static_cast<const char*>(j.dev) + jo, n, cudaMemcpyDeviceToHost, st_));
      });
      B200_CHECK(cudaEventRecord(ev_[b], st_));
    };
    if (nb > 0) issue(0);
    for (std::size_t k = 0; k < nb; ++k) {
      const int b = static_cast<int>(k & 1);
      if (k + 1 < nb) issue(k + 1);  // the other block: its previous contents were copied out below
      B200_CHECK(cudaEventSynchronize(ev_[b]));
      std::vector<CopyJob> drain;
      for_each_piece(jobs, k, [&](const StagedCopy& j, std::size_t jo, std::size_t bo, std::size_t n) {
        drain.push_back({static_cast<char*>(j.host) + jo, buf_[b] + bo, n});
      });
      parallel_copy(drain.data(), drain.size());
    }
  }

 private:
  static std::size_t blocks(const std::vector<StagedCopy>& jobs) {
    std::size_t total = 0;
    for (const StagedCopy& j : jobs) total += j.bytes;
    return (total + kStageBytes - 1) / kStageBytes;
  }
  cudaStream_t st_;
  char* buf_[2] = {nullptr, nullptr};
  cudaEvent_t ev_[2] = {nullptr, nullptr};
};

}  // namespace

EngineResult run_engine_host(const HostModelView& H, const EngineOptions& opt, HostOutputs& out) {
  cudaStream_t st;
  B200_CHECK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  struct StreamGuard {
    cudaStream_t s;
    ~StreamGuard() { cudaStreamDestroy(s); }
  } guard{st};
  const int m = H.m, n = H.n;
  const long long nnz = H.col_start[n];
  const std::size_t mm = static_cast<std::size_t>(m), nn = static_cast<std::size_t>(n);
  const std::size_t nz = static_cast<std::size_t>(nnz);
  DevBuf<double> c, cl, cu, rl, ru, v, x, y, z, dr, pr;
  DevBuf<int> cs, ri;
  c.alloc(nn), cl.alloc(nn), cu.alloc(nn), rl.alloc(mm), ru.alloc(mm), cs.alloc(nn + 1), ri.alloc(nz), v.alloc(nz);
  x.alloc(nn), z.alloc(nn), pr.alloc(nn), y.alloc(mm), dr.alloc(mm);
  {
    StagingBlocks stage(st);
    const auto d = [](const double* h) { return const_cast<double*>(h); };
    stage.upload({{c.get(), d(H.c), nn * 8}, {cl.get(), d(H.col_lower), nn * 8}, {cu.get(), d(H.col_upper), nn * 8},
                  {rl.get(), d(H.row_lower), mm * 8}, {ru.get(), d(H.row_upper), mm * 8},
                  {cs.get(), const_cast<int*>(H.col_start), (nn + 1) * 4}, {ri.get(), const_cast<int*>(H.row_index), nz * 4},
                  {v.get(), d(H.value), nz * 8}});
  }
  DeviceModel M;
  M.m = m, M.n = n, M.sense = H.sense, M.offset = H.offset, M.nnz = nnz;
  M.c = c.get(), M.col_lower = cl.get(), M.col_upper = cu.get(), M.row_lower = rl.get(), M.row_upper = ru.get();
  M.col_start = cs.get(), M.row_index = ri.get(), M.value = v.get();
  DeviceOutputs o{x.get(), y.get(), z.get(), dr.get(), pr.get()};
  EngineResult R = run_engine(M, opt, o, st);
  out.x = pooled_vector(n), out.y = pooled_vector(m), out.z = pooled_vector(n);
  std::vector<StagedCopy> back = {{x.get(), out.x.data(), nn * 8}, {y.get(), out.y.data(), mm * 8},
                                  {z.get(), out.z.data(), nn * 8}};
  if (R.have_dual_ray) out.dual_ray.resize(m), back.push_back({dr.get(), out.dual_ray.data(), mm * 8});
  if (R.have_primal_ray) out.primal_ray.resize(n), back.push_back({pr.get(), out.primal_ray.data(), nn * 8});
  {
    StagingBlocks stage(st);
    stage.download(back);
  }
  B200_CHECK(cudaStreamSynchronize(st));
  return R;
}

}  // namespace b200
