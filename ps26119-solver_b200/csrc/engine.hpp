// engine.hpp — host-side interface of the GPU r²HPDHG engine (no CUDA types).
//
// The engine mirrors the reference's first-order path:
//   EngineOptions  ≙ pdhg::EngineOptions (src/pdhg/engine.h:27-48) + ScalingOptions
//                    (src/pdhg/scaling.h:32-46)
//   run_engine     ≙ pdhg::solve_r2hpdhg (src/pdhg/r2hpdhg.cpp:11-162) on a model whose
//                    arrays are already on the device, including EngineContext setup and
//                    finish (src/pdhg/engine.cpp:195-307)
//   GpuBackend     ≙ the pdhg::Backend plugin interface (src/pdhg/backend.h:36-69)
#pragma once

#include <cstdint>
#include <memory>
#include <string>
#include <vector>

namespace b200 {

enum class Status { Optimal, Infeasible, Unbounded, IterationLimit, TimeLimit, NumericalError, NotSolved };
const char* status_name(Status s);

struct ScalingOptions {
  int geometric_mean_iterations = 12;
  double geometric_mean_min_log10_range = 4.5;
  int ruiz_iterations = 10;
  bool pock_chambolle = true;
  bool bound_objective_rescaling = true;
};

struct EngineOptions {
  double tolerance = 1e-8;
  long long iteration_limit = 100000000LL;
  double time_limit = 3600.0;
  int check_every = 64;
  bool mixed = false;
  bool exact = false;  // reference summation order in every reduction
  ScalingOptions scaling;
  double reflection = 1.0;
  double restart_sufficient = 0.2, restart_necessary = 0.5, restart_artificial = 0.36;
  double pid_kp = 0.99, pid_ki = 0.01, pid_kd = 0.0, pid_integral_decay = 0.3;
  double pid_max_log_step = 2.302585092994046;
  // PDLP-style restarted averaged PDHG instead of r²HPDHG (pdlp.cpp; engine.h:44-46 defaults)
  bool pdlp = false;
  double pdlp_restart_necessary = 0.8, pdlp_primal_weight_smoothing = 0.5;
  // warm start in the ORIGINAL space (host memory), engine.cpp:237-266
  std::vector<double> warm_x, warm_y;
  double warm_primal_weight = 0.0;
  // mixed precision: checks without a 10% gain of the best relative KKT before the switch to fp64
  // (PrecisionPolicy, engine.cpp:61-79, uses 10)
  int mixed_stall_checks = 10;
  // termination normalisation overrides (set by the presolve wrapper), engine.h:31
  double kkt_b_norm = -1, kkt_c_norm = -1, kkt_obj_shift = 0;
  int verbosity = 0;
};

// A model whose arrays live on the current device (borrowed, not owned).
struct DeviceModel {
  int m = 0, n = 0, sense = 1;
  double offset = 0.0;
  const double *c = nullptr, *col_lower = nullptr, *col_upper = nullptr, *row_lower = nullptr, *row_upper = nullptr;
  const int *col_start = nullptr, *row_index = nullptr;
  const double* value = nullptr;
  long long nnz = 0;  // col_start[n], provided by the caller
};

struct EngineResult {
  Status status = Status::NotSolved;
  long long iterations = 0;
  double objective = 0, dual_objective = 0, primal_residual = 0, dual_residual = 0, gap = 0;
  double primal_weight = 0, eta = 0;
  long long iterations_to_fast = -1, switch_iteration = -1, restarts = 0, checks = 0;
  std::string message;
  double setup_seconds = 0, loop_seconds = 0, finish_seconds = 0, seconds = 0;
  long long kernel_launches = 0;
  double iter_kernel_ms = 0;
  double teardown_seconds = 0;  // releasing the engine's device state after the loop
  long long iter_kernel_launches = 0;
  bool have_dual_ray = false, have_primal_ray = false;
  // in-process check of the reported point on the engine's model (device-computed)
  int check = -1;
  double check_primal = 0, check_dual = 0, check_gap = 0;
  // the iteration kernels' launch variants (spmv.cuh kSlabVariants) and whether this solve
  // measured them itself (the autotuner's first solve of a shape class)
  int slab_variant_primal = 0, slab_variant_dual = 0, tuned = 0;
};

// Where run_engine leaves its outputs (device pointers, each may be null).
struct DeviceOutputs {
  double* x = nullptr;      // n, original space
  double* y = nullptr;      // m, original sense (z = c − Aᵀy)
  double* z = nullptr;      // n
  double* dual_ray = nullptr;    // m (Infeasible)
  double* primal_ray = nullptr;  // n (Unbounded)
};

// For the calling thread's later solves: run the r²HPDHG epochs in the device's group (one grouped
// launch per half-step with every other grouped solve in flight) instead of on the solve's own
// stream. Results are the same either way. The request loop's slot threads set it.
void set_grouped_engine(bool on);

// Runs r²HPDHG on the device model. `stream` is a cudaStream_t (nullptr = own stream).
EngineResult run_engine(const DeviceModel& M, const EngineOptions& opt, const DeviceOutputs& out, void* stream);

// Host convenience: uploads a host CSC model, runs the engine, downloads the outputs.
struct HostModelView {
  int m = 0, n = 0, sense = 1;
  double offset = 0.0;
  const double *c, *col_lower, *col_upper, *row_lower, *row_upper;
  const int *col_start, *row_index;
  const double* value;
};
struct HostOutputs {
  std::vector<double> x, y, z, dual_ray, primal_ray;
};
// A per-thread pool of solution-sized host vectors (x, y, z), kept within the host reuse limit
// (host_keep): pooled_vector(n) returns n zeros, in a pooled buffer's memory when one is large
// enough (no fresh pages to fault in); pool_vector hands a finished vector's memory back.
std::vector<double> pooled_vector(std::size_t n);
void pool_vector(std::vector<double>&& v);
EngineResult run_engine_host(const HostModelView& M, const EngineOptions& opt, HostOutputs& out);

// Throws a runtime_error when no usable CUDA device exists (the C API reports it as
// NOT_SOLVED "CUDA backend unavailable: …", cpu_backend.cpp:293-310).
void require_device();

// ----------------------------------------------------------------------------- backend
// The pdhg::Backend plugin interface (backend.h:36-69) on the GPU, over a model uploaded
// from host memory and scaled on the device. Vectors are addressed by integer handles.
class GpuBackend {
 public:
  static std::unique_ptr<GpuBackend> create(const HostModelView& M, const ScalingOptions& so, bool exact);
  virtual ~GpuBackend() = default;
  virtual void set_precision(bool mixed) = 0;
  virtual bool mixed() const = 0;
  virtual int create_vector(bool dual) = 0;
  virtual void upload(int v, const double* src) = 0;
  virtual void download(int v, double* dst) = 0;
  virtual void fill(int v, double a) = 0;
  virtual void copy(int dst, int src) = 0;
  virtual void axpby(double a, int x, double b, int y) = 0;
  virtual void spmv(int x, int out) = 0;
  virtual void spmv_t(int y, int out) = 0;
  virtual double dot(int a, int b) = 0;
  virtual double norm2(int a) = 0;
  virtual double diff_norm2(int a, int b) = 0;
  virtual void primal_step(int x, int aty, double tau, int xh) = 0;
  virtual void dual_step(int y, int ax, double sigma, int yh) = 0;
  virtual void r2h_primal(int x, int x0, int aty, double tau, double w, double rho, int xh, int xb) = 0;
  virtual void r2h_dual(int y, int y0, int ax, double sigma, double w, double rho, int yh, int yb) = 0;
  // fused forms used by the engine: Ãᵀy + r2h_primal, Ãx̄ + r2h_dual in one kernel each
  virtual void fused_primal(int y, int x, int x0, double tau, double w, double rho, int xh, int xb) = 0;
  virtual void fused_dual(int xb, int y, int y0, double sigma, double w, double rho, int yh, int yb) = 0;
  // [primal_residual, dual_residual, primal_obj, dual_obj, b_norm, c_norm, primal_max_rel, dual_max_rel]
  virtual void kkt(int xs, int ys, double* out) = 0;
  // scaled data, same `which` codes as the reference shim (0 Ã vals … 8 col_scale)
  virtual long long scaled_get(int which, double* dst) = 0;
  virtual long long scaled_structure(int which, int* row_ptr, int* col) = 0;
  // [bound_scale, obj_scale, log10_range, geometric_mean_applied]
  virtual void scalars(double* out) = 0;
  virtual double norm2_estimate() = 0;
  virtual void sync() = 0;
};

}  // namespace b200
