// c_api.cpp — the C ABI (include/ps26119.h, include/ps26119_backend.h). Exceptions never
// cross this boundary (reference src/core/c_api.cpp:1-304 for the five reference symbols).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <exception>
#include <memory>
#include <new>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/ps26119.h"
#include "../../include/ps26119_backend.h"
#include "certify.hpp"
#include "io.hpp"
#include "parallel.hpp"
#include "solver.hpp"
#include "serve.hpp"

using namespace b200;

namespace {

thread_local ps26119_stats g_stats{};
thread_local std::string g_backend_error;

void set_text(char* dst, std::size_t cap, const std::string& s) { std::snprintf(dst, cap, "%s", s.c_str()); }

void clear(ps26119_result* r) {  // c_api.cpp:22-26
  std::memset(r, 0, sizeof *r);
  r->status = PS26119_NOT_SOLVED;
  r->check = -1;
}

// C options -> Options (c_api.cpp:29-56). Returns an error text, or nullptr.
const char* to_options(const ps26119_options* opt, int num_rows, int num_cols, Options& o) {
  if (!opt) return nullptr;
  switch (opt->algorithm) {
    case PS26119_ALG_ORACLE: o.algorithm = Algorithm::Oracle; break;
    case PS26119_ALG_PDLP: o.algorithm = Algorithm::Pdlp; break;
    case PS26119_ALG_R2HPDHG: o.algorithm = Algorithm::R2hpdhg; break;
    case PS26119_ALG_SIMPLEX: o.algorithm = Algorithm::Simplex; break;
    case PS26119_ALG_AUTO: o.algorithm = Algorithm::Auto; break;
    default: return "unknown algorithm";
  }
  if (opt->precision != PS26119_PREC_FP64 && opt->precision != PS26119_PREC_MIXED) return "unknown precision";
  o.precision = opt->precision == PS26119_PREC_MIXED ? Precision::Mixed : Precision::Fp64;
  o.use_gpu = opt->use_gpu != 0;
  if (!(opt->tolerance >= 0) || !std::isfinite(opt->tolerance)) return "tolerance must be a finite number >= 0";
  if (!(opt->time_limit >= 0)) return "time_limit must be >= 0 (0 = default)";
  if (opt->iteration_limit < 0) return "iteration_limit must be >= 0 (0 = default)";
  if (opt->threads < 0) return "threads must be >= 0 (0 = all cores)";
  if (opt->tolerance > 0) o.tolerance = opt->tolerance;
  if (opt->time_limit > 0) o.time_limit = opt->time_limit;
  if (opt->iteration_limit > 0) o.iteration_limit = opt->iteration_limit;
  o.verbosity = opt->verbosity;
  o.threads = opt->threads;
  if (opt->warm_x) o.warm_x.assign(opt->warm_x, opt->warm_x + num_cols);
  if (opt->warm_y) o.warm_y.assign(opt->warm_y, opt->warm_y + num_rows);
  return nullptr;
}

const char* apply_engine_options(const ps26119_engine_options* eo, Options& o) {
  if (!eo) return nullptr;
  if (eo->check_every < 0) return "check_every must be >= 0";
  o.presolve = eo->presolve != 0;
  if (eo->check_every > 0) o.check_every = eo->check_every;
  o.exact = eo->exact_reductions != 0;
  if (eo->ruiz_iterations >= 0) o.scaling.ruiz_iterations = eo->ruiz_iterations;
  if (eo->pock_chambolle >= 0) o.scaling.pock_chambolle = eo->pock_chambolle != 0;
  if (eo->bound_objective_rescaling >= 0) o.scaling.bound_objective_rescaling = eo->bound_objective_rescaling != 0;
  if (eo->reflection != 0) o.reflection = eo->reflection;
  if (!(eo->warm_primal_weight >= 0)) return "warm_primal_weight must be >= 0";
  o.warm_primal_weight = eo->warm_primal_weight;
  if (eo->mixed_stall_checks < 0) return "mixed_stall_checks must be >= 0";
  if (eo->mixed_stall_checks > 0) o.mixed_stall_checks = eo->mixed_stall_checks;
  return nullptr;
}

void fill_stats(const Solution& s, long long m, long long n, long long nnz) {
  const EngineResult& R = s.engine_result;
  g_stats = ps26119_stats{};
  g_stats.setup_seconds = R.setup_seconds;
  g_stats.loop_seconds = R.loop_seconds;
  g_stats.finish_seconds = R.finish_seconds;
  g_stats.presolve_seconds = s.presolve_seconds;
  g_stats.primal_weight = R.primal_weight;
  g_stats.eta = R.eta;
  g_stats.checks = R.checks;
  g_stats.restarts = R.restarts;
  g_stats.iterations_to_fast = R.iterations_to_fast;
  g_stats.switch_iteration = R.switch_iteration;
  g_stats.kernel_launches = R.kernel_launches;
  g_stats.m = m, g_stats.n = n, g_stats.nnz = nnz;
  g_stats.spmv_kernel_ms = R.iter_kernel_ms;
  g_stats.spmv_kernel_launches = R.iter_kernel_launches;
  g_stats.teardown_seconds = R.teardown_seconds;
  g_stats.slab_variant_primal = R.slab_variant_primal;
  g_stats.slab_variant_dual = R.slab_variant_dual;
  g_stats.tuned = R.tuned;
}

void fill(const Solution& s, ps26119_result* result) {  // c_api.cpp:58-71
  result->status = static_cast<int>(s.status);
  result->objective = s.objective;
  result->dual_objective = s.dual_objective;
  result->primal_residual = s.primal_residual;
  result->dual_residual = s.dual_residual;
  result->gap = s.gap;
  result->certified_bound = s.certified_bound;
  result->iterations = s.iterations;
  result->seconds = s.seconds;
  result->check = s.check == "PASS" ? 1 : s.check == "FAIL" ? 0 : -1;
  set_text(result->engine, sizeof result->engine, s.engine);
  set_text(result->message, sizeof result->message, s.message);
}

int solve_host(int num_rows, int num_cols, int sense, double obj_offset, const double* c, const double* col_lower,
               const double* col_upper, const double* row_lower, const double* row_upper, const int* col_start,
               const int* row_index, const double* value, const ps26119_options* opt,
               const ps26119_engine_options* eo, ps26119_result* result, double* x, double* y, double* z,
               double* dual_ray, double* primal_ray) {
  const auto call_t0 = std::chrono::steady_clock::now();
  if (!result) return PS26119_INVALID_ARGUMENT;
  clear(result);
  auto invalid = [&](const char* why) {
    result->status = PS26119_INVALID_ARGUMENT;
    set_text(result->message, sizeof result->message, why);
    return result->status;
  };
  if (num_rows < 0 || num_cols < 0) return invalid("negative dimension");
  if (!col_start) return invalid("col_start is NULL");
  if (num_cols > 0 && (!c || !col_lower || !col_upper)) return invalid("column data is NULL");
  if (num_rows > 0 && (!row_lower || !row_upper)) return invalid("row bounds are NULL");
  const int nnz = col_start[num_cols];
  if (nnz < 0) return invalid("col_start[n] < 0");
  if (nnz > 0 && (!row_index || !value)) return invalid("matrix arrays are NULL");
  try {
    phase_log_begin(opt && opt->verbosity >= 1);
    auto t_model = std::chrono::steady_clock::now();
    // the calling thread's host copy of the model: its memory is reused by the next call on
    // this thread (within the host reuse limit, host_keep), which then copies into pages that
    // are already mapped instead of page-faulting fresh ones
    struct ModelHolder {
      Model m;
      std::size_t accounted = 0;
      ~ModelHolder() { host_keep(accounted, 0); }
    };
    static thread_local ModelHolder t_model_copy;
    struct KeepModel {
      ModelHolder& h;
      ~KeepModel() {
        if (!host_keep(h.accounted, capacity_bytes(h.m))) h.m = Model{};
      }
    } keep_model{t_model_copy};
    Model& m = t_model_copy.m;
    m.is_integer.clear();
    m.num_rows = num_rows;
    m.num_cols = num_cols;
    m.sense = sense;
    m.obj_offset = obj_offset;
    // copied on the host threads: one thread's memcpy of a large model's arrays is several times
    // slower than the memory allows
    const std::size_t n = static_cast<std::size_t>(num_cols), rows = static_cast<std::size_t>(num_rows),
                      k = static_cast<std::size_t>(nnz);
    size_for_copy(m.obj, n), size_for_copy(m.col_lower, n), size_for_copy(m.col_upper, n);
    size_for_copy(m.row_lower, rows), size_for_copy(m.row_upper, rows);
    size_for_copy(m.col_start, n + 1), size_for_copy(m.row_index, k), size_for_copy(m.value, k);
    const CopyJob copies[] = {{m.obj.data(), c, 8 * n},
                              {m.col_lower.data(), col_lower, 8 * n},
                              {m.col_upper.data(), col_upper, 8 * n},
                              {m.row_lower.data(), row_lower, 8 * rows},
                              {m.row_upper.data(), row_upper, 8 * rows},
                              {m.col_start.data(), col_start, 4 * (n + 1)},
                              {m.row_index.data(), row_index, 4 * k},
                              {m.value.data(), value, 8 * k}};
    parallel_copy(copies, sizeof copies / sizeof copies[0]);
    if (auto err = m.validate(); !err.empty()) {
      phase_log_begin(false);
      return invalid(("invalid model: " + err).c_str());
    }
    phase_note("model", std::chrono::duration<double>(std::chrono::steady_clock::now() - t_model).count());
    Options o;
    if (const char* bad = to_options(opt, num_rows, num_cols, o)) return phase_log_begin(false), invalid(bad);
    if (const char* bad = apply_engine_options(eo, o)) return phase_log_begin(false), invalid(bad);
    o.model_validated = true;  // validated just above
    Solution s = solve(m, o);
    fill(s, result);
    fill_stats(s, s.engine_result.iterations > 0 ? num_rows : 0, num_cols, nnz);
    g_stats.call_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - call_t0).count();
    std::vector<CopyJob> outs;  // the caller's outputs, copied on the host threads
    auto out = [&outs](double* dst, const std::vector<double>& v, int len) {
      if (dst && v.size() == static_cast<std::size_t>(len)) outs.push_back({dst, v.data(), sizeof(double) * len});
    };
    out(x, s.x, num_cols);
    out(y, s.y, num_rows);
    out(z, s.z, num_cols);
    out(dual_ray, s.dual_ray, num_rows);
    out(primal_ray, s.primal_ray, num_cols);
    parallel_copy(outs.data(), outs.size());
    pool_vector(std::move(s.x)), pool_vector(std::move(s.y)), pool_vector(std::move(s.z));  // for the next call
    phase_note("call", std::chrono::duration<double>(std::chrono::steady_clock::now() - call_t0).count());
    phase_log_end("solve_lp");
    return result->status;
  } catch (const std::bad_alloc&) {
    phase_log_begin(false);
    result->status = PS26119_NOT_SOLVED;
    set_text(result->message, sizeof result->message, "out of memory");
    return result->status;
  } catch (const std::exception& e) {
    phase_log_begin(false);
    result->status = PS26119_NUMERICAL_ERROR;
    set_text(result->message, sizeof result->message, e.what());
    return result->status;
  } catch (...) {
    phase_log_begin(false);
    result->status = PS26119_NUMERICAL_ERROR;
    set_text(result->message, sizeof result->message, "unknown error");
    return result->status;
  }
}

}  // namespace

namespace b200 {
// Sets the calling thread's last-error text (read through ps26119_backend_last_error); used by
// entry points defined outside this file.
void set_backend_error(const std::string& text) { g_backend_error = text; }
}  // namespace b200

struct ps26119_backend {
  std::unique_ptr<GpuBackend> impl;
};

extern "C" {

const char* ps26119_version(void) { return "0.1.0+b200"; }

void ps26119_default_options(ps26119_options* opt) {  // c_api.cpp:179-192
  if (!opt) return;
  opt->algorithm = PS26119_ALG_AUTO;
  opt->precision = PS26119_PREC_FP64;
  opt->use_gpu = 0;
  opt->tolerance = 1e-8;
  opt->time_limit = 3600.0;
  opt->iteration_limit = 100000000LL;
  opt->verbosity = 0;
  opt->threads = 1;
  opt->warm_x = nullptr;
  opt->warm_y = nullptr;
}

void ps26119_default_engine_options(ps26119_engine_options* eo) {
  if (!eo) return;
  eo->presolve = 1;
  eo->check_every = 64;
  eo->exact_reductions = 0;
  eo->ruiz_iterations = -1;
  eo->pock_chambolle = -1;
  eo->bound_objective_rescaling = -1;
  eo->reflection = 0.0;
  eo->warm_primal_weight = 0.0;
  eo->mixed_stall_checks = 0;
  eo->reserved = 0;
}

int ps26119_solve_lp(int num_rows, int num_cols, int sense, double obj_offset, const double* c,
                     const double* col_lower, const double* col_upper, const double* row_lower,
                     const double* row_upper, const int* col_start, const int* row_index, const double* value,
                     const ps26119_options* opt, ps26119_result* result, double* x, double* y, double* z) {
  return solve_host(num_rows, num_cols, sense, obj_offset, c, col_lower, col_upper, row_lower, row_upper, col_start,
                    row_index, value, opt, nullptr, result, x, y, z, nullptr, nullptr);
}

int ps26119_solve_lp_ex(int num_rows, int num_cols, int sense, double obj_offset, const double* c,
                        const double* col_lower, const double* col_upper, const double* row_lower,
                        const double* row_upper, const int* col_start, const int* row_index, const double* value,
                        const ps26119_options* opt, ps26119_result* result, double* x, double* y, double* z,
                        double* dual_ray, double* primal_ray) {
  return solve_host(num_rows, num_cols, sense, obj_offset, c, col_lower, col_upper, row_lower, row_upper, col_start,
                    row_index, value, opt, nullptr, result, x, y, z, dual_ray, primal_ray);
}

int ps26119_solve_lp_engine(int num_rows, int num_cols, int sense, double obj_offset, const double* c,
                            const double* col_lower, const double* col_upper, const double* row_lower,
                            const double* row_upper, const int* col_start, const int* row_index,
                            const double* value, const ps26119_options* opt, const ps26119_engine_options* eo,
                            ps26119_result* result, double* x, double* y, double* z, double* dual_ray,
                            double* primal_ray) {
  return solve_host(num_rows, num_cols, sense, obj_offset, c, col_lower, col_upper, row_lower, row_upper, col_start,
                    row_index, value, opt, eo, result, x, y, z, dual_ray, primal_ray);
}

int ps26119_solve_mps(const char* path, const ps26119_options* opt, ps26119_result* result,
                      const char* solution_path) {  // c_api.cpp:161-202
  if (!result) return PS26119_INVALID_ARGUMENT;
  clear(result);
  auto invalid = [&](const std::string& why) {
    result->status = PS26119_INVALID_ARGUMENT;
    set_text(result->message, sizeof result->message, why);
    return result->status;
  };
  if (!path) return invalid("path is NULL");
  if (solution_path) {  // fail before solving: the solution file must be writable
    std::FILE* probe = std::fopen(solution_path, "r");
    const bool existed = probe != nullptr;
    if (probe) std::fclose(probe);
    std::FILE* f = std::fopen(solution_path, "a");
    if (!f) return invalid(std::string("cannot write the solution file '") + solution_path + "'");
    std::fclose(f);
    if (!existed) std::remove(solution_path);
  }
  try {
    Model m;
    ModelInfo info;
    std::string err;
    if (!read_mps(path, m, info, err)) return invalid("read error: " + err);
    if (opt && (opt->warm_x || opt->warm_y)) return invalid("warm start is not supported by ps26119_solve_mps");
    Options o;
    if (const char* bad = to_options(opt, m.num_rows, m.num_cols, o)) return invalid(bad);
    Solution s = solve(m, o);
    if (info.has_integers())
      s.message = std::string("LP relaxation (integrality ignored)") + (s.message.empty() ? "" : "; ") + s.message;
    s.model_fingerprint = fingerprint_hex(m);
    fill(s, result);
    if (solution_path && !write_solution(solution_path, m, info, s, err))
      set_text(result->message, sizeof result->message, "solved, but " + err);
    return result->status;
  } catch (const std::bad_alloc&) {
    result->status = PS26119_NOT_SOLVED;
    set_text(result->message, sizeof result->message, "out of memory");
    return result->status;
  } catch (const std::exception& e) {
    result->status = PS26119_NUMERICAL_ERROR;
    set_text(result->message, sizeof result->message, e.what());
    return result->status;
  }
}

int ps26119_solve_lp_device(int num_rows, int num_cols, int sense, double obj_offset, const double* d_c,
                            const double* d_col_lower, const double* d_col_upper, const double* d_row_lower,
                            const double* d_row_upper, const int* d_col_start, const int* d_row_index,
                            const double* d_value, const ps26119_options* opt, const ps26119_engine_options* eo,
                            ps26119_result* result, double* d_x, double* d_y, double* d_z, void* stream) {
  const auto call_t0 = std::chrono::steady_clock::now();
  if (!result) return PS26119_INVALID_ARGUMENT;
  clear(result);
  auto invalid = [&](const char* why) {
    result->status = PS26119_INVALID_ARGUMENT;
    set_text(result->message, sizeof result->message, why);
    return result->status;
  };
  if (num_rows < 0 || num_cols < 0) return invalid("negative dimension");
  if (sense != 1 && sense != -1) return invalid("sense must be +1 or -1");
  if (!d_col_start) return invalid("col_start is NULL");
  if (num_cols > 0 && (!d_c || !d_col_lower || !d_col_upper)) return invalid("column data is NULL");
  if (num_rows > 0 && (!d_row_lower || !d_row_upper)) return invalid("row bounds are NULL");
  try {
    Options o;
    if (const char* bad = to_options(opt, 0, 0, o)) return invalid(bad);
    if (const char* bad = apply_engine_options(eo, o)) return invalid(bad);
    if (opt && (opt->warm_x || opt->warm_y)) return invalid("warm start is not supported by the device entry point");
    if (o.algorithm != Algorithm::Auto && o.algorithm != Algorithm::R2hpdhg)
      return invalid("the device entry point runs r2hpdhg only");
    require_device();
    int nnz = 0;
    if (cudaMemcpy(&nnz, d_col_start + num_cols, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
      return invalid("col_start is not a device pointer on the current device");
    if (nnz < 0) return invalid("col_start[n] < 0");
    if (nnz > 0 && (!d_row_index || !d_value)) return invalid("matrix arrays are NULL");
    DeviceModel M;
    M.m = num_rows, M.n = num_cols, M.sense = sense, M.offset = obj_offset, M.nnz = nnz;
    M.c = d_c, M.col_lower = d_col_lower, M.col_upper = d_col_upper, M.row_lower = d_row_lower;
    M.row_upper = d_row_upper, M.col_start = d_col_start, M.row_index = d_row_index, M.value = d_value;
    EngineOptions e;
    e.tolerance = o.tolerance;
    e.time_limit = o.time_limit;
    e.iteration_limit = o.iteration_limit;
    e.check_every = o.check_every;
    e.mixed = o.precision == Precision::Mixed;
    e.exact = o.exact;
    e.scaling = o.scaling;
    e.reflection = o.reflection;
    e.warm_primal_weight = o.warm_primal_weight;
    e.mixed_stall_checks = o.mixed_stall_checks;
    e.verbosity = o.verbosity;
    const EngineResult R = run_engine(M, e, DeviceOutputs{d_x, d_y, d_z, nullptr, nullptr}, stream);
    Solution s;
    s.status = R.status;
    s.iterations = R.iterations;
    s.objective = R.objective;
    s.dual_objective = R.dual_objective;
    s.primal_residual = R.primal_residual;
    s.dual_residual = R.dual_residual;
    s.gap = R.gap;
    s.seconds = R.seconds;
    s.message = R.message;
    s.engine_result = R;
    if (s.status == Status::Optimal) {  // gate on the device-computed check (solve.cpp:163-184)
      s.check = R.check ? "PASS" : "FAIL";
      if (!R.check && o.tolerance < 1e-6) {
        s.status = Status::NumericalError;
        s.message += std::string(s.message.empty() ? "" : "; ") + "Optimal withdrawn, in-process check failed";
      }
    }
    fill(s, result);
    fill_stats(s, num_rows, num_cols, nnz);
    g_stats.call_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - call_t0).count();
    return result->status;
  } catch (const std::bad_alloc&) {
    result->status = PS26119_NOT_SOLVED;
    set_text(result->message, sizeof result->message, "out of memory");
    return result->status;
  } catch (const std::exception& e) {
    result->status = PS26119_NUMERICAL_ERROR;
    set_text(result->message, sizeof result->message, e.what());
    return result->status;
  }
}

void ps26119_last_stats(ps26119_stats* out) {
  if (out) *out = g_stats;
}

// ------------------------------------------------------------------ backend ABI
const char* ps26119_backend_last_error(void) { return g_backend_error.c_str(); }

#define B200_GUARD(body)                                  \
  try {                                                   \
    if (!b || !b->impl) {                                 \
      g_backend_error = "null backend";                   \
      return PS26119_INVALID_ARGUMENT;                    \
    }                                                     \
    body;                                                 \
    return 0;                                             \
  } catch (const std::bad_alloc&) {                       \
    g_backend_error = "out of memory";                    \
    return PS26119_NOT_SOLVED;                            \
  } catch (const std::exception& e) {                     \
    g_backend_error = e.what();                           \
    return PS26119_NUMERICAL_ERROR;                       \
  }
// inside B200_GUARD: a NULL host pointer argument is an invalid argument, not a crash
#define B200_NEED(p)                            \
  if (!(p)) {                                   \
    g_backend_error = "NULL pointer argument";  \
    return PS26119_INVALID_ARGUMENT;            \
  }

int ps26119_backend_new(ps26119_backend** out, int num_rows, int num_cols, int sense, double obj_offset,
                        const double* c, const double* col_lower, const double* col_upper, const double* row_lower,
                        const double* row_upper, const int* col_start, const int* row_index, const double* value,
                        const ps26119_scaling_options* so, int exact) {
  if (!out) return PS26119_INVALID_ARGUMENT;
  *out = nullptr;
  try {
    Model m;
    m.num_rows = num_rows, m.num_cols = num_cols, m.sense = sense, m.obj_offset = obj_offset;
    auto invalid = [](const char* why) {
      g_backend_error = why;
      return PS26119_INVALID_ARGUMENT;
    };
    if (num_rows < 0 || num_cols < 0 || !col_start) return invalid("invalid dimensions or NULL col_start");
    if (num_cols > 0 && (!c || !col_lower || !col_upper)) return invalid("column data is NULL");
    if (num_rows > 0 && (!row_lower || !row_upper)) return invalid("row bounds are NULL");
    const int nnz = col_start[num_cols];
    if (nnz < 0) return invalid("col_start[n] < 0");
    if (nnz > 0 && (!row_index || !value)) return invalid("matrix arrays are NULL");
    m.obj.assign(c, c + num_cols);
    m.col_lower.assign(col_lower, col_lower + num_cols);
    m.col_upper.assign(col_upper, col_upper + num_cols);
    m.row_lower.assign(row_lower, row_lower + num_rows);
    m.row_upper.assign(row_upper, row_upper + num_rows);
    m.col_start.assign(col_start, col_start + num_cols + 1);
    m.row_index.assign(row_index, row_index + nnz);
    m.value.assign(value, value + nnz);
    if (auto err = m.validate(); !err.empty()) {
      g_backend_error = "invalid model: " + err;
      return PS26119_INVALID_ARGUMENT;
    }
    ScalingOptions sc;
    if (so) {
      sc.geometric_mean_iterations = so->geometric_mean_iterations;
      sc.geometric_mean_min_log10_range = so->geometric_mean_min_log10_range;
      sc.ruiz_iterations = so->ruiz_iterations;
      sc.pock_chambolle = so->pock_chambolle != 0;
      sc.bound_objective_rescaling = so->bound_objective_rescaling != 0;
    }
    auto* b = new ps26119_backend;
    try {
      b->impl = GpuBackend::create(m.view(), sc, exact != 0);
    } catch (...) {
      delete b;
      throw;
    }
    *out = b;
    return 0;
  } catch (const std::bad_alloc&) {
    g_backend_error = "out of memory";
    return PS26119_NOT_SOLVED;
  } catch (const std::exception& e) {
    g_backend_error = std::string("CUDA backend unavailable: ") + e.what();
    return PS26119_NOT_SOLVED;
  }
}

void ps26119_backend_free(ps26119_backend* b) { delete b; }

int ps26119_backend_set_precision(ps26119_backend* b, int mixed) { B200_GUARD(b->impl->set_precision(mixed != 0)) }
int ps26119_backend_create(ps26119_backend* b, int dual) {
  try {
    if (!b || !b->impl) return -1;
    return b->impl->create_vector(dual != 0);
  } catch (const std::exception& e) {
    g_backend_error = e.what();
    return -1;
  }
}
int ps26119_backend_upload(ps26119_backend* b, int v, const double* src) { B200_GUARD(B200_NEED(src); b->impl->upload(v, src)) }
int ps26119_backend_download(ps26119_backend* b, int v, double* dst) { B200_GUARD(B200_NEED(dst); b->impl->download(v, dst)) }
int ps26119_backend_fill(ps26119_backend* b, int v, double a) { B200_GUARD(b->impl->fill(v, a)) }
int ps26119_backend_copy(ps26119_backend* b, int dst, int src) { B200_GUARD(b->impl->copy(dst, src)) }
int ps26119_backend_axpby(ps26119_backend* b, double a, int x, double bb, int y) { B200_GUARD(b->impl->axpby(a, x, bb, y)) }
int ps26119_backend_spmv(ps26119_backend* b, int x, int out) { B200_GUARD(b->impl->spmv(x, out)) }
int ps26119_backend_spmv_t(ps26119_backend* b, int y, int out) { B200_GUARD(b->impl->spmv_t(y, out)) }
int ps26119_backend_dot(ps26119_backend* b, int x, int y, double* out) { B200_GUARD(B200_NEED(out); *out = b->impl->dot(x, y)) }
int ps26119_backend_norm2(ps26119_backend* b, int x, double* out) { B200_GUARD(B200_NEED(out); *out = b->impl->norm2(x)) }
int ps26119_backend_diff_norm2(ps26119_backend* b, int x, int y, double* out) { B200_GUARD(B200_NEED(out); *out = b->impl->diff_norm2(x, y)) }
int ps26119_backend_primal_step(ps26119_backend* b, int x, int aty, double tau, int xh) {
  B200_GUARD(b->impl->primal_step(x, aty, tau, xh))
}
int ps26119_backend_dual_step(ps26119_backend* b, int y, int ax, double sigma, int yh) {
  B200_GUARD(b->impl->dual_step(y, ax, sigma, yh))
}
int ps26119_backend_r2h_primal(ps26119_backend* b, int x, int x0, int aty, double tau, double w, double rho, int xh,
                               int xb) {
  B200_GUARD(b->impl->r2h_primal(x, x0, aty, tau, w, rho, xh, xb))
}
int ps26119_backend_r2h_dual(ps26119_backend* b, int y, int y0, int ax, double sigma, double w, double rho, int yh,
                             int yb) {
  B200_GUARD(b->impl->r2h_dual(y, y0, ax, sigma, w, rho, yh, yb))
}
int ps26119_backend_fused_primal(ps26119_backend* b, int y, int x, int x0, double tau, double w, double rho, int xh,
                                 int xb) {
  B200_GUARD(b->impl->fused_primal(y, x, x0, tau, w, rho, xh, xb))
}
int ps26119_backend_fused_dual(ps26119_backend* b, int xb, int y, int y0, double sigma, double w, double rho, int yh,
                               int yb) {
  B200_GUARD(b->impl->fused_dual(xb, y, y0, sigma, w, rho, yh, yb))
}
int ps26119_backend_kkt(ps26119_backend* b, int xs, int ys, double* out) { B200_GUARD(B200_NEED(out); b->impl->kkt(xs, ys, out)) }
int ps26119_backend_sync(ps26119_backend* b) { B200_GUARD(b->impl->sync()) }
long long ps26119_backend_scaled_get(ps26119_backend* b, int which, double* dst) {
  try {
    return b && b->impl ? b->impl->scaled_get(which, dst) : -1;
  } catch (const std::exception& e) {
    g_backend_error = e.what();
    return -1;
  }
}
long long ps26119_backend_scaled_structure(ps26119_backend* b, int which, int* row_ptr, int* col) {
  try {
    return b && b->impl ? b->impl->scaled_structure(which, row_ptr, col) : -1;
  } catch (const std::exception& e) {
    g_backend_error = e.what();
    return -1;
  }
}
int ps26119_backend_scalars(ps26119_backend* b, double* out) { B200_GUARD(B200_NEED(out); b->impl->scalars(out)) }
int ps26119_backend_norm2_estimate(ps26119_backend* b, double* out) { B200_GUARD(B200_NEED(out); *out = b->impl->norm2_estimate()) }

}  // extern "C"

extern "C" int ps26119_solve_batch(int num_rows, int num_cols, int sense, double obj_offset, const double* c,
                                   const double* col_lower, const double* col_upper, const double* row_lower,
                                   const double* row_upper, const int* col_start, const int* row_index,
                                   const double* value, int num_scenarios, const ps26119_scenario* scenarios,
                                   const ps26119_options* opt, const ps26119_engine_options* engine,
                                   ps26119_result* results, double* x, double* y, double* z) {
  if (num_scenarios < 0 || (num_scenarios > 0 && (!results || !scenarios))) return PS26119_INVALID_ARGUMENT;
  for (int k = 0; k < num_scenarios; ++k) clear(&results[k]);
  auto fail = [&](int status, const std::string& why) {
    for (int k = 0; k < num_scenarios; ++k) {
      results[k].status = status;
      set_text(results[k].message, sizeof results[k].message, why);
    }
    return status;
  };
  if (num_rows < 0 || num_cols < 0) return fail(PS26119_INVALID_ARGUMENT, "negative dimension");
  if (!col_start) return fail(PS26119_INVALID_ARGUMENT, "col_start is NULL");
  if (num_cols > 0 && (!c || !col_lower || !col_upper)) return fail(PS26119_INVALID_ARGUMENT, "column data is NULL");
  if (num_rows > 0 && (!row_lower || !row_upper)) return fail(PS26119_INVALID_ARGUMENT, "row bounds are NULL");
  const int nnz = col_start[num_cols];
  if (nnz < 0) return fail(PS26119_INVALID_ARGUMENT, "col_start[n] < 0");
  if (nnz > 0 && (!row_index || !value)) return fail(PS26119_INVALID_ARGUMENT, "matrix arrays are NULL");
  try {
    Model m;
    m.num_rows = num_rows;
    m.num_cols = num_cols;
    m.sense = sense;
    m.obj_offset = obj_offset;
    m.obj.assign(c, c + num_cols);
    m.col_lower.assign(col_lower, col_lower + num_cols);
    m.col_upper.assign(col_upper, col_upper + num_cols);
    m.row_lower.assign(row_lower, row_lower + num_rows);
    m.row_upper.assign(row_upper, row_upper + num_rows);
    m.col_start.assign(col_start, col_start + num_cols + 1);
    m.row_index.assign(row_index, row_index + nnz);
    m.value.assign(value, value + nnz);
    Options o;
    if (const char* err = to_options(opt, num_rows, num_cols, o)) return fail(PS26119_INVALID_ARGUMENT, err);
    if (const char* err = apply_engine_options(engine, o)) return fail(PS26119_INVALID_ARGUMENT, err);
    std::vector<Scenario> sc(static_cast<std::size_t>(num_scenarios));
    auto take = [](const double* a, int len) { return a ? std::vector<double>(a, a + len) : std::vector<double>(); };
    for (int k = 0; k < num_scenarios; ++k) {
      const ps26119_scenario& s = scenarios[k];
      sc[k].obj = take(s.obj, num_cols);
      sc[k].col_lower = take(s.col_lower, num_cols);
      sc[k].col_upper = take(s.col_upper, num_cols);
      sc[k].row_lower = take(s.row_lower, num_rows);
      sc[k].row_upper = take(s.row_upper, num_rows);
    }
    const std::vector<Solution> sols = solve_batch(m, sc, o);
    long long launches = 0;
    for (int k = 0; k < num_scenarios; ++k) {
      const Solution& s = sols[k];
      fill(s, &results[k]);
      launches = std::max(launches, s.engine_result.kernel_launches);
      const std::size_t ok = static_cast<std::size_t>(k);
      if (x && s.x.size() == static_cast<std::size_t>(num_cols))
        std::copy(s.x.begin(), s.x.end(), x + ok * num_cols);
      if (y && s.y.size() == static_cast<std::size_t>(num_rows))
        std::copy(s.y.begin(), s.y.end(), y + ok * num_rows);
      if (z && s.z.size() == static_cast<std::size_t>(num_cols))
        std::copy(s.z.begin(), s.z.end(), z + ok * num_cols);
    }
    g_stats = ps26119_stats{};
    g_stats.kernel_launches = launches;
    g_stats.m = num_rows, g_stats.n = num_cols, g_stats.nnz = nnz;
    if (num_scenarios > 0) {
      g_stats.setup_seconds = sols[0].setup_seconds;
      g_stats.spmv_kernel_ms = sols[0].engine_result.iter_kernel_ms;
      g_stats.spmv_kernel_launches = sols[0].engine_result.iter_kernel_launches;
    }
    return 0;
  } catch (const std::bad_alloc&) {
    return fail(PS26119_NOT_SOLVED, "out of memory");
  } catch (const std::exception& e) {
    return fail(PS26119_NUMERICAL_ERROR, e.what());
  }
}

namespace {
// A validated host Model from the C arrays, or an error text.
const char* model_from(int m, int n, int sense, double offset, const double* c, const double* cl, const double* cu,
                       const double* rl, const double* ru, const int* cs, const int* ri, const double* v, Model& M) {
  if (m < 0 || n < 0) return "negative dimension";
  if (!cs) return "col_start is NULL";
  if (n > 0 && (!c || !cl || !cu)) return "column data is NULL";
  if (m > 0 && (!rl || !ru)) return "row bounds are NULL";
  const int nnz = cs[n];
  if (nnz < 0) return "col_start[n] < 0";
  if (nnz > 0 && (!ri || !v)) return "matrix arrays are NULL";
  M.num_rows = m, M.num_cols = n, M.sense = sense, M.obj_offset = offset;
  M.obj.assign(c, c + n), M.col_lower.assign(cl, cl + n), M.col_upper.assign(cu, cu + n);
  M.row_lower.assign(rl, rl + m), M.row_upper.assign(ru, ru + m);
  M.col_start.assign(cs, cs + n + 1), M.row_index.assign(ri, ri + nnz), M.value.assign(v, v + nnz);
  static thread_local std::string err;
  err = M.validate();
  return err.empty() ? nullptr : err.c_str();
}
}  // namespace

extern "C" int ps26119_certified_bound(int num_rows, int num_cols, int sense, double obj_offset, const double* c,
                                       const double* col_lower, const double* col_upper, const double* row_lower,
                                       const double* row_upper, const int* col_start, const int* row_index,
                                       const double* value, const double* y, int use_implied_bounds, double* out) {
  if (!out || (num_rows > 0 && !y)) return PS26119_INVALID_ARGUMENT;
  try {
    Model M;
    if (model_from(num_rows, num_cols, sense, obj_offset, c, col_lower, col_upper, row_lower, row_upper, col_start,
                   row_index, value, M))
      return PS26119_INVALID_ARGUMENT;
    const SafeBound b = certified_dual_bound(M, std::vector<double>(y, y + num_rows), use_implied_bounds != 0);
    out[0] = b.finite ? 1.0 : 0.0;
    out[1] = b.bound;
    out[2] = b.unbounded_row_terms;
    out[3] = b.unbounded_col_terms;
    return 0;
  } catch (const std::bad_alloc&) {
    return PS26119_NOT_SOLVED;
  } catch (const std::exception&) {
    return PS26119_NUMERICAL_ERROR;
  }
}

extern "C" int ps26119_check_certificate(int kind, int num_rows, int num_cols, int sense, double obj_offset,
                                         const double* c, const double* col_lower, const double* col_upper,
                                         const double* row_lower, const double* row_upper, const int* col_start,
                                         const int* row_index, const double* value, const double* x,
                                         const double* ray, double* out) {
  if (!out || (kind != 0 && kind != 1)) return PS26119_INVALID_ARGUMENT;
  const int len = kind == 0 ? num_rows : num_cols;
  if (len > 0 && !ray) return PS26119_INVALID_ARGUMENT;
  if (kind == 1 && num_cols > 0 && !x) return PS26119_INVALID_ARGUMENT;
  try {
    Model M;
    if (model_from(num_rows, num_cols, sense, obj_offset, c, col_lower, col_upper, row_lower, row_upper, col_start,
                   row_index, value, M))
      return PS26119_INVALID_ARGUMENT;
    const std::vector<double> r(ray, ray + len);
    const CertificateCheck k = kind == 0 ? check_infeasibility_certificate(M, r)
                                         : check_unboundedness_certificate(M, std::vector<double>(x, x + num_cols), r);
    out[0] = k.present, out[1] = k.passed, out[2] = k.rigorous, out[3] = k.measure, out[4] = k.violation;
    return 0;
  } catch (const std::bad_alloc&) {
    return PS26119_NOT_SOLVED;
  } catch (const std::exception&) {
    return PS26119_NUMERICAL_ERROR;
  }
}

// ============================================================ serving (serve.hpp)
struct ps26119_server {
  b200::Server server;
  explicit ps26119_server(const b200::ServerOptions& o) : server(o) {}
};

extern "C" ps26119_server* ps26119_server_create(const ps26119_server_options* opt) {
  b200::ServerOptions o;
  if (opt) {
    if (opt->slots < 0 || !(opt->hbm_budget_bytes >= 0) || !(opt->dry_run_seconds >= 0)) return nullptr;
    o.slots = opt->slots;
    o.hbm_budget_bytes = opt->hbm_budget_bytes;
    o.dry_run_seconds = opt->dry_run_seconds;
    o.grouped = opt->solo_engines == 0;
  }
  try {
    return new ps26119_server(o);
  } catch (...) {
    return nullptr;
  }
}

extern "C" long long ps26119_server_submit(ps26119_server* server, int num_rows, int num_cols, int sense,
                                           double obj_offset, const double* c, const double* col_lower,
                                           const double* col_upper, const double* row_lower, const double* row_upper,
                                           const int* col_start, const int* row_index, const double* value,
                                           const ps26119_options* opt, ps26119_result* error) {
  if (error) clear(error);
  auto invalid = [&](const std::string& why) {
    if (error) {
      error->status = PS26119_INVALID_ARGUMENT;
      set_text(error->message, sizeof error->message, why);
    }
    return -static_cast<long long>(PS26119_INVALID_ARGUMENT);
  };
  if (!server) return invalid("server is NULL");
  try {
    Model m;
    if (const char* bad = model_from(num_rows, num_cols, sense, obj_offset, c, col_lower, col_upper, row_lower,
                                     row_upper, col_start, row_index, value, m))
      return invalid(std::string("invalid model: ") + bad);
    Options o;
    if (const char* bad = to_options(opt, num_rows, num_cols, o)) return invalid(bad);
    return server->server.submit(std::move(m), std::move(o));
  } catch (const std::bad_alloc&) {
    return invalid("out of memory");
  } catch (const std::exception& e) {
    return invalid(e.what());
  }
}

extern "C" int ps26119_server_poll(ps26119_server* server, long long id, int wait, ps26119_result* result, double* x,
                                   double* y, double* z, ps26119_request_times* times) {
  if (!server) return -1;
  Solution s;
  b200::RequestTimes t;
  int r;
  try {
    r = server->server.take(id, wait != 0, s, t);
  } catch (...) {  // no exception crosses the C boundary
    return -1;
  }
  if (r != 1) return r;
  if (result) {
    clear(result);
    fill(s, result);
  }
  auto out = [](double* dst, const std::vector<double>& v) {
    if (dst && !v.empty()) std::memcpy(dst, v.data(), sizeof(double) * v.size());
  };
  out(x, s.x);
  out(y, s.y);
  out(z, s.z);
  if (times) *times = ps26119_request_times{t.submitted, t.started, t.finished};
  return 1;
}

extern "C" void ps26119_server_destroy(ps26119_server* server) { delete server; }
