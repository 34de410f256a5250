// solver.hpp — host-side model, options, solution and the solve() dispatcher around the
// GPU engine. Mirrors the reference's contracts:
//   Model     include/ps26119/model.h:18-70      (CSC, validate, fingerprint, row_activity)
//   Options   include/ps26119/options.h:37-82    (the fields this library honours)
//   Solution  include/ps26119/solution.h:21-86
//   solve()   src/core/solve.cpp:194-609          (presolve wrapper, direct solve, gate)
//   presolve  src/core/presolve.{h,cpp}            (R1-R4 + primal/dual postsolve)
//   checker   src/core/solution_checker.{h,cpp}
//   batch     include/ps26119/batch.h:22-33, src/pdhg/batch.cpp:129-441
#pragma once

#include <cstdint>
#include <limits>
#include <string>
#include <vector>

#include "engine.hpp"

namespace b200 {

constexpr double kInf = std::numeric_limits<double>::infinity();
constexpr double kNaN = std::numeric_limits<double>::quiet_NaN();

struct Model {
  int num_rows = 0, num_cols = 0, sense = 1;
  double obj_offset = 0.0;
  std::vector<double> obj, col_lower, col_upper, row_lower, row_upper;
  std::vector<int> col_start, row_index;
  std::vector<double> value;
  std::vector<char> is_integer;  // from a file with integer markers; empty = all continuous (the
                                 // solve is the LP relaxation; only the fingerprint uses it)

  std::size_t nnz() const { return value.size(); }
  std::string validate() const;        // model.cpp:93-160
  std::string crossed_bounds() const;  // model.cpp:162-167
  double objective_value(const std::vector<double>& x) const;
  std::vector<double> row_activity(const std::vector<double>& x) const;
  std::uint64_t fingerprint() const;   // model.cpp:53-85 (FNV-1a)
  HostModelView view() const;
};

enum class Algorithm { Auto, Oracle, Pdlp, R2hpdhg, Simplex };
enum class Precision { Fp64, Mixed };

struct Options {
  Algorithm algorithm = Algorithm::Auto;
  Precision precision = Precision::Fp64;
  bool use_gpu = false;
  double tolerance = 1e-8;
  double time_limit = 3600.0;
  long long iteration_limit = 100000000LL;
  int verbosity = 0;
  int threads = 1;
  bool presolve = true;
  int check_every = 64;
  bool exact = false;
  ScalingOptions scaling;
  double reflection = 1.0;
  std::vector<double> warm_x, warm_y;
  double warm_primal_weight = 0.0;
  double kkt_b_norm = -1, kkt_c_norm = -1, kkt_obj_shift = 0;
  int mixed_stall_checks = 10;  // PrecisionPolicy's stall window (engine.cpp:61-79)
  // Internal: the caller has validated this model (the C API does, before its copy is solved), so
  // the solve skips repeating that pass over it, and over presolve's reduced model, which is
  // valid by construction. Off for every other caller.
  bool model_validated = false;
};

struct Solution {
  Status status = Status::NotSolved;
  std::vector<double> x, y, z, dual_ray, primal_ray;
  double objective = kNaN, dual_objective = kNaN, primal_residual = kNaN, dual_residual = kNaN, gap = kNaN;
  long long iterations = 0;
  double seconds = 0, setup_seconds = 0;
  double certified_bound = kNaN;
  double primal_weight = kNaN;
  std::string check;  // "PASS" / "FAIL" / "" (not applicable / not certified)
  double check_primal = kNaN, check_dual = kNaN, check_gap = kNaN;
  std::string engine = "r2hpdhg-b200", precision = "fp64", message;
  EngineResult engine_result;  // statistics of the last engine run
  double presolve_seconds = 0;
  std::string model_fingerprint;  // set by solve_batch: the scenario model's (batch.cpp:113-127)
  long long iterations_to_fast = -1;
};

// The in-process optimality check (solution_checker.cpp:61-133).
struct CheckReport {
  double max_primal_violation = 0, max_dual_violation = 0, max_complementarity = 0;
  double primal_objective = 0, dual_objective = 0, relative_gap = 0;
  bool primal_ok = false, dual_ok = false, gap_ok = false;
  bool passed() const { return primal_ok && dual_ok && gap_ok; }
  std::string summary() const;
};
CheckReport check_solution(const Model& lp, const std::vector<double>& x, const std::vector<double>& row_dual);

// fp64 KKT statistics of (x, y) on the original model with multipliers sense·y, as the
// reference's kkt_general defines them (src/pdhg/cpu_backend.cpp:225-284, KktStats in
// src/pdhg/termination.h:35-60); the presolve wrapper's test of a postsolved point
// (original_kkt in src/core/solve.cpp:77-84).
struct OriginalKkt {
  double primal_residual = 0, dual_residual = 0, primal_obj = 0, dual_obj = 0, b_norm = 0, c_norm = 0;
  double primal_max_rel = 0, dual_max_rel = 0;
  bool converged(double eps) const;
};
OriginalKkt original_kkt(const Model& model, const std::vector<double>& x, const std::vector<double>& y);

// Presolve R1-R4 with postsolve (presolve.h:22-65).
struct PresolveResult {
  enum class Outcome { Reduced, Infeasible, Unchanged } outcome = Outcome::Unchanged;
  Model reduced;
  std::string message;
  int removed_rows = 0, removed_cols = 0, tightened_bounds = 0;
  std::vector<int> row_map, col_map;
  std::vector<double> fixed_value;
  struct Singleton {
    int row, col;
    double a;
    bool set_lower, set_upper;
  };
  std::vector<Singleton> singletons;
};
PresolveResult presolve(const Model& model);
// The same into `r`, reusing the capacity of its vectors (the dispatcher keeps one per thread).
void presolve_into(const Model& model, PresolveResult& r);
Solution postsolve(const Model& original, const PresolveResult& r, const Solution& reduced);

// One 64-bit FNV-1a digest of everything presolve decided: outcome, counts, row and column maps,
// fixed values, singleton records (in order) and the reduced model's fingerprint. Two presolves
// agree when their digests do (the CLI's `info` prints it).
std::uint64_t presolve_digest(const PresolveResult& r);

// The library entry point: never throws (solve.cpp:194-210).
Solution solve(const Model& model, const Options& options);

// Host buffers kept between calls. A call on a large model spends more time page-faulting
// fresh multi-hundred-megabyte vectors than copying into them, so the dispatcher keeps, per
// thread, its model copy, presolve scratch and reduced model, and the certified bound's term
// arrays, and reuses their memory on the next call. All threads together keep at most
// PS26119_HOST_REUSE_MB MiB (default 2048; 0 keeps nothing); beyond that a thread frees its
// buffers after the call. host_keep(accounted, bytes): a holder that has `accounted` bytes
// counted asks to keep `bytes`; true: kept (and counted), false: the caller frees them.
bool host_keep(std::size_t& accounted, std::size_t bytes);
std::size_t capacity_bytes(const Model& m);

// Host phase timings of one entry-point call: phase_log_begin(on) starts a log on this thread
// (nothing is recorded when `on` is false), phase_note adds one phase, phase_log_end prints the
// phases to stderr on one line and closes the log.
void phase_log_begin(bool on);
void phase_note(const char* name, double seconds);
void phase_log_end(const char* what);

// Differences from the base model; an empty vector means "same as the base" (batch.h:22-28).
struct Scenario {
  std::vector<double> obj, col_lower, col_upper, row_lower, row_upper;
};
// K LPs sharing the base's matrix, solved in lockstep on the GPU (batch.h:32-33): one Solution
// per scenario, in order. Never throws. Runs on the GPU whatever options.use_gpu says (the
// reference's batch is CPU-only; this is its replacement).
std::vector<Solution> solve_batch(const Model& base, const std::vector<Scenario>& scenarios, const Options& options);

// Model::fingerprint of the base model with each scenario's vectors (empty = the base's).
std::vector<std::uint64_t> scenario_fingerprints(const Model& base, const std::vector<Scenario>& scenarios);

}  // namespace b200
