// host_probe.cpp — test driver: the library's host passes on model files, for the bitwise
// comparisons with the reference in tests/test_presolve.py and tests/test_check.py. It links
// the library's host objects (solver, certify, io); the GPU entry points those objects
// reference are defined below as stubs that are never called (no solve runs here).
//
//   host_probe postsolve <out.bin> (<model> <red_x.bin> <red_y.bin>)...
//     presolve, then postsolve of the reduced point. One presolve result and the solution
//     vectors are reused from job to job, as repeated solves on one thread reuse them. For each
//     job out.bin receives the sizes of x, y and z (int64 each), then x, y, z and the objective
//     (float64); a job whose model presolve does not reduce writes three sizes of -1 only.
//   host_probe digest <out.txt> <model>...
//     presolve of each model into one reused result: its digest (as `ps26119 info` prints it),
//     one line per model.
//   host_probe kkt <out.bin> (<model> <x.bin> <y.bin>)...
//     original_kkt of the point: per job 11 float64 — the 8 statistics, then converged() at
//     1e-4, 1e-8 and 1e-9.
//   host_probe check <out.bin> (<model> <x.bin> <y.bin>)...
//     check_solution and certified_dual_bound (with implied bounds) of the point on the
//     model: per job 7 float64 — passed, max primal violation, max dual violation, relative
//     gap, primal objective, dual objective, certified bound.
#include <cstdio>
#include <stdexcept>
#include <string>
#include <vector>

#include "batch.hpp"
#include "certify.hpp"
#include "io.hpp"
#include "solver.hpp"

namespace b200 {
EngineResult run_engine_host(const HostModelView&, const EngineOptions&, HostOutputs&) {
  throw std::runtime_error("no engine in the host probe");
}
const char* status_name(Status) { return "?"; }
void require_device() {}
std::vector<BatchOutcome> run_batch_host(const HostModelView&, const std::vector<BatchScenarioView>&,
                                         const std::vector<int>&, const EngineOptions&,
                                         std::chrono::steady_clock::time_point) {
  throw std::runtime_error("no engine in the host probe");
}
}  // namespace b200

using namespace b200;

static std::vector<double> read_doubles(const char* path) {
  std::vector<double> v;
  if (std::FILE* f = std::fopen(path, "rb")) {
    double d;
    while (std::fread(&d, sizeof d, 1, f) == 1) v.push_back(d);
    std::fclose(f);
  }
  return v;
}

static int postsolve_jobs(std::FILE* out, int argc, char** argv) {
  PresolveResult pr;
  for (int a = 0; a + 2 < argc; a += 3) {
    Model M;
    ModelInfo info;
    std::string err;
    if (!read_model(argv[a], M, info, err)) {
      std::fprintf(stderr, "%s: %s\n", argv[a], err.c_str());
      return 3;
    }
    presolve_into(M, pr);
    if (pr.outcome != PresolveResult::Outcome::Reduced) {
      const long long none[3] = {-1, -1, -1};
      std::fwrite(none, sizeof none[0], 3, out);
      continue;
    }
    Solution red;
    red.status = Status::Optimal;
    red.x = read_doubles(argv[a + 1]);
    red.y = read_doubles(argv[a + 2]);
    Solution s = postsolve(M, pr, red);
    const long long sizes[3] = {static_cast<long long>(s.x.size()), static_cast<long long>(s.y.size()),
                                static_cast<long long>(s.z.size())};
    std::fwrite(sizes, sizeof sizes[0], 3, out);
    std::fwrite(s.x.data(), sizeof(double), s.x.size(), out);
    std::fwrite(s.y.data(), sizeof(double), s.y.size(), out);
    std::fwrite(s.z.data(), sizeof(double), s.z.size(), out);
    std::fwrite(&s.objective, sizeof(double), 1, out);
    pool_vector(std::move(s.x)), pool_vector(std::move(s.y)), pool_vector(std::move(s.z));
  }
  return 0;
}

static int check_jobs(std::FILE* out, int argc, char** argv) {
  for (int a = 0; a + 2 < argc; a += 3) {
    Model M;
    ModelInfo info;
    std::string err;
    if (!read_model(argv[a], M, info, err)) {
      std::fprintf(stderr, "%s: %s\n", argv[a], err.c_str());
      return 3;
    }
    const std::vector<double> x = read_doubles(argv[a + 1]), y = read_doubles(argv[a + 2]);
    const CheckReport r = check_solution(M, x, y);
    const SafeBound b = certified_dual_bound(M, y, true);
    const double rec[7] = {r.passed() ? 1.0 : 0.0, r.max_primal_violation, r.max_dual_violation, r.relative_gap,
                           r.primal_objective, r.dual_objective, b.bound};
    std::fwrite(rec, sizeof(double), 7, out);
  }
  return 0;
}

static int kkt_jobs(std::FILE* out, int argc, char** argv) {
  for (int a = 0; a + 2 < argc; a += 3) {
    Model M;
    ModelInfo info;
    std::string err;
    if (!read_model(argv[a], M, info, err)) {
      std::fprintf(stderr, "%s: %s\n", argv[a], err.c_str());
      return 3;
    }
    const std::vector<double> x = read_doubles(argv[a + 1]), y = read_doubles(argv[a + 2]);
    const OriginalKkt k = original_kkt(M, x, y);
    const double rec[11] = {k.primal_residual, k.dual_residual, k.primal_obj,    k.dual_obj,
                            k.b_norm,          k.c_norm,        k.primal_max_rel, k.dual_max_rel,
                            k.converged(1e-4) ? 1.0 : 0.0, k.converged(1e-8) ? 1.0 : 0.0,
                            k.converged(1e-9) ? 1.0 : 0.0};
    std::fwrite(rec, sizeof(double), 11, out);
  }
  return 0;
}

static int digest_jobs(std::FILE* out, int argc, char** argv) {
  PresolveResult pr;
  for (int a = 0; a < argc; ++a) {
    Model M;
    ModelInfo info;
    std::string err;
    if (!read_model(argv[a], M, info, err)) {
      std::fprintf(stderr, "%s: %s\n", argv[a], err.c_str());
      return 3;
    }
    presolve_into(M, pr);
    std::fprintf(out, "%016llx\n", static_cast<unsigned long long>(presolve_digest(pr)));
  }
  return 0;
}

int main(int argc, char** argv) {
  const std::string cmd = argc > 1 ? argv[1] : "";
  if (cmd == "digest" && argc >= 4) {
    std::FILE* out = std::fopen(argv[2], "w");
    if (!out) return 3;
    const int rc = digest_jobs(out, argc - 3, argv + 3);
    std::fclose(out);
    return rc;
  }
  if (argc < 6 || (argc - 3) % 3 != 0) {
    std::fprintf(stderr, "usage: host_probe digest <out.txt> <model>... | postsolve|check|kkt <out.bin> (<model> <a.bin> <b.bin>)...\n");
    return 2;
  }
  std::FILE* out = std::fopen(argv[2], "wb");
  if (!out) return 3;
  const int rc = cmd == "postsolve" ? postsolve_jobs(out, argc - 3, argv + 3)
                 : cmd == "check"   ? check_jobs(out, argc - 3, argv + 3)
                 : cmd == "kkt"     ? kkt_jobs(out, argc - 3, argv + 3)
                                    : 2;
  std::fclose(out);
  return rc;
}
