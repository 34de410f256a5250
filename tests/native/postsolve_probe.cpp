// postsolve_probe.cpp — test driver: the library's presolve and postsolve on model files, for
// the bitwise comparison with the reference's postsolve in tests/test_presolve.py. It links the
// library's host objects (solver, certify, io); the GPU entry points those objects reference
// are defined below as stubs that are never called (no solve runs here).
//
//   postsolve_probe <out.bin> (<model> <red_x.bin> <red_y.bin>)...
//
// One presolve result and the solution vectors are reused from job to job, as repeated solves
// on one thread reuse them. For each job out.bin receives the sizes of x, y and z (int64 each),
// then x, y, z and the objective (float64); a job whose model presolve does not reduce writes
// three sizes of -1 and nothing else.
#include <cstdio>
#include <stdexcept>
#include <string>
#include <vector>

#include "batch.hpp"
#include "io.hpp"
#include "solver.hpp"

namespace b200 {
EngineResult run_engine_host(const HostModelView&, const EngineOptions&, HostOutputs&) {
  throw std::runtime_error("no engine in the postsolve probe");
}
const char* status_name(Status) { return "?"; }
void require_device() {}
std::vector<BatchOutcome> run_batch_host(const HostModelView&, const std::vector<BatchScenarioView>&,
                                         const std::vector<int>&, const EngineOptions&,
                                         std::chrono::steady_clock::time_point) {
  throw std::runtime_error("no engine in the postsolve probe");
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

int main(int argc, char** argv) {
  if (argc < 5 || (argc - 2) % 3 != 0) {
    std::fprintf(stderr, "usage: postsolve_probe <out.bin> (<model> <red_x.bin> <red_y.bin>)...\n");
    return 2;
  }
  std::FILE* out = std::fopen(argv[1], "wb");
  if (!out) return 3;
  PresolveResult pr;
  for (int a = 2; a + 2 < argc; a += 3) {
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
  std::fclose(out);
  return 0;
}
