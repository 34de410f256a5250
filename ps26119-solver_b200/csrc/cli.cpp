// cli.cpp — the ps26119 command-line tool on the GPU engines (≙ the reference's apps/cli/main.cpp
// for the commands this library covers):
//
//   ps26119 --version
//   ps26119 info  <file.mps|file.lpm>...
//   ps26119 convert <file.mps|file.lpm> <out.lpm>
//   ps26119 solve <file.mps|file.lpm> [--algorithm auto|r2hpdhg|pdlp] [--precision fp64|mixed] [--gpu]
//                 [--tol e] [--time-limit s] [--iteration-limit n] [--no-presolve] [--exact]
//                 [--out file.sol] [-v|-vv]
//   ps26119 batch <base> <scenario>... [--out-dir d] [--tol e] [--time-limit s] [--iteration-limit n]
//
// Every solve runs on the GPU (--gpu is accepted for compatibility and implied).
// Exit codes as the reference's: 0 optimal, 1 infeasible / unbounded / limit, 2 usage,
// 3 read error, 4 cannot write the output, 5 numerical error / not solved.
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "io.hpp"
#include "solver.hpp"

using namespace b200;

namespace {

constexpr int kExitUsage = 2, kExitRead = 3, kExitWrite = 4;

void usage(std::FILE* f) {
  std::fprintf(f,
               "ps26119 (B200 engines) — LP solver on the GPU\n"
               "usage:\n"
               "  ps26119 --version\n"
               "  ps26119 info  <file.mps|file.lpm>...\n"
               "  ps26119 convert <file.mps|file.lpm> <out.lpm>\n"
               "  ps26119 solve <file.mps|file.lpm> [options]\n"
               "  ps26119 batch <base> <scenario>... [--out-dir d] [--tol e] [--time-limit s] [--iteration-limit n]\n"
               "solve options:\n"
               "  --algorithm auto|r2hpdhg|pdlp    (default auto = r2hpdhg)\n"
               "  --precision fp64|mixed\n"
               "  --gpu                             accepted; every solve runs on the GPU\n"
               "  --tol <eps>  --time-limit <s>  --iteration-limit <n>\n"
               "  --no-presolve                     skip the safe presolve + postsolve\n"
               "  --exact                           take every sum in the reference's order\n"
               "  --out <file>                      write the solution file\n"
               "  -v | -vv                          verbosity\n"
               "exit codes: 0 optimal, 1 infeasible/unbounded/limit, 2 usage, 3 read error,\n"
               "            4 cannot write output, 5 numerical error / not solved\n");
}

int exit_code(Status s) {
  switch (s) {
    case Status::Optimal: return 0;
    case Status::Infeasible:
    case Status::Unbounded:
    case Status::IterationLimit:
    case Status::TimeLimit: return 1;
    default: return 5;
  }
}

double number_arg(const char* flag, const char* s) {
  char* end = nullptr;
  const double v = std::strtod(s, &end);
  if (end == s || *end != '\0' || !std::isfinite(v) || !(v > 0)) {
    std::fprintf(stderr, "%s needs a positive number, got '%s'\n", flag, s);
    std::exit(kExitUsage);
  }
  return v;
}

// Whether the solution file can be written, checked before a long solve rather than after it:
// an existing file must be writable in place; a new one must be creatable in its directory.
bool writable(const std::string& path) {
  struct stat st;
  if (::stat(path.c_str(), &st) == 0) return !S_ISDIR(st.st_mode) && ::access(path.c_str(), W_OK) == 0;
  const std::size_t slash = path.find_last_of('/');
  const std::string dir = slash == std::string::npos ? "." : (slash == 0 ? "/" : path.substr(0, slash));
  return ::access(dir.c_str(), W_OK | X_OK) == 0;
}

bool load(const std::string& path, Model& m, ModelInfo& info) {
  std::string err;
  if (!read_model(path, m, info, err)) {
    std::fprintf(stderr, "read error: %s\n", err.c_str());
    return false;
  }
  for (const auto& w : info.warnings) std::fprintf(stderr, "reader warning: %s\n", w.c_str());
  return true;
}

// One file's summary. `r` is reused from file to file the way the solve path reuses its
// presolve result on a thread, so a digest printed here is the one a repeated solve sees.
int info_one(const char* path, PresolveResult& r) {
  Model m;
  ModelInfo info;
  if (!load(path, m, info)) return kExitRead;
  int eq = 0, ranged = 0, free_rows = 0, fixed = 0, boxed = 0, free_cols = 0, ints = 0;
  for (int i = 0; i < m.num_rows; ++i) {
    const double lo = m.row_lower[i], up = m.row_upper[i];
    if (lo == up) ++eq;
    else if (std::isfinite(lo) && std::isfinite(up)) ++ranged;
    else if (!std::isfinite(lo) && !std::isfinite(up)) ++free_rows;
  }
  for (int j = 0; j < m.num_cols; ++j) {
    const double lo = m.col_lower[j], up = m.col_upper[j];
    if (lo == up) ++fixed;
    else if (std::isfinite(lo) && std::isfinite(up)) ++boxed;
    else if (!std::isfinite(lo) && !std::isfinite(up)) ++free_cols;
    if (j < static_cast<int>(info.is_integer.size()) && info.is_integer[j]) ++ints;
  }
  std::printf("model              %s\n", info.name.c_str());
  std::printf("  sense              %s\n", m.sense > 0 ? "minimise" : "maximise");
  std::printf("  rows               %d  (equality %d, ranged %d, free %d)\n", m.num_rows, eq, ranged, free_rows);
  std::printf("  columns            %d  (fixed %d, boxed %d, free %d, integer %d)\n", m.num_cols, fixed, boxed,
              free_cols, ints);
  std::printf("  nonzeros           %zu\n", m.nnz());
  std::printf("  fingerprint        %s\n", fingerprint_hex(m).c_str());
  if (auto c = m.crossed_bounds(); !c.empty()) {
    std::printf("  note               %s (infeasible)\n", c.c_str());
    return 0;
  }
  // what the safe presolve (R1-R4) would do, and a digest of all its decisions
  if (m.validate().empty()) {
    const auto t0 = std::chrono::steady_clock::now();
    presolve_into(m, r);
    const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    const char* what = r.outcome == PresolveResult::Outcome::Reduced      ? "reduced"
                       : r.outcome == PresolveResult::Outcome::Infeasible ? "infeasible"
                                                                           : "unchanged";
    std::printf("  presolve           %s: removed %d rows, %d columns, %d bounds tightened\n", what, r.removed_rows,
                r.removed_cols, r.tightened_bounds);
    if (r.outcome == PresolveResult::Outcome::Reduced)
      std::printf("  reduced            %d rows, %d columns, %zu nonzeros\n", r.reduced.num_rows, r.reduced.num_cols,
                  r.reduced.nnz());
    std::printf("  presolve digest    %016llx\n", static_cast<unsigned long long>(presolve_digest(r)));
    std::printf("  presolve time      %.1f ms\n", ms);
  }
  return 0;
}

int cmd_info(int argc, char** argv) {
  if (argc < 1) {
    usage(stderr);
    return kExitUsage;
  }
  PresolveResult r;
  for (int k = 0; k < argc; ++k)
    if (const int rc = info_one(argv[k], r)) return rc;
  return 0;
}

int cmd_solve(int argc, char** argv) {
  std::string path, out;
  Options opt;
  opt.use_gpu = true;
  for (int i = 0; i < argc; ++i) {
    const std::string a = argv[i];
    auto next = [&]() -> const char* {
      if (i + 1 >= argc) {
        std::fprintf(stderr, "missing value for %s\n", a.c_str());
        std::exit(kExitUsage);
      }
      return argv[++i];
    };
    if (a == "--algorithm") {
      const std::string v = next();
      if (v == "auto") opt.algorithm = Algorithm::Auto;
      else if (v == "r2hpdhg") opt.algorithm = Algorithm::R2hpdhg;
      else if (v == "pdlp") opt.algorithm = Algorithm::Pdlp;
      else {
        std::fprintf(stderr, "unknown or unsupported algorithm '%s' (auto, r2hpdhg, pdlp)\n", v.c_str());
        return kExitUsage;
      }
    } else if (a == "--precision") {
      const std::string v = next();
      if (v == "fp64") opt.precision = Precision::Fp64;
      else if (v == "mixed") opt.precision = Precision::Mixed;
      else {
        std::fprintf(stderr, "unknown precision '%s'\n", v.c_str());
        return kExitUsage;
      }
    } else if (a == "--gpu") {
      opt.use_gpu = true;
    } else if (a == "--tol") {
      opt.tolerance = number_arg("--tol", next());
    } else if (a == "--time-limit") {
      opt.time_limit = number_arg("--time-limit", next());
    } else if (a == "--iteration-limit") {
      opt.iteration_limit = static_cast<long long>(number_arg("--iteration-limit", next()));
    } else if (a == "--no-presolve") {
      opt.presolve = false;
    } else if (a == "--presolve") {
      opt.presolve = true;
    } else if (a == "--exact") {
      opt.exact = true;
    } else if (a == "--threads") {
      (void)next();  // host threads are chosen by the library
    } else if (a == "--out") {
      out = next();
    } else if (a == "-v") {
      opt.verbosity = 1;
    } else if (a == "-vv") {
      opt.verbosity = 2;
    } else if (!a.empty() && a[0] == '-') {
      std::fprintf(stderr, "unknown option %s\n", a.c_str());
      return kExitUsage;
    } else if (path.empty()) {
      path = a;
    } else {
      std::fprintf(stderr, "more than one input file\n");
      return kExitUsage;
    }
  }
  if (path.empty()) {
    usage(stderr);
    return kExitUsage;
  }
  if (!out.empty() && !writable(out)) {
    std::fprintf(stderr, "cannot write the solution file '%s'\n", out.c_str());
    return kExitWrite;
  }
  Model m;
  ModelInfo info;
  if (!load(path, m, info)) return kExitRead;
  Solution s = solve(m, opt);
  if (info.has_integers())
    s.message = std::string("LP relaxation (integrality ignored)") + (s.message.empty() ? "" : "; ") + s.message;
  s.model_fingerprint = fingerprint_hex(m);
  std::printf("model      %s  rows %d  cols %d  nnz %zu  fingerprint %s\n", info.name.c_str(), m.num_rows, m.num_cols,
              m.nnz(), s.model_fingerprint.c_str());
  std::printf("status     %s\n", status_name(s.status));
  std::printf("engine     %s (%s)\n", s.engine.c_str(), s.precision.c_str());
  std::printf("objective  %.12g\n", s.objective);
  std::printf("residuals  primal %.2e  dual %.2e  gap %.2e\n", s.primal_residual, s.dual_residual, s.gap);
  const bool claim = s.status == Status::Infeasible || s.status == Status::Unbounded;
  if (claim)
    std::printf("check      %s\n", s.check.empty() ? "NOT CERTIFIED (no certificate)"
                                                  : (s.check + "  (" + (s.status == Status::Infeasible ? "Farkas" : "ray") +
                                                     " certificate verified on the original model)").c_str());
  else if (!s.check.empty())
    std::printf("check      %s  (in-process, original model: primal %.1e  dual %.1e  gap %.1e)\n", s.check.c_str(),
                s.check_primal, s.check_dual, s.check_gap);
  if (s.certified_bound == s.certified_bound && !claim) {
    if (std::isfinite(s.certified_bound))
      std::printf("certified  %s %.12g  (rounding-proof %s bound from y)\n", m.sense > 0 ? "optimum >=" : "optimum <=",
                  s.certified_bound, m.sense > 0 ? "lower" : "upper");
    else
      std::printf("certified  none  (y gives no finite rounding-proof bound)\n");
  }
  std::printf("iterations %lld   seconds %.3f   (setup %.3f)\n", s.iterations, s.seconds, s.setup_seconds);
  if (!s.message.empty()) std::printf("message    %s\n", s.message.c_str());
  if (!out.empty()) {
    std::string err;
    if (!write_solution(out, m, info, s, err)) {
      std::fprintf(stderr, "%s\n", err.c_str());
      return kExitWrite;
    }
  }
  return exit_code(s.status);
}

int cmd_batch(int argc, char** argv) {
  std::string out_dir;
  Options opt;
  opt.use_gpu = true;
  std::vector<std::string> files;
  for (int i = 0; i < argc; ++i) {
    const std::string a = argv[i];
    auto next = [&]() -> const char* {
      if (i + 1 >= argc) {
        std::fprintf(stderr, "missing value for %s\n", a.c_str());
        std::exit(kExitUsage);
      }
      return argv[++i];
    };
    if (a == "--out-dir") out_dir = next();
    else if (a == "--tol") opt.tolerance = number_arg("--tol", next());
    else if (a == "--time-limit") opt.time_limit = number_arg("--time-limit", next());
    else if (a == "--iteration-limit") opt.iteration_limit = static_cast<long long>(number_arg("--iteration-limit", next()));
    else if (a == "--threads") (void)next();
    else if (a == "--exact") opt.exact = true;
    else if (a == "-v") opt.verbosity = 1;
    else if (a == "-vv") opt.verbosity = 2;
    else if (!a.empty() && a[0] == '-') {
      std::fprintf(stderr, "unknown option %s\n", a.c_str());
      return kExitUsage;
    } else {
      files.push_back(a);
    }
  }
  if (files.size() < 2) {
    usage(stderr);
    return kExitUsage;
  }
  Model base;
  ModelInfo base_info;
  if (!load(files[0], base, base_info)) return kExitRead;
  std::vector<Scenario> sc;
  std::vector<std::string> names, model_names;
  for (std::size_t f = 1; f < files.size(); ++f) {  // main.cpp:399-416: a shared matrix is required
    Model s;
    ModelInfo si;
    if (!load(files[f], s, si)) return kExitRead;
    if (s.num_rows != base.num_rows || s.num_cols != base.num_cols || s.sense != base.sense ||
        s.col_start != base.col_start || s.row_index != base.row_index || s.value != base.value) {
      std::fprintf(stderr, "%s: matrix or sense differs from the base model (batch needs a shared A)\n",
                   files[f].c_str());
      return kExitUsage;
    }
    sc.push_back(Scenario{s.obj, s.col_lower, s.col_upper, s.row_lower, s.row_upper});
    const auto slash = files[f].find_last_of('/');
    std::string nm = files[f].substr(slash == std::string::npos ? 0 : slash + 1);
    names.push_back(nm.substr(0, nm.rfind('.')));
    model_names.push_back(si.name);
  }
  const std::vector<Solution> sols = solve_batch(base, sc, opt);
  int worst = 0;
  for (std::size_t k = 0; k < sols.size(); ++k) {
    const Solution& s = sols[k];
    std::printf("%-28s %-14s obj %.12g  it %lld  t %.3fs%s%s\n", names[k].c_str(), status_name(s.status), s.objective,
                s.iterations, s.seconds, s.message.empty() ? "" : "  ", s.message.c_str());
    worst = std::max(worst, exit_code(s.status));
    if (!out_dir.empty()) {
      ModelInfo info = base_info;
      info.name = model_names[k];
      std::string err;
      if (!write_solution(out_dir + "/" + names[k] + ".sol", base, info, s, err)) {
        std::fprintf(stderr, "%s\n", err.c_str());
        worst = std::max(worst, kExitWrite);
      }
    }
  }
  return worst;
}

}  // namespace

int main(int argc, char** argv) {
  try {
    if (argc < 2) {
      usage(stderr);
      return kExitUsage;
    }
    const std::string cmd = argv[1];
    if (cmd == "--version") {
      std::printf("ps26119 0.1.0+b200\n");
      return 0;
    }
    if (cmd == "--help" || cmd == "-h") {
      usage(stdout);
      return 0;
    }
    if (cmd == "info") return cmd_info(argc - 2, argv + 2);
    if (cmd == "convert") {  // convert <in.mps|in.lpm> <out.lpm>
      if (argc != 4) {
        usage(stderr);
        return kExitUsage;
      }
      Model m;
      ModelInfo info;
      if (!load(argv[2], m, info)) return kExitRead;
      std::string err;
      if (!write_lpm(argv[3], m, info, err)) {
        std::fprintf(stderr, "%s\n", err.c_str());
        return kExitWrite;
      }
      return 0;
    }
    if (cmd == "solve") return cmd_solve(argc - 2, argv + 2);
    if (cmd == "batch") return cmd_batch(argc - 2, argv + 2);
    std::fprintf(stderr, "unknown command %s\n", cmd.c_str());
    usage(stderr);
    return kExitUsage;
  } catch (const std::bad_alloc&) {
    std::fprintf(stderr, "fatal: out of memory\n");
  } catch (const std::exception& e) {
    std::fprintf(stderr, "fatal: %s\n", e.what());
  }
  return 5;
}
