// ref_shim.cpp — test infrastructure: a flat extern "C" view of the REFERENCE solver
// (JaiVerma20/ps26119-solver), compiled together with the reference's own sources into
// oracle/_ref/libps26119_ref.so by oracle/Makefile. Nothing in the product links this file;
// only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference legs load it,
// and only as the checker or the timed CPU baseline.
//
// What it exposes (reference file:line it drives):
//   ref_solve        ps26119::solve (src/core/solve.cpp:194) with Options{algorithm=R2hpdhg,
//                    presolve, precision, threads, ...} — the engine-to-engine comparison.
//   ref_batch        ps26119::solve_batch (src/pdhg/batch.cpp:129).
//   ref_scaled_*     pdhg::make_scaled_problem (src/pdhg/scaling.cpp:37) and
//                    la::estimate_norm2 (src/la/csr.cpp:86) — setup parity.
//   ref_backend_*    pdhg::make_cpu_backend() ops (src/pdhg/cpu_backend.cpp:31-215), the
//                    op-by-op comparison that tests/unit/test_gpu.cpp:33-95 performs.
//   ref_check        core::check_solution (src/core/solution_checker.cpp:61) and
//                    certified_dual_bound (src/core/safe_bound.cpp:178); ref_check_file the
//                    same on a model file read by the reference's readers.
//   ref_bound        certified_dual_bound with the implied-bounds switch and its term counts.
//   ref_certificate  check_infeasibility_certificate / check_unboundedness_certificate
//                    (src/core/certificates.cpp:14, 88).
//   ref_presolve_file  the reference reader then ps26119::presolve (src/core/presolve.cpp:22-156)
//                    on a model file: a digest of every presolve decision, in the serialisation
//                    the library's `ps26119 info` prints (outcome, counts, maps, fixed values,
//                    singletons, reduced fingerprint; 8-byte words, FNV-1a).
//   ref_postsolve_file the reference reader, presolve, then postsolve (src/core/presolve.cpp:158-193)
//                    of a given reduced (x, y): the original x, y, z and objective.
//   ref_kkt_file     the presolve wrapper's KKT test of a point on the original model
//                    (original_kkt, src/core/solve.cpp:77-84; pdhg::kkt_general).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "core/certificates.h"
#include "io/lpm_reader.h"
#include "io/mps_reader.h"
#include "core/presolve.h"
#include "core/safe_bound.h"
#include "core/solution_checker.h"
#include "la/csr.h"
#include "pdhg/backend.h"
#include "pdhg/scaling.h"
#include "ps26119/batch.h"
#include "ps26119/solve.h"

using namespace ps26119;

namespace {

Model make_model(int m, int n, int sense, double offset, const double* c, const double* cl, const double* cu,
                 const double* rl, const double* ru, const int* cs, const int* ri, const double* v) {
  Model M;
  M.num_rows = m;
  M.num_cols = n;
  M.sense = sense;
  M.obj_offset = offset;
  M.obj.assign(c, c + n);
  M.col_lower.assign(cl, cl + n);
  M.col_upper.assign(cu, cu + n);
  M.row_lower.assign(rl, rl + m);
  M.row_upper.assign(ru, ru + m);
  M.col_start.assign(cs, cs + n + 1);
  const int nnz = cs[n];
  M.row_index.assign(ri, ri + nnz);
  M.value.assign(v, v + nnz);
  return M;
}

// info layout shared with oracle/reference.py
enum {
  kStatus, kObjective, kDualObjective, kPrimalRes, kDualRes, kGap, kIterations, kSeconds, kSetupSeconds,
  kPrimalWeight, kCertified, kCheck, kItFast, kInfoLen
};

void fill_info(const Solution& s, double* info) {
  info[kStatus] = static_cast<double>(s.status);
  info[kObjective] = s.objective;
  info[kDualObjective] = s.dual_objective;
  info[kPrimalRes] = s.primal_residual;
  info[kDualRes] = s.dual_residual;
  info[kGap] = s.gap;
  info[kIterations] = static_cast<double>(s.iterations);
  info[kSeconds] = s.seconds;
  info[kSetupSeconds] = s.setup_seconds;
  info[kPrimalWeight] = s.primal_weight;
  info[kCertified] = s.certified_bound;
  info[kCheck] = s.check == "PASS" ? 1.0 : (s.check == "FAIL" ? 0.0 : -1.0);
  info[kItFast] = static_cast<double>(s.iterations_to_fast);
}

void copy_out(const std::vector<double>& v, double* dst, std::size_t len) {
  if (dst && v.size() == len) std::memcpy(dst, v.data(), len * sizeof(double));
}

struct RefBackend {
  Model model;
  pdhg::ScaledProblem sp;
  std::unique_ptr<pdhg::Backend> b;
};

}  // namespace

extern "C" {

int ref_info_len(void) { return kInfoLen; }

// Engine-level solve through ps26119::solve. names/values: engine_params (may be 0 long).
int ref_solve(int m, int n, int sense, double offset, const double* c, const double* cl, const double* cu,
              const double* rl, const double* ru, const int* cs, const int* ri, const double* v, int presolve,
              int precision, int threads, double tol, long long iteration_limit, double time_limit, int check_every,
              int n_params, const char* const* names, const double* values, const double* warm_x,
              const double* warm_y, double* x, double* y, double* z, double* dual_ray, double* primal_ray,
              double* info, char* msg, int msglen) {
  const Model M = make_model(m, n, sense, offset, c, cl, cu, rl, ru, cs, ri, v);
  Options o;
  o.algorithm = Algorithm::R2hpdhg;
  o.presolve = presolve != 0;
  o.precision = precision ? Precision::Mixed : Precision::Fp64;
  o.threads = threads;
  if (tol > 0) o.tolerance = tol;
  if (iteration_limit > 0) o.iteration_limit = iteration_limit;
  if (time_limit > 0) o.time_limit = time_limit;
  if (check_every > 0) o.termination_check_every = check_every;
  for (int k = 0; k < n_params; ++k) {
    // "algorithm" (2 = PDLP) and "use_gpu" (the reference's CUDA backend, in the library built
    // with it) are this shim's own switches, not engine parameters
    if (std::string(names[k]) == "algorithm") o.algorithm = values[k] == 2 ? Algorithm::Pdlp : Algorithm::R2hpdhg;
    else if (std::string(names[k]) == "use_gpu") o.use_gpu = values[k] != 0;
    else o.engine_params.emplace_back(names[k], values[k]);
  }
  if (warm_x) o.warm_x.assign(warm_x, warm_x + n);
  if (warm_y) o.warm_y.assign(warm_y, warm_y + m);
  const Solution s = solve(M, o);
  fill_info(s, info);
  copy_out(s.x, x, static_cast<std::size_t>(n));
  copy_out(s.y, y, static_cast<std::size_t>(m));
  copy_out(s.z, z, static_cast<std::size_t>(n));
  copy_out(s.dual_ray, dual_ray, static_cast<std::size_t>(m));
  copy_out(s.primal_ray, primal_ray, static_cast<std::size_t>(n));
  if (msg && msglen > 0) std::snprintf(msg, static_cast<std::size_t>(msglen), "%s", s.message.c_str());
  return static_cast<int>(s.status);
}

// Batched solve over K scenarios sharing A. Scenario vectors are K×n / K×m row-major
// (scenario k at offset k·n); a NULL array means "same as the base" for every scenario.
int ref_batch(int m, int n, int sense, double offset, const double* c, const double* cl, const double* cu,
              const double* rl, const double* ru, const int* cs, const int* ri, const double* v, int K,
              const double* sc_obj, const double* sc_cl, const double* sc_cu, const double* sc_rl,
              const double* sc_ru, int threads, double tol, long long iteration_limit, double* x, double* y,
              double* info) {
  const Model M = make_model(m, n, sense, offset, c, cl, cu, rl, ru, cs, ri, v);
  std::vector<Scenario> sc(static_cast<std::size_t>(K));
  auto take = [](const double* a, int k, int len) {
    return a ? std::vector<double>(a + static_cast<std::size_t>(k) * len, a + static_cast<std::size_t>(k + 1) * len)
             : std::vector<double>();
  };
  for (int k = 0; k < K; ++k) {
    sc[k].obj = take(sc_obj, k, n);
    sc[k].col_lower = take(sc_cl, k, n);
    sc[k].col_upper = take(sc_cu, k, n);
    sc[k].row_lower = take(sc_rl, k, m);
    sc[k].row_upper = take(sc_ru, k, m);
  }
  Options o;
  o.threads = threads;
  if (tol > 0) o.tolerance = tol;
  if (iteration_limit > 0) o.iteration_limit = iteration_limit;
  const auto sols = solve_batch(M, sc, o);
  for (int k = 0; k < K; ++k) {
    fill_info(sols[k], info + static_cast<std::size_t>(k) * kInfoLen);
    if (x) copy_out(sols[k].x, x + static_cast<std::size_t>(k) * n, static_cast<std::size_t>(n));
    if (y) copy_out(sols[k].y, y + static_cast<std::size_t>(k) * m, static_cast<std::size_t>(m));
  }
  return K;
}

// ---------------------------------------------------------------- scaled problem + backend
void* ref_backend_new(int m, int n, int sense, double offset, const double* c, const double* cl, const double* cu,
                      const double* rl, const double* ru, const int* cs, const int* ri, const double* v,
                      int ruiz_iterations, int pock_chambolle, int bound_objective_rescaling,
                      int geometric_mean_iterations, double geometric_mean_min_log10_range) {
  auto* r = new RefBackend;
  r->model = make_model(m, n, sense, offset, c, cl, cu, rl, ru, cs, ri, v);
  pdhg::ScalingOptions so;
  so.ruiz_iterations = ruiz_iterations;
  so.pock_chambolle = pock_chambolle != 0;
  so.bound_objective_rescaling = bound_objective_rescaling != 0;
  so.geometric_mean_iterations = geometric_mean_iterations;
  so.geometric_mean_min_log10_range = geometric_mean_min_log10_range;
  r->sp = pdhg::make_scaled_problem(r->model, so);
  r->b = pdhg::make_cpu_backend();
  r->b->setup(r->sp);
  return r;
}
void ref_backend_free(void* h) { delete static_cast<RefBackend*>(h); }

// Scaled data: which = 0 A(CSR) vals, 1 At(CSR) vals, 2 c, 3 col_lower, 4 col_upper,
// 5 row_lower, 6 row_upper, 7 row_scale, 8 col_scale. Returns the element count.
long long ref_scaled_get(void* h, int which, double* dst) {
  const auto& sp = static_cast<RefBackend*>(h)->sp;
  const std::vector<double>* src = nullptr;
  switch (which) {
    case 0: src = &sp.A.val; break;
    case 1: src = &sp.At.val; break;
    case 2: src = &sp.c; break;
    case 3: src = &sp.col_lower; break;
    case 4: src = &sp.col_upper; break;
    case 5: src = &sp.row_lower; break;
    case 6: src = &sp.row_upper; break;
    case 7: src = &sp.row_scale; break;
    case 8: src = &sp.col_scale; break;
    default: return -1;
  }
  if (dst) std::memcpy(dst, src->data(), src->size() * sizeof(double));
  return static_cast<long long>(src->size());
}
// Structure of A (which=0) or At (which=1) as int32 row_ptr (rows+1) and col (nnz).
long long ref_scaled_structure(void* h, int which, int* row_ptr, int* col) {
  const auto& sp = static_cast<RefBackend*>(h)->sp;
  const la::Csr<double>& M = which == 0 ? sp.A : sp.At;
  if (row_ptr)
    for (int i = 0; i <= M.rows; ++i) row_ptr[i] = static_cast<int>(M.row_ptr[i]);
  if (col) std::memcpy(col, M.col.data(), M.col.size() * sizeof(int));
  return M.nnz();
}
// scalars: [bound_scale, obj_scale, log10_range, geometric_mean_applied]
void ref_scaled_scalars(void* h, double* out) {
  const auto& sp = static_cast<RefBackend*>(h)->sp;
  out[0] = sp.bound_scale;
  out[1] = sp.obj_scale;
  out[2] = sp.log10_range;
  out[3] = sp.geometric_mean_applied ? 1.0 : 0.0;
}
double ref_norm2(void* h) {
  const auto& sp = static_cast<RefBackend*>(h)->sp;
  return la::estimate_norm2(sp.A, sp.At);
}

void ref_backend_set_precision(void* h, int mixed) {
  static_cast<RefBackend*>(h)->b->set_precision(mixed ? Precision::Mixed : Precision::Fp64);
}
int ref_backend_create(void* h, int dual) {
  return static_cast<RefBackend*>(h)->b->create(dual ? pdhg::Space::Dual : pdhg::Space::Primal);
}
void ref_backend_upload(void* h, int v, const double* src, long long len) {
  static_cast<RefBackend*>(h)->b->upload(v, std::vector<double>(src, src + len));
}
void ref_backend_download(void* h, int v, double* dst, long long len) {
  std::vector<double> out;
  static_cast<RefBackend*>(h)->b->download(v, out);
  copy_out(out, dst, static_cast<std::size_t>(len));
}
void ref_backend_fill(void* h, int v, double a) { static_cast<RefBackend*>(h)->b->fill(v, a); }
void ref_backend_copy(void* h, int dst, int src) { static_cast<RefBackend*>(h)->b->copy(dst, src); }
void ref_backend_axpby(void* h, double a, int x, double b, int y) { static_cast<RefBackend*>(h)->b->axpby(a, x, b, y); }
void ref_backend_spmv(void* h, int x, int out) { static_cast<RefBackend*>(h)->b->spmv(x, out); }
void ref_backend_spmv_t(void* h, int y, int out) { static_cast<RefBackend*>(h)->b->spmv_t(y, out); }
double ref_backend_dot(void* h, int a, int b) { return static_cast<RefBackend*>(h)->b->dot(a, b); }
double ref_backend_norm2(void* h, int a) { return static_cast<RefBackend*>(h)->b->norm2(a); }
double ref_backend_diff_norm2(void* h, int a, int b) { return static_cast<RefBackend*>(h)->b->diff_norm2(a, b); }
void ref_backend_primal_step(void* h, int x, int aty, double tau, int xh) {
  static_cast<RefBackend*>(h)->b->primal_step(x, aty, tau, xh);
}
void ref_backend_dual_step(void* h, int y, int ax, double sigma, int yh) {
  static_cast<RefBackend*>(h)->b->dual_step(y, ax, sigma, yh);
}
void ref_backend_r2h_primal(void* h, int x, int x0, int aty, double tau, double w, double rho, int xh, int xb) {
  static_cast<RefBackend*>(h)->b->r2h_primal(x, x0, aty, tau, w, rho, xh, xb);
}
void ref_backend_r2h_dual(void* h, int y, int y0, int ax, double sigma, double w, double rho, int yh, int yb) {
  static_cast<RefBackend*>(h)->b->r2h_dual(y, y0, ax, sigma, w, rho, yh, yb);
}
// KKT: out = [primal_residual, dual_residual, primal_obj, dual_obj, b_norm, c_norm,
//             primal_max_rel, dual_max_rel]
void ref_backend_kkt(void* h, int xs, int ys, double* out) {
  const pdhg::KktStats k = static_cast<RefBackend*>(h)->b->kkt(xs, ys);
  out[0] = k.primal_residual;
  out[1] = k.dual_residual;
  out[2] = k.primal_obj;
  out[3] = k.dual_obj;
  out[4] = k.b_norm;
  out[5] = k.c_norm;
  out[6] = k.primal_max_rel;
  out[7] = k.dual_max_rel;
}

// ---------------------------------------------------------------- verification
// out = [passed, max_primal_violation, max_dual_violation, relative_gap, primal_obj, dual_obj,
//        certified_bound]
void ref_check(int m, int n, int sense, double offset, const double* c, const double* cl, const double* cu,
               const double* rl, const double* ru, const int* cs, const int* ri, const double* v, const double* x,
               const double* y, double* out) {
  const Model M = make_model(m, n, sense, offset, c, cl, cu, rl, ru, cs, ri, v);
  const std::vector<double> xv(x, x + n), yv(y, y + m);
  const CheckReport r = check_solution(M, xv, yv);
  out[0] = r.passed() ? 1.0 : 0.0;
  out[1] = r.max_primal_violation;
  out[2] = r.max_dual_violation;
  out[3] = r.relative_gap;
  out[4] = r.primal_objective;
  out[5] = r.dual_objective;
  out[6] = certified_dual_bound(M, yv, true).bound;
}

// ref_check on the model read from a file by the reference's readers (x: n values, y: m
// values of that model). Returns 1, or 0 when the file does not read.
int ref_check_file(const char* path, const double* x, const double* y, double* out) {
  Model M;
  const std::string p(path);
  std::string err;
  bool ok = false;
  if (p.size() > 4 && p.compare(p.size() - 4, 4, ".lpm") == 0) ok = io::read_lpm(p, M).ok;
  else ok = io::read_mps(p, M, err);
  if (!ok) return 0;
  const std::vector<double> xv(x, x + M.num_cols), yv(y, y + M.num_rows);
  const CheckReport r = check_solution(M, xv, yv);
  out[0] = r.passed() ? 1.0 : 0.0;
  out[1] = r.max_primal_violation;
  out[2] = r.max_dual_violation;
  out[3] = r.relative_gap;
  out[4] = r.primal_objective;
  out[5] = r.dual_objective;
  out[6] = certified_dual_bound(M, yv, true).bound;
  return 1;
}

// The reference's readers: fingerprint of the model read from `path` (.lpm or .mps), dims[3] =
// rows, cols, nnz. Returns 1 on success, 0 on a read error (message in fp).
int ref_read_fingerprint(const char* path, char* fp, int cap, long long* dims) {
  Model m;
  const std::string p(path);
  bool ok = false;
  std::string err;
  if (p.size() > 4 && p.compare(p.size() - 4, 4, ".lpm") == 0) {
    const auto r = io::read_lpm(p, m);
    ok = r.ok;
    err = r.error;
  } else {
    ok = io::read_mps(p, m, err);
  }
  std::snprintf(fp, static_cast<std::size_t>(cap), "%s", ok ? m.fingerprint_hex().c_str() : err.c_str());
  if (ok) dims[0] = m.num_rows, dims[1] = m.num_cols, dims[2] = static_cast<long long>(m.nnz());
  return ok ? 1 : 0;
}

// Digest of a PresolveResult; word order: outcome (0 reduced, 1 infeasible, 2 unchanged),
// removed rows, removed cols, tightened bounds, |row_map| and entries, |col_map| and entries,
// |fixed_value| and values (−0 as +0, NaN canonical), |singletons| and (row, col, a, set_lower,
// set_upper) each, reduced fingerprint (0 unless reduced).
int ref_presolve_file(const char* path, char* out, int cap, long long* counts) {
  Model m;
  const std::string p(path);
  std::string err;
  bool ok = false;
  if (p.size() > 4 && p.compare(p.size() - 4, 4, ".lpm") == 0) {
    const auto r = io::read_lpm(p, m);
    ok = r.ok;
    err = r.error;
  } else {
    ok = io::read_mps(p, m, err);
  }
  if (!ok) {
    std::snprintf(out, static_cast<std::size_t>(cap), "%s", err.c_str());
    return 0;
  }
  const PresolveResult r = presolve(m);
  std::uint64_t h = 0xcbf29ce484222325ULL;
  auto word = [&](std::uint64_t v) {
    for (int k = 0; k < 8; ++k) h ^= (v >> (8 * k)) & 0xffu, h *= 0x100000001b3ULL;
  };
  auto f64 = [&](double v) {
    if (v == 0.0) v = 0.0;
    std::uint64_t bits;
    if (std::isnan(v)) bits = 0x7ff8000000000000ULL;
    else std::memcpy(&bits, &v, sizeof bits);
    word(bits);
  };
  const int oc = r.outcome == PresolveResult::Outcome::Reduced ? 0 : r.outcome == PresolveResult::Outcome::Infeasible ? 1 : 2;
  word(static_cast<std::uint64_t>(oc));
  word(static_cast<std::uint64_t>(r.removed_rows)), word(static_cast<std::uint64_t>(r.removed_cols));
  word(static_cast<std::uint64_t>(r.tightened_bounds));
  word(r.row_map.size());
  for (int i : r.row_map) word(static_cast<std::uint64_t>(static_cast<std::int64_t>(i)));
  word(r.col_map.size());
  for (int j : r.col_map) word(static_cast<std::uint64_t>(static_cast<std::int64_t>(j)));
  word(r.fixed_value.size());
  for (double v : r.fixed_value) f64(v);
  word(r.singletons.size());
  for (const auto& t : r.singletons) {
    word(static_cast<std::uint64_t>(static_cast<std::int64_t>(t.row)));
    word(static_cast<std::uint64_t>(static_cast<std::int64_t>(t.col)));
    f64(t.a);
    word(t.set_lower ? 1u : 0u), word(t.set_upper ? 1u : 0u);
  }
  word(oc == 0 ? r.reduced.fingerprint() : 0);
  std::snprintf(out, static_cast<std::size_t>(cap), "%016llx", static_cast<unsigned long long>(h));
  counts[0] = oc, counts[1] = r.removed_rows, counts[2] = r.removed_cols, counts[3] = r.tightened_bounds;
  return 1;
}

// Reads a model file, presolves it and postsolves the reduced point (red_x: nx values, red_y:
// ny values; a size that does not match the reduced model means "no point", as in the
// reference). x and z hold n values, y m values; sizes[0..2] receive the sizes of x, y and z
// after postsolve (0 for a cleared vector). Returns 1, or 0 when the file does not read or
// presolve does not reduce the model.
int ref_postsolve_file(const char* path, const double* red_x, long long nx, const double* red_y, long long ny,
                       double* x, double* y, double* z, double* objective, long long* sizes) {
  Model m;
  const std::string p(path);
  std::string err;
  bool ok = false;
  if (p.size() > 4 && p.compare(p.size() - 4, 4, ".lpm") == 0) ok = io::read_lpm(p, m).ok;
  else ok = io::read_mps(p, m, err);
  if (!ok) return 0;
  const PresolveResult r = presolve(m);
  if (r.outcome != PresolveResult::Outcome::Reduced) return 0;
  Solution red;
  red.status = Status::Optimal;
  red.x.assign(red_x, red_x + nx);
  red.y.assign(red_y, red_y + ny);
  const Solution s = postsolve(m, r, red);
  std::copy(s.x.begin(), s.x.end(), x);
  std::copy(s.y.begin(), s.y.end(), y);
  std::copy(s.z.begin(), s.z.end(), z);
  *objective = s.objective;
  sizes[0] = static_cast<long long>(s.x.size());
  sizes[1] = static_cast<long long>(s.y.size());
  sizes[2] = static_cast<long long>(s.z.size());
  return 1;
}

// pdhg::kkt_general (src/pdhg/cpu_backend.cpp:225-284) of (x, sense·y) on the model read from a
// file, as original_kkt (src/core/solve.cpp:77-84) forms it: out[8] = primal residual, dual
// residual, primal objective, dual objective, b norm, c norm, primal max rel, dual max rel;
// out[8] = converged(eps). Returns 1, or 0 when the file does not read.
int ref_kkt_file(const char* path, const double* x, const double* y, double eps, double* out) {
  Model M;
  const std::string p(path);
  std::string err;
  bool ok = false;
  if (p.size() > 4 && p.compare(p.size() - 4, 4, ".lpm") == 0) ok = io::read_lpm(p, M).ok;
  else ok = io::read_mps(p, M, err);
  if (!ok) return 0;
  const la::Csr<double> A = la::csr_from_model(M), At = la::csr_transpose_from_model(M);
  const pdhg::LpView lp{M.num_rows, M.num_cols, M.sense, M.obj.data(), M.col_lower.data(), M.col_upper.data(),
                        M.row_lower.data(), M.row_upper.data()};
  std::vector<double> ymin(y, y + M.num_rows);
  for (double& v : ymin) v *= M.sense;
  const pdhg::KktStats k = pdhg::kkt_general(A, At, lp, std::vector<double>(x, x + M.num_cols), ymin);
  const double vals[9] = {k.primal_residual, k.dual_residual, k.primal_obj, k.dual_obj, k.b_norm, k.c_norm,
                          k.primal_max_rel, k.dual_max_rel, k.converged(eps) ? 1.0 : 0.0};
  std::copy(vals, vals + 9, out);
  return 1;
}

// out[4] = finite, bound, unbounded_row_terms, unbounded_col_terms
void ref_bound(int m, int n, int sense, double offset, const double* c, const double* cl, const double* cu,
               const double* rl, const double* ru, const int* cs, const int* ri, const double* v, const double* y,
               int use_implied, double* out) {
  const Model M = make_model(m, n, sense, offset, c, cl, cu, rl, ru, cs, ri, v);
  const SafeBound b = certified_dual_bound(M, std::vector<double>(y, y + m), use_implied != 0);
  out[0] = b.finite ? 1.0 : 0.0;
  out[1] = b.bound;
  out[2] = b.unbounded_row_terms;
  out[3] = b.unbounded_col_terms;
}

// kind 0: infeasibility (ray = m row multipliers); kind 1: unboundedness (x, ray: n each).
// out[5] = present, passed, rigorous, measure, violation
void ref_certificate(int kind, int m, int n, int sense, double offset, const double* c, const double* cl,
                     const double* cu, const double* rl, const double* ru, const int* cs, const int* ri,
                     const double* v, const double* x, const double* ray, double* out) {
  const Model M = make_model(m, n, sense, offset, c, cl, cu, rl, ru, cs, ri, v);
  const CertificateCheck k = kind == 0 ? check_infeasibility_certificate(M, std::vector<double>(ray, ray + m))
                                       : check_unboundedness_certificate(M, std::vector<double>(x, x + n),
                                                                         std::vector<double>(ray, ray + n));
  out[0] = k.present, out[1] = k.passed, out[2] = k.rigorous, out[3] = k.measure, out[4] = k.violation;
}

}  // extern "C"
