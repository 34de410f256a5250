// solver.cpp — model contract, presolve/postsolve, in-process check and the solve()
// dispatcher around the GPU engine. Each function follows the reference function named in
// its comment (file:line in the reference project); the engine itself runs on the GPU.
#include "solver.hpp"
#include "batch.hpp"
#include "certify.hpp"
#include "parallel.hpp"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <new>
#include <sstream>
#include <stdexcept>
#include <thread>

namespace b200 {

// ============================================================ Model (model.cpp)
std::string Model::validate() const {  // model.cpp:93-151
  std::ostringstream err;
  const auto n = static_cast<std::size_t>(num_cols);
  const auto m = static_cast<std::size_t>(num_rows);
  if (num_rows < 0 || num_cols < 0) return "negative dimension";
  if (sense != 1 && sense != -1) return "sense must be +1 or -1";
  if (!std::isfinite(obj_offset)) return "obj_offset is not finite";
  if (obj.size() != n) return "obj has wrong size";
  if (col_lower.size() != n || col_upper.size() != n) return "column bounds have wrong size";
  if (row_lower.size() != m || row_upper.size() != m) return "row bounds have wrong size";
  if (col_start.size() != n + 1) return "col_start must have num_cols+1 entries";
  if (col_start[0] != 0) return "col_start[0] must be 0";
  if (row_index.size() != value.size()) return "row_index and value differ in size";
  if (static_cast<std::size_t>(col_start[n]) != value.size()) return "col_start[n] != nnz";
  // Columns are checked in parallel ranges; each range reports its first failing column and the
  // smallest such column's message is returned, the same message a sequential scan gives. The
  // column pointers are scanned first: the parallel pass covers only the columns before the first
  // one whose pointers decrease or pass nnz, so no range reads outside the entry arrays.
  const std::size_t nnz = value.size();
  std::size_t lim = n;
  for (std::size_t j = 0; j < n; ++j)
    if (col_start[j + 1] < col_start[j] || static_cast<std::size_t>(col_start[j + 1]) > nnz) {
      lim = j;
      break;
    }
  // A column whose row indices are in range, strictly increasing and whose values are finite has
  // no error: that is checked with sequential reads only. Any other column is examined by the
  // entry-by-entry rules (first error in entry order), with a row-stamp array for duplicates.
  auto column_error = [&](std::size_t j, std::vector<int>& seen) -> std::string {
    if (!std::isfinite(obj[j])) return "objective coefficient of column " + std::to_string(j) + " is not finite";
    bool clean = true;
    int prev = -1;
    for (int k = col_start[j]; k < col_start[j + 1] && clean; ++k) {
      const int i = row_index[k];
      clean = i > prev && static_cast<std::size_t>(i) < m && std::isfinite(value[k]);
      prev = i;
    }
    if (clean) return std::string();
    if (seen.empty()) seen.assign(m, -1);
    for (int k = col_start[j]; k < col_start[j + 1]; ++k) {
      const int i = row_index[k];
      if (i < 0 || static_cast<std::size_t>(i) >= m) return "row index out of range in column " + std::to_string(j);
      if (seen[i] == static_cast<int>(j))
        return "duplicate entry (" + std::to_string(i) + "," + std::to_string(j) + ")";
      seen[i] = static_cast<int>(j);
      if (!std::isfinite(value[k]))
        return "matrix entry (" + std::to_string(i) + "," + std::to_string(j) + ") is not finite";
    }
    return std::string();
  };
  std::vector<std::pair<std::size_t, std::string>> first;  // (column, message), one per failing range
  std::mutex mu;
  parallel_ranges(static_cast<long long>(lim), [&](long long jb, long long je) {
    std::vector<int> seen;
    for (long long j = jb; j < je; ++j) {
      std::string e = column_error(static_cast<std::size_t>(j), seen);
      if (!e.empty()) {
        std::lock_guard<std::mutex> lock(mu);
        first.emplace_back(static_cast<std::size_t>(j), std::move(e));
        return;
      }
    }
  });
  if (!first.empty()) return std::min_element(first.begin(), first.end())->second;
  if (lim < n) {  // the first column whose pointers decrease (one exists after a pointer past nnz)
    for (std::size_t j = lim; j < n; ++j)
      if (col_start[j + 1] < col_start[j]) {
        err << "col_start not monotone at column " << j;
        return err.str();
      }
  }
  auto check_bounds = [&](const std::vector<double>& lo, const std::vector<double>& up, const char* what) {
    for (std::size_t k = 0; k < lo.size(); ++k) {
      const bool nan = std::isnan(lo[k]) || std::isnan(up[k]);
      if (!nan && lo[k] != kInf && up[k] != -kInf) continue;  // the common case builds no message
      std::ostringstream e;
      if (nan) e << what << " bound " << k << " is NaN";
      else if (lo[k] == kInf) e << what << " lower bound " << k << " is +inf";
      else e << what << " upper bound " << k << " is -inf";
      return e.str();
    }
    return std::string();
  };
  if (auto s = check_bounds(col_lower, col_upper, "column"); !s.empty()) return s;
  return check_bounds(row_lower, row_upper, "row");
}

std::string Model::crossed_bounds() const {  // model.cpp:153-167
  auto first = [](const std::vector<double>& lo, const std::vector<double>& up, const char* what) {
    for (std::size_t k = 0; k < lo.size() && k < up.size(); ++k)
      if (lo[k] > up[k]) {
        std::ostringstream e;
        e << what << " " << k << " has lower bound " << lo[k] << " > upper bound " << up[k];
        return e.str();
      }
    return std::string();
  };
  if (auto s = first(col_lower, col_upper, "column"); !s.empty()) return s;
  return first(row_lower, row_upper, "row");
}

double Model::objective_value(const std::vector<double>& x) const {  // model.cpp:169-173
  double v = obj_offset;
  for (int j = 0; j < num_cols; ++j) v += obj[j] * x[j];
  return v;
}

namespace {
// The host threads a pass may use (as parallel_ranges).
int host_threads() { return host_thread_limit(); }
// Host threads for an O(nnz) pass over a model with `nnz` entries (one below 2^18 entries).
int pass_threads(long long nnz) { return nnz < (1LL << 18) ? 1 : host_threads(); }

// Groups the entries of the column-major matrix by block of 2^kRowShift rows, for passes that
// update rows without atomics. Chunk c (one per thread) is the column range [n·c/T, n·(c+1)/T).
// Every entry gets a slot; the slots of block b are [start[b], start[b+1]), and inside a block
// chunk 0's entries come first, then chunk 1's, and so on, each chunk's in column order. So the
// entries of any one row are in increasing column order, the order of a sequential column-major
// pass. place(q, i, j, k) is called once for entry k (row i, column j) with its slot q, on the
// thread of the entry's chunk.
constexpr int kRowShift = 14;  // 16,384 rows: a block's rows fit in one core's cache
// Bucketing holds 8-12 bytes per entry; above this many entries the passes that use it fall
// back to forms without scratch (atomics, or one sequential pass). The tests build a copy with
// a small limit to run those forms on small models.
#ifndef PS26119_BUCKET_MAX_ENTRIES
#define PS26119_BUCKET_MAX_ENTRIES (1LL << 28)
#endif
constexpr long long kBucketMaxEntries = PS26119_BUCKET_MAX_ENTRIES;
template <class Place>
void bucket_rows(const Model& M, int T, std::vector<long long>& start, Place place) {
  const int m = M.num_rows, n = M.num_cols;
  const int nb = (m >> kRowShift) + 1;
  std::vector<long long> at(static_cast<std::size_t>(T) * nb, 0);  // chunk c's next slot in block b: at[c·nb + b]
  auto cols = [&](long long c, int& jb, int& je) {
    jb = static_cast<int>(static_cast<long long>(n) * c / T), je = static_cast<int>(static_cast<long long>(n) * (c + 1) / T);
  };
  parallel_ranges(
      T,
      [&](long long cb, long long ce) {
        for (long long c = cb; c < ce; ++c) {
          int jb, je;
          cols(c, jb, je);
          long long* h = &at[static_cast<std::size_t>(c) * nb];
          for (int k = M.col_start[jb]; k < M.col_start[je]; ++k) ++h[M.row_index[k] >> kRowShift];
        }
      },
      1);
  start.assign(static_cast<std::size_t>(nb) + 1, 0);
  long long pos = 0;  // blocks in order, and inside a block the chunks in order
  for (int b = 0; b < nb; ++b) {
    start[b] = pos;
    for (int c = 0; c < T; ++c) {
      const long long cnt = at[static_cast<std::size_t>(c) * nb + b];
      at[static_cast<std::size_t>(c) * nb + b] = pos;
      pos += cnt;
    }
  }
  start[nb] = pos;
  parallel_ranges(
      T,
      [&](long long cb, long long ce) {
        for (long long c = cb; c < ce; ++c) {
          int jb, je;
          cols(c, jb, je);
          long long* h = &at[static_cast<std::size_t>(c) * nb];
          for (int j = jb; j < je; ++j)
            for (int k = M.col_start[j]; k < M.col_start[j + 1]; ++k) {
              const int i = M.row_index[k];
              place(h[i >> kRowShift]++, i, j, k);
            }
        }
      },
      1);
}

// The bucketed entries of row_activity (row, product), kept per thread between calls within the
// host reuse limit.
struct ActivityScratch {
  std::vector<int> row;
  std::vector<double> prod;
  std::size_t accounted = 0;
  ~ActivityScratch() { host_keep(accounted, 0); }
};
thread_local ActivityScratch t_activity;
}  // namespace

std::vector<double> Model::row_activity(const std::vector<double>& x) const {  // model.cpp:175-180
  std::vector<double> ax = pooled_vector(static_cast<std::size_t>(num_rows));  // zeros
  const int T = pass_threads(static_cast<long long>(nnz()));
  if (T == 1 || static_cast<long long>(nnz()) > kBucketMaxEntries) {
    for (int j = 0; j < num_cols; ++j)
      for (int k = col_start[j]; k < col_start[j + 1]; ++k) ax[row_index[k]] += value[k] * x[j];
    return ax;
  }
  // Each product is formed as in the sequential pass, and each row adds its products in
  // increasing column order (bucket_rows), so every ax[i] has the sequential pass's bits.
  ActivityScratch& S = t_activity;
  struct Keep {
    ActivityScratch& s;
    ~Keep() {
      if (!host_keep(s.accounted, 4 * s.row.capacity() + 8 * s.prod.capacity()))
        std::vector<int>().swap(s.row), std::vector<double>().swap(s.prod);
    }
  } keep{S};
  size_for_copy(S.row, nnz()), size_for_copy(S.prod, nnz());
  std::vector<long long> start;
  bucket_rows(*this, T, start, [&](long long q, int i, int j, int k) {
    S.row[q] = i;
    S.prod[q] = value[k] * x[j];
  });
  parallel_ranges(
      static_cast<long long>(start.size()) - 1,
      [&](long long bb, long long be) {
        for (long long q = start[bb]; q < start[be]; ++q) ax[S.row[q]] += S.prod[q];
      },
      1);
  return ax;
}

namespace {
// FNV-1a over a byte stream, continued from state h.
std::uint64_t fnv1a(std::uint64_t h, const std::vector<unsigned char>& bytes) {
  for (unsigned char c : bytes) h ^= c, h *= 0x100000001b3ULL;
  return h;
}
constexpr std::uint64_t kFnvOffset = 0xcbf29ce484222325ULL;

// The canonical byte stream a fingerprint hashes (model.cpp:20-85): integers and doubles as
// 8-byte little-endian words, −0 as +0, every NaN as the one quiet NaN.
struct CanonicalBytes {
  std::vector<unsigned char> buf;
  void word(std::uint64_t v) {
    const auto* b = reinterpret_cast<const unsigned char*>(&v);
    buf.insert(buf.end(), b, b + sizeof v);
  }
  void i64(std::int64_t v) { word(static_cast<std::uint64_t>(v)); }
  void f64(double v) {
    if (v == 0.0) v = 0.0;
    std::uint64_t bits;
    if (std::isnan(v)) bits = 0x7ff8000000000000ULL;
    else std::memcpy(&bits, &v, sizeof bits);
    word(bits);
  }
  void f64s(const std::vector<double>& v) {
    word(v.size());
    for (double d : v) f64(d);
  }
};

// Dimensions, sense, offset and the five vectors.
void canonical_head(const Model& M, const std::vector<double>& obj, const std::vector<double>& cl,
                    const std::vector<double>& cu, const std::vector<double>& rl, const std::vector<double>& ru,
                    CanonicalBytes& out) {
  out.i64(M.num_rows), out.i64(M.num_cols), out.i64(M.sense), out.f64(M.obj_offset);
  out.f64s(obj), out.f64s(cl), out.f64s(cu), out.f64s(rl), out.f64s(ru);
}
// The matrix (each column's entries in row order) and the integrality flags.
void canonical_tail(const Model& M, CanonicalBytes& out) {
  out.word(M.value.size());
  out.buf.reserve(out.buf.size() + 16 * M.value.size() + 16 * static_cast<std::size_t>(M.num_cols) + 16);
  std::vector<std::pair<int, double>> col;
  for (int j = 0; j < M.num_cols; ++j) {
    col.clear();
    for (int k = M.col_start[j]; k < M.col_start[j + 1]; ++k) col.emplace_back(M.row_index[k], M.value[k]);
    std::sort(col.begin(), col.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
    out.i64(static_cast<std::int64_t>(col.size()));
    for (const auto& [i, v] : col) out.i64(i), out.f64(v);
  }
  for (int j = 0; j < M.num_cols; ++j) out.i64(j < static_cast<int>(M.is_integer.size()) && M.is_integer[j] ? 1 : 0);
}
}  // namespace

std::uint64_t Model::fingerprint() const {  // model.cpp:20-85: FNV-1a over the canonical numbers
  CanonicalBytes head, tail;
  canonical_head(*this, obj, col_lower, col_upper, row_lower, row_upper, head);
  canonical_tail(*this, tail);
  return fnv1a(fnv1a(kFnvOffset, head.buf), tail.buf);
}

// Fingerprints of the base model with each scenario's vectors (an empty vector keeps the
// base's): the matrix part of the byte stream is built once, the scenarios are hashed on the
// host's threads.
std::vector<std::uint64_t> scenario_fingerprints(const Model& base, const std::vector<Scenario>& scenarios) {
  CanonicalBytes tail;
  canonical_tail(base, tail);
  std::vector<std::uint64_t> out(scenarios.size());
  parallel_ranges(static_cast<long long>(scenarios.size()), [&](long long kb, long long ke) {
    for (long long k = kb; k < ke; ++k) {
      const Scenario& s = scenarios[static_cast<std::size_t>(k)];
      auto pick = [](const std::vector<double>& v, const std::vector<double>& d) -> const std::vector<double>& {
        return v.empty() ? d : v;
      };
      CanonicalBytes head;
      canonical_head(base, pick(s.obj, base.obj), pick(s.col_lower, base.col_lower), pick(s.col_upper, base.col_upper),
                     pick(s.row_lower, base.row_lower), pick(s.row_upper, base.row_upper), head);
      out[static_cast<std::size_t>(k)] = fnv1a(fnv1a(kFnvOffset, head.buf), tail.buf);
    }
  }, 2);
  return out;
}

HostModelView Model::view() const {
  HostModelView v;
  v.m = num_rows, v.n = num_cols, v.sense = sense, v.offset = obj_offset;
  v.c = obj.data(), v.col_lower = col_lower.data(), v.col_upper = col_upper.data();
  v.row_lower = row_lower.data(), v.row_upper = row_upper.data();
  v.col_start = col_start.data(), v.row_index = row_index.data(), v.value = value.data();
  return v;
}

// ============================================================ check (solution_checker.cpp)
namespace {
std::vector<double> pooled_storage(std::size_t n);  // defined with the vector pool below

struct DualTerm {
  double violation, contribution, complementarity;
};
DualTerm evaluate_multiplier(double mult, double lo, double up, double val) {  // solution_checker.cpp:30-48
  DualTerm t{0.0, 0.0, 0.0};
  if (mult > 0.0) {
    if (lo == -kInf) t.violation = mult;
    else t.contribution = mult * lo, t.complementarity = mult * std::fabs(val - lo);
  } else if (mult < 0.0) {
    if (up == kInf) t.violation = -mult;
    else t.contribution = mult * up, t.complementarity = -mult * std::fabs(up - val);
  }
  return t;
}
double bound_violation(double val, double lo, double up) {
  double v = 0.0;
  if (lo != -kInf) v = std::max(v, (lo - val) / (1.0 + std::fabs(lo)));
  if (up != kInf) v = std::max(v, (val - up) / (1.0 + std::fabs(up)));
  return v;
}
}  // namespace

CheckReport check_solution(const Model& lp, const std::vector<double>& x, const std::vector<double>& row_dual) {
  CheckReport rep;
  const int m = lp.num_rows, n = lp.num_cols;
  const double sense = lp.sense;
  auto reject = [&rep]() {
    rep.max_primal_violation = rep.max_dual_violation = rep.relative_gap = kInf;
    rep.primal_ok = rep.dual_ok = rep.gap_ok = false;
    return rep;
  };
  if (static_cast<int>(x.size()) != n || static_cast<int>(row_dual.size()) != m) return reject();
  // Element-wise work runs on the host threads: each element's terms are those of the
  // sequential pass, maxima combine exactly in any order, and the two sums are taken afterwards
  // in the sequential pass's order (rows, then columns).
  std::atomic<bool> finite{true};
  parallel_ranges(std::max<long long>(n, m), [&](long long b, long long e) {
    bool ok = true;
    for (long long k = b; k < e; ++k)
      ok = ok && (k >= n || std::isfinite(x[k])) && (k >= m || std::isfinite(row_dual[k]));
    if (!ok) finite.store(false, std::memory_order_relaxed);
  });
  if (!finite.load()) return reject();
  std::mutex mu;
  auto fold = [&mu](double& into, double v) {  // with mu held
    into = std::max(into, v);
  };
  double c_scale = 1.0;
  parallel_ranges(n, [&](long long jb, long long je) {  // column bound violations and max |c_j|
    double pv = 0.0, cs = 1.0;
    for (long long j = jb; j < je; ++j) {
      pv = std::max(pv, bound_violation(x[j], lp.col_lower[j], lp.col_upper[j]));
      cs = std::max(cs, std::fabs(lp.obj[j]));
    }
    std::lock_guard<std::mutex> lock(mu);
    fold(rep.max_primal_violation, pv), fold(c_scale, cs);
  });
  std::vector<double> ax = lp.row_activity(x);
  std::vector<double> row_term = pooled_storage(static_cast<std::size_t>(m));
  parallel_ranges(m, [&](long long ib, long long ie) {  // row violations and multiplier terms
    double pv = 0.0, dv = 0.0, cp = 0.0;
    for (long long i = ib; i < ie; ++i) {
      pv = std::max(pv, bound_violation(ax[i], lp.row_lower[i], lp.row_upper[i]));
      const DualTerm t = evaluate_multiplier(sense * row_dual[i], lp.row_lower[i], lp.row_upper[i], ax[i]);
      dv = std::max(dv, t.violation / c_scale);
      cp = std::max(cp, t.complementarity);
      row_term[i] = t.contribution;
    }
    std::lock_guard<std::mutex> lock(mu);
    fold(rep.max_primal_violation, pv), fold(rep.max_dual_violation, dv), fold(rep.max_complementarity, cp);
  });
  std::vector<double> col_term = pooled_storage(static_cast<std::size_t>(n));
  std::vector<double> obj_term = pooled_storage(static_cast<std::size_t>(n));
  parallel_ranges(n, [&](long long jb, long long je) {  // reduced costs and their terms
    double dv = 0.0, cp = 0.0;
    for (long long j = jb; j < je; ++j) {
      double aty = 0.0;  // (Aᵀ·sense·y)_j in the column's entry order
      for (int k = lp.col_start[j]; k < lp.col_start[j + 1]; ++k) aty += lp.value[k] * (sense * row_dual[lp.row_index[k]]);
      const double c = sense * lp.obj[j];
      const DualTerm t = evaluate_multiplier(c - aty, lp.col_lower[j], lp.col_upper[j], x[j]);
      dv = std::max(dv, t.violation / c_scale);
      cp = std::max(cp, t.complementarity);
      col_term[j] = t.contribution;
      obj_term[j] = c * x[j];
    }
    std::lock_guard<std::mutex> lock(mu);
    fold(rep.max_dual_violation, dv), fold(rep.max_complementarity, cp);
  });
  double dual_obj_min = 0.0, primal_obj_min = 0.0;
  for (int i = 0; i < m; ++i) dual_obj_min += row_term[i];
  for (int j = 0; j < n; ++j) dual_obj_min += col_term[j], primal_obj_min += obj_term[j];
  pool_vector(std::move(ax)), pool_vector(std::move(row_term)), pool_vector(std::move(col_term));
  pool_vector(std::move(obj_term));
  rep.primal_objective = sense * primal_obj_min + lp.obj_offset;
  rep.dual_objective = sense * dual_obj_min + lp.obj_offset;
  rep.relative_gap = std::fabs(rep.primal_objective - rep.dual_objective) /
                     (1.0 + std::fabs(rep.primal_objective) + std::fabs(rep.dual_objective));
  if (!std::isfinite(rep.primal_objective) || !std::isfinite(rep.dual_objective)) return reject();
  rep.primal_ok = rep.max_primal_violation <= 1e-6;
  rep.dual_ok = rep.max_dual_violation <= 1e-6;
  rep.gap_ok = rep.relative_gap <= 1e-6;
  return rep;
}

bool OriginalKkt::converged(double eps) const {  // termination.h:51-55 (obj_shift 0)
  const double rprim = primal_residual / (1.0 + b_norm), rdual = dual_residual / (1.0 + c_norm);
  const double gap = std::fabs(primal_obj - dual_obj) / (1.0 + std::fabs(primal_obj) + std::fabs(dual_obj));
  if (std::max({rprim, rdual, gap}) > eps) return false;
  if (eps >= 1e-6) return true;  // tolerances.h:34-36, the verifier's 1e-6
  return primal_max_rel <= 1e-6 && dual_max_rel <= 1e-6 && gap <= 1e-6;
}

OriginalKkt original_kkt(const Model& model, const std::vector<double>& x, const std::vector<double>& y) {
  // kkt_general (cpu_backend.cpp:225-284) on the original model with multipliers sense·y.
  // Element-wise terms are computed on the host threads; every sum is then taken in the
  // reference's order (rows, then columns), adding exactly the terms it adds, and the maxima
  // combine exactly in any order.
  const int m = model.num_rows, n = model.num_cols;
  // A·x row-sequential in column order (kkt_general's CSR product): row_activity adds every
  // row's terms in increasing column order, exactly that order.
  std::vector<double> ax = model.row_activity(x);
  // per row: viol², max(|lo|,|up|)², the dual objective term and the dual residual term (each
  // with a flag: whether the reference adds it)
  std::vector<double> r_viol = pooled_storage(static_cast<std::size_t>(m)), r_b = pooled_storage(static_cast<std::size_t>(m));
  std::vector<double> r_d = pooled_storage(static_cast<std::size_t>(m)), r_rd = pooled_storage(static_cast<std::size_t>(m));
  // per column: c_j², c_j·x_j, the dual residual term and the dual objective term (flagged)
  std::vector<double> c_c = pooled_storage(static_cast<std::size_t>(n)), c_p = pooled_storage(static_cast<std::size_t>(n));
  std::vector<double> c_rd = pooled_storage(static_cast<std::size_t>(n)), c_d = pooled_storage(static_cast<std::size_t>(n));
  std::vector<char> r_flag(static_cast<std::size_t>(m)), c_flag(static_cast<std::size_t>(n));  // bit 0: d, bit 1: rd
  std::mutex mu;
  double pmax = 0, dmax = 0, cinf = 0;
  auto ev = [](double v, double lo, double up) {
    if (v < lo) return (lo - v) / (1.0 + std::fabs(lo));
    if (v > up) return (v - up) / (1.0 + std::fabs(up));
    return 0.0;
  };
  parallel_ranges(m, [&](long long ib, long long ie) {
    double pm = 0, dm = 0;
    for (long long i = ib; i < ie; ++i) {
      const double lo = model.row_lower[i], up = model.row_upper[i];
      const double viol = ax[i] < lo ? lo - ax[i] : (ax[i] > up ? ax[i] - up : 0.0);
      r_viol[i] = viol * viol;
      pm = std::max(pm, ev(ax[i], lo, up));
      const double bl = std::isfinite(lo) ? std::fabs(lo) : 0.0, bu = std::isfinite(up) ? std::fabs(up) : 0.0;
      r_b[i] = std::max(bl, bu) * std::max(bl, bu);
      const double yi = y[i] * model.sense;
      char f = 0;
      if (yi > 0) {
        if (std::isfinite(lo)) r_d[i] = yi * lo, f = 1;
        else r_rd[i] = yi * yi, f = 2, dm = std::max(dm, yi);
      } else if (yi < 0) {
        if (std::isfinite(up)) r_d[i] = yi * up, f = 1;
        else r_rd[i] = yi * yi, f = 2, dm = std::max(dm, -yi);
      }
      r_flag[i] = f;
    }
    std::lock_guard<std::mutex> lock(mu);
    pmax = std::max(pmax, pm), dmax = std::max(dmax, dm);
  });
  parallel_ranges(n, [&](long long jb, long long je) {
    double pm = 0, dm = 0, ci = 0;
    for (long long j = jb; j < je; ++j) {
      double aty = 0;  // (Aᵀ·sense·y)_j in the column's entry order (the transpose's CSR product)
      for (int k = model.col_start[j]; k < model.col_start[j + 1]; ++k)
        aty += model.value[k] * (y[model.row_index[k]] * model.sense);
      const double cj = model.sense * model.obj[j];
      c_c[j] = cj * cj;
      ci = std::max(ci, std::fabs(cj));
      c_p[j] = cj * x[j];
      pm = std::max(pm, ev(x[j], model.col_lower[j], model.col_upper[j]));
      const double lam = cj - aty, lo = model.col_lower[j], up = model.col_upper[j];
      double z;
      if (std::isfinite(lo) && std::isfinite(up)) z = lam;
      else if (std::isfinite(lo)) z = std::max(lam, 0.0);
      else if (std::isfinite(up)) z = std::min(lam, 0.0);
      else z = 0.0;
      c_rd[j] = (lam - z) * (lam - z);
      dm = std::max(dm, std::fabs(lam - z));
      char f = 0;
      if (z > 0) c_d[j] = z * lo, f = 1;
      else if (z < 0) c_d[j] = z * up, f = 1;
      c_flag[j] = f;
    }
    std::lock_guard<std::mutex> lock(mu);
    pmax = std::max(pmax, pm), dmax = std::max(dmax, dm), cinf = std::max(cinf, ci);
  });
  double rp2 = 0, rd2 = 0, b2 = 0, c2 = 0, p = 0, d = 0;
  for (int i = 0; i < m; ++i) {
    rp2 += r_viol[i];
    b2 += r_b[i];
    if (r_flag[i] == 1) d += r_d[i];
    else if (r_flag[i] == 2) rd2 += r_rd[i];
  }
  for (int j = 0; j < n; ++j) {
    c2 += c_c[j];
    p += c_p[j];
    rd2 += c_rd[j];
    if (c_flag[j]) d += c_d[j];
  }
  for (auto* v : {&ax, &r_viol, &r_b, &r_d, &r_rd, &c_c, &c_p, &c_rd, &c_d}) pool_vector(std::move(*v));
  OriginalKkt k;
  k.primal_residual = std::sqrt(rp2), k.dual_residual = std::sqrt(rd2);
  k.primal_obj = p, k.dual_obj = d;
  k.b_norm = std::sqrt(b2), k.c_norm = std::sqrt(c2);
  k.primal_max_rel = pmax, k.dual_max_rel = dmax / (1.0 + cinf);
  return k;
}

std::string CheckReport::summary() const {
  char buf[256];
  std::snprintf(buf, sizeof buf, "primal viol %.1e  dual viol %.1e  compl %.1e  gap %.1e  => %s", max_primal_violation,
                max_dual_violation, max_complementarity, relative_gap, passed() ? "PASS" : "FAIL");
  return buf;
}

// ============================================================ presolve (presolve.cpp)
namespace {
constexpr double kFeasTol = 1e-9;
bool within(double v, double lo, double up) {
  return v >= lo - kFeasTol * (1 + std::fabs(lo)) && v <= up + kFeasTol * (1 + std::fabs(up));
}
}  // namespace

namespace {
// Presolve's per-thread scratch (kept between calls, within the host reuse limit).
struct PresolveScratch {
  std::vector<int> row_xor, row_cnt, col_cnt, new_row;
  std::vector<double> rl, ru, cl, cu;
  std::vector<char> row_alive, col_alive;
  std::vector<int> pairs;  // (row, column) of every entry, grouped by row block (row_tags)
  std::vector<int> cand;   // the rows or columns a presolve loop acts on
  std::size_t accounted = 0;
  std::size_t bytes() const {
    return 4 * (row_xor.capacity() + row_cnt.capacity() + col_cnt.capacity() + new_row.capacity() +
                pairs.capacity() + cand.capacity()) +
           8 * (rl.capacity() + ru.capacity() + cl.capacity() + cu.capacity()) + row_alive.capacity() +
           col_alive.capacity();
  }
  void release() {  // frees the memory (clear() alone keeps the capacity)
    std::vector<int>().swap(row_xor), std::vector<int>().swap(row_cnt), std::vector<int>().swap(col_cnt);
    std::vector<int>().swap(new_row), std::vector<int>().swap(pairs), std::vector<int>().swap(cand);
    std::vector<double>().swap(rl), std::vector<double>().swap(ru), std::vector<double>().swap(cl);
    std::vector<double>().swap(cu);
    std::vector<char>().swap(row_alive), std::vector<char>().swap(col_alive);
  }
  ~PresolveScratch() { host_keep(accounted, 0); }
};
thread_local PresolveScratch t_presolve;

// An ordered scan of [0, len) in T chunks on the host threads: count(b, e) returns the number of
// items chunk [b, e) will write, size(total) is called once with the sum, then fill(b, e, at)
// writes the chunk's items starting at `at`, the number of items of the chunks before it.
template <class Count, class Size, class Fill>
void ordered_scan(long long len, int T, Count count, Size size, Fill fill) {
  if (len < T) T = static_cast<int>(std::max<long long>(len, 1));
  std::vector<long long> at(static_cast<std::size_t>(T) + 1, 0);
  auto lo = [&](long long c) { return len * c / T; };
  parallel_ranges(
      T,
      [&](long long cb, long long ce) {
        for (long long c = cb; c < ce; ++c) at[static_cast<std::size_t>(c) + 1] = count(lo(c), lo(c + 1));
      },
      1);
  for (int c = 0; c < T; ++c) at[static_cast<std::size_t>(c) + 1] += at[static_cast<std::size_t>(c)];
  size(at[static_cast<std::size_t>(T)]);
  parallel_ranges(
      T,
      [&](long long cb, long long ce) {
        for (long long c = cb; c < ce; ++c) fill(lo(c), lo(c + 1), at[static_cast<std::size_t>(c)]);
      },
      1);
}

// The indices i in [0, count) with pred(i), in increasing order, into `out`; pred is evaluated
// on the host threads (it must only read).
template <class Pred>
void select_in_order(int count, Pred pred, std::vector<int>& out) {
  out.clear();
  const int T = count < 65536 ? 1 : host_threads();
  if (T == 1) {
    for (int i = 0; i < count; ++i)
      if (pred(i)) out.push_back(i);
    return;
  }
  std::vector<std::vector<int>> part(static_cast<std::size_t>(T));
  parallel_ranges(
      T,
      [&](long long cb, long long ce) {
        for (long long c = cb; c < ce; ++c) {
          const int ib = static_cast<int>(static_cast<long long>(count) * c / T);
          const int ie = static_cast<int>(static_cast<long long>(count) * (c + 1) / T);
          for (int i = ib; i < ie; ++i)
            if (pred(i)) part[static_cast<std::size_t>(c)].push_back(i);
        }
      },
      1);
  for (const auto& p : part) out.insert(out.end(), p.begin(), p.end());
}

// Per row: the number of entries and the XOR of their column indices. Both are commutative, so
// any order of the entries gives the arrays of a sequential pass. With several host threads the
// entries are bucketed by row block (bucket_rows), then each block is applied by one thread
// with plain stores into rows that fit in its cache: atomics on random rows would serialise the
// cache misses instead.
void row_tags(const Model& M, std::vector<int>& row_xor, std::vector<int>& row_cnt, std::vector<int>& pairs) {
  const int m = M.num_rows, n = M.num_cols;
  row_xor.assign(static_cast<std::size_t>(m), 0);
  row_cnt.assign(static_cast<std::size_t>(m), 0);
  const int T = pass_threads(static_cast<long long>(M.nnz()));
  if (T == 1) {
    for (int j = 0; j < n; ++j)
      for (int k = M.col_start[j]; k < M.col_start[j + 1]; ++k) row_xor[M.row_index[k]] ^= j, ++row_cnt[M.row_index[k]];
    return;
  }
  if (static_cast<long long>(M.nnz()) > kBucketMaxEntries) {  // no scratch: relaxed integer atomics
    parallel_ranges(n, [&](long long jb, long long je) {
      for (long long j = jb; j < je; ++j)
        for (int k = M.col_start[j]; k < M.col_start[j + 1]; ++k) {
          __atomic_fetch_xor(&row_xor[M.row_index[k]], static_cast<int>(j), __ATOMIC_RELAXED);
          __atomic_fetch_add(&row_cnt[M.row_index[k]], 1, __ATOMIC_RELAXED);
        }
    });
    return;
  }
  size_for_copy(pairs, 2 * M.nnz());
  std::vector<long long> start;
  bucket_rows(M, T, start, [&](long long q, int i, int j, int) { pairs[2 * q] = i, pairs[2 * q + 1] = j; });
  parallel_ranges(
      static_cast<long long>(start.size()) - 1,
      [&](long long bb, long long be) {
        for (long long q = start[bb]; q < start[be]; ++q) {
          const int i = pairs[2 * q];
          row_xor[i] ^= pairs[2 * q + 1], ++row_cnt[i];
        }
      },
      1);
}

void clear_model(Model& R) {  // empties every vector, keeping its capacity
  R.num_rows = R.num_cols = 0, R.sense = 1, R.obj_offset = 0.0;
  R.obj.clear(), R.col_lower.clear(), R.col_upper.clear(), R.row_lower.clear(), R.row_upper.clear();
  R.col_start.clear(), R.row_index.clear(), R.value.clear(), R.is_integer.clear();
}
}  // namespace

std::size_t capacity_bytes(const Model& m) {
  return 8 * (m.obj.capacity() + m.col_lower.capacity() + m.col_upper.capacity() + m.row_lower.capacity() +
              m.row_upper.capacity() + m.value.capacity()) +
         4 * (m.col_start.capacity() + m.row_index.capacity()) + m.is_integer.capacity();
}

bool host_keep(std::size_t& accounted, std::size_t bytes) {
  static const std::size_t limit = [] {
    const char* env = std::getenv("PS26119_HOST_REUSE_MB");
    const long long mb = env ? std::atoll(env) : 2048;
    return mb > 0 ? static_cast<std::size_t>(mb) << 20 : std::size_t{0};
  }();
  static std::mutex mu;
  static std::size_t total = 0;
  std::lock_guard<std::mutex> lock(mu);
  total -= accounted;
  accounted = 0;
  if (bytes == 0 || total + bytes > limit) return false;
  total += bytes;
  accounted = bytes;
  return true;
}

namespace {
struct VectorPool {
  std::vector<std::vector<double>> free;
  std::size_t accounted = 0;
  std::size_t bytes() const {
    std::size_t b = 0;
    for (const auto& v : free) b += 8 * v.capacity();
    return b;
  }
  ~VectorPool() { host_keep(accounted, 0); }
};
thread_local VectorPool t_vectors;
}  // namespace

namespace {
// n elements in the smallest pooled buffer that holds them (a fresh vector when none does);
// the values are unspecified: the caller overwrites every one
std::vector<double> pooled_storage(std::size_t n) {
  VectorPool& P = t_vectors;
  long long best = -1;
  for (std::size_t k = 0; k < P.free.size(); ++k)
    if (P.free[k].capacity() >= n && (best < 0 || P.free[k].capacity() < P.free[static_cast<std::size_t>(best)].capacity()))
      best = static_cast<long long>(k);
  std::vector<double> v;
  if (best >= 0) {
    v.swap(P.free[static_cast<std::size_t>(best)]);
    P.free.erase(P.free.begin() + best);
    host_keep(P.accounted, P.bytes());
  }
  size_for_copy(v, n);
  return v;
}
}  // namespace

std::vector<double> pooled_vector(std::size_t n) {
  std::vector<double> v = pooled_storage(n);
  parallel_ranges(static_cast<long long>(n), [&](long long b, long long e) { std::fill(v.data() + b, v.data() + e, 0.0); },
                  1LL << 18);
  return v;
}

void pool_vector(std::vector<double>&& v) {
  if (v.capacity() < (std::size_t{1} << 16)) return;  // small ones are cheap to allocate
  VectorPool& P = t_vectors;
  P.free.push_back(std::move(v));
  if (P.free.size() > 8) P.free.erase(P.free.begin());  // the 8 most recent
  if (!host_keep(P.accounted, P.bytes())) std::vector<std::vector<double>>().swap(P.free);
}

PresolveResult presolve(const Model& M) {
  PresolveResult r;
  presolve_into(M, r);
  return r;
}

void presolve_into(const Model& M, PresolveResult& r) {  // presolve.cpp:22-156 (LP: no integer columns here)
  r.outcome = PresolveResult::Outcome::Unchanged;
  r.message.clear();
  r.removed_rows = r.removed_cols = r.tightened_bounds = 0;
  r.row_map.clear(), r.col_map.clear(), r.singletons.clear();
  // The reduced model is left as the last call built it (its vectors keep their sizes for the
  // build below) and emptied on every way out that does not build it.
  struct ClearUnlessReduced {
    PresolveResult& r;
    ~ClearUnlessReduced() {
      if (r.outcome != PresolveResult::Outcome::Reduced) clear_model(r.reduced);
    }
  } clear_unless_reduced{r};
  PresolveScratch& S = t_presolve;
  const int m = M.num_rows, n = M.num_cols;
  // A singleton row's one remaining column is recovered as the XOR of the row's live column
  // indices (kept up to date as columns are removed), and its coefficient by a scan of that
  // column: the same (j, a) the reference finds by walking the row (presolve.cpp:60-66), with
  // no row-wise copy of A.
  std::vector<int>& row_xor = S.row_xor;
  std::vector<int>& row_cnt = S.row_cnt;
  row_tags(M, row_xor, row_cnt, S.pairs);
  std::vector<double>&rl = S.rl, &ru = S.ru, &cl = S.cl, &cu = S.cu;
  size_for_copy(rl, M.row_lower.size()), size_for_copy(ru, M.row_upper.size());
  size_for_copy(cl, M.col_lower.size()), size_for_copy(cu, M.col_upper.size());
  const CopyJob bounds[] = {{rl.data(), M.row_lower.data(), 8 * rl.size()},
                            {ru.data(), M.row_upper.data(), 8 * ru.size()},
                            {cl.data(), M.col_lower.data(), 8 * cl.size()},
                            {cu.data(), M.col_upper.data(), 8 * cu.size()}};
  parallel_copy(bounds, 4);
  std::vector<char>&row_alive = S.row_alive, &col_alive = S.col_alive;
  row_alive.assign(static_cast<std::size_t>(m), 1);
  std::vector<int>& col_cnt = S.col_cnt;
  size_for_copy(col_alive, static_cast<std::size_t>(n)), size_for_copy(col_cnt, static_cast<std::size_t>(n));
  size_for_copy(r.fixed_value, static_cast<std::size_t>(n));
  parallel_ranges(n, [&](long long jb, long long je) {
    for (long long j = jb; j < je; ++j)
      col_alive[j] = 1, col_cnt[j] = M.col_start[j + 1] - M.col_start[j], r.fixed_value[j] = kNaN;
  });
  double offset = M.obj_offset;
  auto infeasible = [&](const std::string& why) {
    r.outcome = PresolveResult::Outcome::Infeasible;
    r.message = why;
  };
  // keeps the scratch for the next call on this thread, or frees it beyond the reuse limit
  struct KeepScratch {
    PresolveScratch& s;
    ~KeepScratch() {
      if (!host_keep(s.accounted, s.bytes())) s.release();
    }
  } keep{S};
  // Within the row loop of a pass no row's count or liveness changes but the row's own, and
  // within the column loop no column's bounds, count or liveness changes but the column's own.
  // So each loop's candidates are known when it starts: they are found on the host threads and
  // then processed one by one in index order, the order of a full sequential scan.
  std::vector<int>& cand = S.cand;
  bool changed = true;
  while (changed) {
    changed = false;
    select_in_order(m, [&](int i) { return row_alive[i] && row_cnt[i] <= 1; }, cand);
    for (const int i : cand) {  // rows: empty (R1) and singleton (R4)
      if (!row_alive[i]) continue;
      if (row_cnt[i] == 0) {
        if (!within(0.0, rl[i], ru[i])) { infeasible("empty row " + std::to_string(i) + " excludes 0"); return; }
        row_alive[i] = 0;
        ++r.removed_rows;
        changed = true;
      } else if (row_cnt[i] == 1) {
        const int j = row_xor[i];
        double a = 0;
        for (int p = M.col_start[j]; p < M.col_start[j + 1]; ++p)
          if (M.row_index[p] == i) a = M.value[p];
        if (!col_alive[j] || a == 0.0) continue;
        const double lo = a > 0 ? rl[i] / a : ru[i] / a;
        const double hi = a > 0 ? ru[i] / a : rl[i] / a;
        const bool set_lower = lo > cl[j], set_upper = hi < cu[j];
        double nl = set_lower ? lo : cl[j], nu = set_upper ? hi : cu[j];
        if (nl > nu) {
          if (nl - nu > kFeasTol * (1 + std::fabs(nl)))
            { infeasible("singleton row " + std::to_string(i) + " conflicts with the bounds of its column"); return; }
          nl = nu = 0.5 * (nl + nu);
        }
        cl[j] = nl;
        cu[j] = nu;
        r.singletons.push_back({i, j, a, set_lower, set_upper});
        r.tightened_bounds += set_lower + set_upper;
        row_alive[i] = 0;
        --col_cnt[j];
        ++r.removed_rows;
        changed = true;
      }
    }
    select_in_order(n, [&](int j) { return col_alive[j] && (cl[j] == cu[j] || col_cnt[j] == 0); }, cand);
    for (const int j : cand) {  // columns: fixed (R2) and empty (R3)
      if (!col_alive[j]) continue;
      double v;
      if (cl[j] == cu[j]) {
        v = cl[j];
      } else if (col_cnt[j] == 0) {
        const double c = M.sense * M.obj[j];
        v = c > 0 ? cl[j] : (c < 0 ? cu[j] : std::min(std::max(0.0, cl[j]), cu[j]));
        if (!std::isfinite(v)) continue;
      } else {
        continue;
      }
      for (int p = M.col_start[j]; p < M.col_start[j + 1]; ++p) {
        const int i = M.row_index[p];
        if (!row_alive[i]) continue;
        const double t = M.value[p] * v;
        if (std::isfinite(rl[i])) rl[i] -= t;
        if (std::isfinite(ru[i])) ru[i] -= t;
        --row_cnt[i];
        row_xor[i] ^= j;
      }
      offset += M.obj[j] * v;
      r.fixed_value[j] = v;
      col_alive[j] = 0;
      ++r.removed_cols;
      changed = true;
    }
  }
  if (r.removed_rows == 0 && r.removed_cols == 0) {
    r.outcome = PresolveResult::Outcome::Unchanged;
    return;
  }
  Model& R = r.reduced;
  // The maps and the reduced matrix are built by ordered scans on the host threads: each chunk
  // counts its items, the chunks' offsets are their counts' prefix sums, and each chunk then
  // writes its items from its offset, so the output is that of one sequential pass.
  std::vector<int>& new_row = S.new_row;
  size_for_copy(new_row, static_cast<std::size_t>(m));
  ordered_scan(
      m, m < 65536 ? 1 : host_threads(),
      [&](long long b, long long e) {
        long long k = 0;
        for (long long i = b; i < e; ++i) k += row_alive[i] != 0;
        return k;
      },
      [&](long long total) { size_for_copy(r.row_map, static_cast<std::size_t>(total)); },
      [&](long long b, long long e, long long at) {
        for (long long i = b; i < e; ++i) {
          new_row[i] = row_alive[i] ? static_cast<int>(at) : -1;
          if (row_alive[i]) r.row_map[at++] = static_cast<int>(i);
        }
      });
  ordered_scan(
      n, n < 65536 ? 1 : host_threads(),
      [&](long long b, long long e) {
        long long k = 0;
        for (long long j = b; j < e; ++j) k += col_alive[j] != 0;
        return k;
      },
      [&](long long total) { size_for_copy(r.col_map, static_cast<std::size_t>(total)); },
      [&](long long b, long long e, long long at) {
        for (long long j = b; j < e; ++j)
          if (col_alive[j]) r.col_map[at++] = static_cast<int>(j);
      });
  // Every vector of R is sized here and overwritten in full: it keeps its size from the last
  // call, so a repeated call writes each element once (no zero fill before the copy).
  R.sense = M.sense;
  R.obj_offset = offset;
  R.num_rows = static_cast<int>(r.row_map.size());
  R.num_cols = static_cast<int>(r.col_map.size());
  R.is_integer.clear();
  const int nk = R.num_cols;
  size_for_copy(R.obj, r.col_map.size()), size_for_copy(R.col_lower, r.col_map.size());
  size_for_copy(R.col_upper, r.col_map.size()), size_for_copy(R.col_start, r.col_map.size() + 1);
  size_for_copy(R.row_lower, r.row_map.size()), size_for_copy(R.row_upper, r.row_map.size());
  parallel_ranges(nk, [&](long long qb, long long qe) {  // the kept columns' data
    for (long long q = qb; q < qe; ++q) {
      const int j = r.col_map[static_cast<std::size_t>(q)];
      R.obj[q] = M.obj[j], R.col_lower[q] = cl[j], R.col_upper[q] = cu[j];
    }
  });
  parallel_ranges(R.num_rows, [&](long long qb, long long qe) {  // the kept rows' bounds
    for (long long q = qb; q < qe; ++q) {
      const int i = r.row_map[static_cast<std::size_t>(q)];
      R.row_lower[q] = rl[i], R.row_upper[q] = ru[i];
    }
  });
  // The kept columns' entries in kept rows, renumbered. With no row removed, every entry of a
  // kept column is kept under its own row number.
  const bool all_rows = r.removed_rows == 0;
  R.col_start[0] = 0;
  ordered_scan(
      nk, pass_threads(static_cast<long long>(M.nnz())),
      [&](long long qb, long long qe) {
        long long k = 0;
        for (long long q = qb; q < qe; ++q) {
          const int j = r.col_map[static_cast<std::size_t>(q)];
          if (all_rows) {
            k += M.col_start[j + 1] - M.col_start[j];
          } else {
            for (int p = M.col_start[j]; p < M.col_start[j + 1]; ++p) k += new_row[M.row_index[p]] >= 0;
          }
        }
        return k;
      },
      [&](long long total) {
        size_for_copy(R.row_index, static_cast<std::size_t>(total)), size_for_copy(R.value, static_cast<std::size_t>(total));
      },
      [&](long long qb, long long qe, long long at) {
        for (long long q = qb; q < qe; ++q) {
          const int j = r.col_map[static_cast<std::size_t>(q)];
          for (int p = M.col_start[j]; p < M.col_start[j + 1]; ++p) {
            const int i = all_rows ? M.row_index[p] : new_row[M.row_index[p]];
            if (i >= 0) R.row_index[at] = i, R.value[at] = M.value[p], ++at;
          }
          R.col_start[q + 1] = static_cast<int>(at);
        }
      });
  r.outcome = PresolveResult::Outcome::Reduced;
}

namespace {
// Every field of `s` except x, y and z: postsolve rebuilds those on the original model, so
// copying the reduced ones (tens of MB on large models) would only be overwritten. The size
// check makes a field added to Solution fail to compile here until it is copied too.
Solution without_xyz(const Solution& s) {
  static_assert(sizeof(Solution) == 656, "Solution changed: copy the new field in without_xyz");
  Solution o;
  o.status = s.status;
  o.dual_ray = s.dual_ray, o.primal_ray = s.primal_ray;
  o.objective = s.objective, o.dual_objective = s.dual_objective;
  o.primal_residual = s.primal_residual, o.dual_residual = s.dual_residual, o.gap = s.gap;
  o.iterations = s.iterations, o.seconds = s.seconds, o.setup_seconds = s.setup_seconds;
  o.certified_bound = s.certified_bound, o.primal_weight = s.primal_weight;
  o.check = s.check, o.check_primal = s.check_primal, o.check_dual = s.check_dual, o.check_gap = s.check_gap;
  o.engine = s.engine, o.precision = s.precision, o.message = s.message;
  o.engine_result = s.engine_result;
  o.presolve_seconds = s.presolve_seconds;
  o.model_fingerprint = s.model_fingerprint;
  o.iterations_to_fast = s.iterations_to_fast;
  return o;
}
}  // namespace

Solution postsolve(const Model& M, const PresolveResult& r, const Solution& red) {  // presolve.cpp:158-193
  Solution s = without_xyz(red);
  const int m = M.num_rows, n = M.num_cols;
  s.x = pooled_vector(static_cast<std::size_t>(n));
  s.y = pooled_vector(static_cast<std::size_t>(m));
  const bool have_x = red.x.size() == r.col_map.size();
  const bool have_y = red.y.size() == r.row_map.size();
  // element-wise writes to distinct entries (the maps are one-to-one), on the host threads
  parallel_ranges(n, [&](long long jb, long long je) {
    for (long long j = jb; j < je; ++j)
      if (!std::isnan(r.fixed_value[j])) s.x[j] = r.fixed_value[j];
  });
  if (have_x)
    parallel_ranges(static_cast<long long>(r.col_map.size()), [&](long long cb, long long ce) {
      for (long long c = cb; c < ce; ++c) s.x[r.col_map[c]] = red.x[c];
    });
  if (have_y)
    parallel_ranges(static_cast<long long>(r.row_map.size()), [&](long long qb, long long qe) {
      for (long long q = qb; q < qe; ++q) s.y[r.row_map[q]] = red.y[q];
    });
  for (auto it = r.singletons.rbegin(); it != r.singletons.rend(); ++it) {
    const int j = it->col;
    double z = M.obj[j];
    for (int p = M.col_start[j]; p < M.col_start[j + 1]; ++p) z -= M.value[p] * s.y[M.row_index[p]];
    const double zm = M.sense * z;
    if ((zm > 0 && it->set_lower) || (zm < 0 && it->set_upper)) s.y[it->row] = z / it->a;
  }
  s.z = pooled_storage(static_cast<std::size_t>(n));
  parallel_ranges(n, [&](long long jb, long long je) {  // each z_j in its own column order
    for (long long j = jb; j < je; ++j) {
      double z = M.obj[j];
      for (int p = M.col_start[j]; p < M.col_start[j + 1]; ++p) z -= M.value[p] * s.y[M.row_index[p]];
      s.z[j] = z;
    }
  });
  s.objective = M.objective_value(s.x);
  if (!have_x) {
    s.x.clear();
    s.objective = kNaN;
  }
  if (!have_y) s.y.clear(), s.z.clear();
  return s;
}

std::uint64_t presolve_digest(const PresolveResult& r) {
  CanonicalBytes b;
  b.i64(r.outcome == PresolveResult::Outcome::Reduced ? 0 : r.outcome == PresolveResult::Outcome::Infeasible ? 1 : 2);
  b.i64(r.removed_rows), b.i64(r.removed_cols), b.i64(r.tightened_bounds);
  b.word(r.row_map.size());
  for (int i : r.row_map) b.i64(i);
  b.word(r.col_map.size());
  for (int j : r.col_map) b.i64(j);
  b.f64s(r.fixed_value);
  b.word(r.singletons.size());
  for (const auto& t : r.singletons) b.i64(t.row), b.i64(t.col), b.f64(t.a), b.i64(t.set_lower), b.i64(t.set_upper);
  b.word(r.outcome == PresolveResult::Outcome::Reduced ? r.reduced.fingerprint() : 0);
  return fnv1a(kFnvOffset, b.buf);
}

// Maps a Farkas vector of the reduced model to the original rows (presolve.cpp:195-207): kept
// rows keep their multiplier; a column bound made by a removed singleton row moves onto that
// row, newest singleton first, when λ_j = −(Aᵀr)_j points at it.
std::vector<double> postsolve_farkas(const Model& M, const PresolveResult& r, const std::vector<double>& red_ray) {
  std::vector<double> ray(static_cast<std::size_t>(M.num_rows), 0.0);
  if (red_ray.size() != r.row_map.size()) return {};
  for (std::size_t q = 0; q < r.row_map.size(); ++q) ray[r.row_map[q]] = red_ray[q];
  for (auto it = r.singletons.rbegin(); it != r.singletons.rend(); ++it) {
    const int j = it->col;
    double lam = 0.0;
    for (int p = M.col_start[j]; p < M.col_start[j + 1]; ++p) lam -= M.value[p] * ray[M.row_index[p]];
    if ((lam > 0 && it->set_lower) || (lam < 0 && it->set_upper)) ray[it->row] = lam / it->a;
  }
  return ray;
}

// ============================================================ dispatcher (solve.cpp)
namespace {

using clock_t_ = std::chrono::steady_clock;
double since(clock_t_::time_point t0) { return std::chrono::duration<double>(clock_t_::now() - t0).count(); }
// The certified bound's implied-bounds refinement runs only within the time budget (solve.cpp:39).
bool within_bound_budget(double elapsed, double time_limit) { return elapsed < 1.1 * time_limit + 1.0; }

const char* alg_name(Algorithm a) {
  switch (a) {
    case Algorithm::Auto: return "auto";
    case Algorithm::Oracle: return "oracle";
    case Algorithm::Pdlp: return "pdlp";
    case Algorithm::R2hpdhg: return "r2hpdhg";
    default: return "simplex";
  }
}

void note(Solution& s, const std::string& t) { s.message += std::string(s.message.empty() ? "" : "; ") + t; }

thread_local std::vector<std::pair<const char*, double>>* g_phases = nullptr;

// Times a scope as one phase of the current phase log.
struct PhaseTimer {
  const char* name;
  clock_t_::time_point t0 = clock_t_::now();
  explicit PhaseTimer(const char* n) : name(n) {}
  ~PhaseTimer() { phase_note(name, since(t0)); }
};

EngineOptions engine_options(const Options& o) {  // engine.cpp:168-186
  EngineOptions e;
  e.tolerance = o.tolerance;
  e.time_limit = o.time_limit;
  e.iteration_limit = o.iteration_limit;
  e.check_every = o.check_every > 0 ? o.check_every : 64;
  e.mixed = o.precision == Precision::Mixed;
  e.exact = o.exact;
  e.scaling = o.scaling;
  e.reflection = o.reflection;
  e.warm_x = o.warm_x;
  e.warm_y = o.warm_y;
  e.warm_primal_weight = o.warm_primal_weight;
  e.mixed_stall_checks = o.mixed_stall_checks;
  e.kkt_b_norm = o.kkt_b_norm;
  e.kkt_c_norm = o.kkt_c_norm;
  e.kkt_obj_shift = o.kkt_obj_shift;
  e.verbosity = o.verbosity;
  e.pdlp = o.algorithm == Algorithm::Pdlp;
  return e;
}

Solution trivially_infeasible(const Options& options, const std::string& why) {
  Solution s;
  s.status = Status::Infeasible;
  s.precision = options.precision == Precision::Mixed ? "mixed" : "fp64";
  s.message = "bounds cross: " + why;
  return s;
}

// The first-order engine on the GPU for one model (solve.cpp:469-609, LP part).
Solution solve_direct(const Model& model, const Options& options, bool certify = true) {
  const auto t0 = clock_t_::now();
  Solution sol;
  sol.precision = options.precision == Precision::Mixed ? "mixed" : "fp64";
  if (auto err = options.model_validated ? std::string() : model.validate(); !err.empty()) {
    sol.status = Status::NotSolved;
    sol.message = "invalid model: " + err;
    return sol;
  }
  if ((!options.warm_x.empty() && static_cast<int>(options.warm_x.size()) != model.num_cols) ||
      (!options.warm_y.empty() && static_cast<int>(options.warm_y.size()) != model.num_rows)) {
    sol.status = Status::NotSolved;
    sol.message = "warm start vectors have the wrong size";
    return sol;
  }
  auto finite = [](const std::vector<double>& v) { return std::all_of(v.begin(), v.end(), [](double a) { return std::isfinite(a); }); };
  if (!finite(options.warm_x) || !finite(options.warm_y) ||
      !(options.warm_primal_weight >= 0 && std::isfinite(options.warm_primal_weight))) {
    sol.status = Status::NotSolved;
    sol.message = "warm start contains non-finite values";
    return sol;
  }
  if (auto why = model.crossed_bounds(); !why.empty()) return trivially_infeasible(options, why);
  try {
    HostOutputs out;
    const auto te = clock_t_::now();
    const EngineResult R = run_engine_host(model.view(), engine_options(options), out);
    if (g_phases) {
      const double total = since(te);
      phase_note("engine.setup", R.setup_seconds);
      phase_note("engine.loop", R.loop_seconds);
      phase_note("engine.finish", R.finish_seconds);
      phase_note("engine.teardown", R.teardown_seconds);
      phase_note("engine.copies", total - R.setup_seconds - R.loop_seconds - R.finish_seconds - R.teardown_seconds);
    }
    sol.status = R.status;
    sol.iterations = R.iterations;
    sol.objective = R.objective;
    sol.dual_objective = R.dual_objective;
    sol.primal_residual = R.primal_residual;
    sol.dual_residual = R.dual_residual;
    sol.gap = R.gap;
    sol.primal_weight = R.primal_weight;
    sol.setup_seconds = R.setup_seconds;
    sol.message = R.message;
    sol.engine_result = R;
    sol.engine = options.algorithm == Algorithm::Pdlp ? "pdlp-b200" : "r2hpdhg-b200";
    sol.x = std::move(out.x);
    sol.y = std::move(out.y);
    sol.z = std::move(out.z);
    if (R.have_dual_ray) sol.dual_ray = std::move(out.dual_ray);
    if (R.have_primal_ray) sol.primal_ray = std::move(out.primal_ray);
    if (sol.status == Status::Unbounded && !check_unboundedness_certificate(model, sol.x, sol.primal_ray).passed) {
      // A ray from an iterate that is not primal-feasible: find a feasible point with the same
      // engine on the zero-objective model (never unbounded) within what is left of the budget
      // (solve.cpp:552-581). Feasible → the gate checks point + ray; infeasible → that verdict
      // with its own certificate; otherwise an honest limit status.
      Model feas = model;
      std::fill(feas.obj.begin(), feas.obj.end(), 0.0);
      Options fo = options;
      fo.presolve = false;
      fo.warm_x.clear();
      fo.warm_y.clear();
      fo.time_limit = std::max(0.0, options.time_limit - since(t0));
      fo.iteration_limit = std::max<long long>(0, options.iteration_limit - sol.iterations);
      Solution f = solve_direct(feas, fo, false);
      const long long total = sol.iterations + f.iterations;
      if (f.status == Status::Optimal) {
        sol.x = f.x;
        note(sol, "feasible point from a zero-objective solve (" + std::to_string(f.iterations) + " iterations)");
      } else if (f.status == Status::Infeasible) {
        f.message = "unbounded direction found, but the model is infeasible: " + f.message;
        f.primal_ray.clear();
        sol = f;
      } else {
        sol.status = f.status;
        note(sol, std::string("no feasible point found for the ray (") + status_name(f.status) + ")");
        sol.primal_ray.clear();
      }
      sol.iterations = total;
    }
  } catch (const std::bad_alloc&) {
    sol = Solution{};
    sol.status = Status::NotSolved;
    sol.message = "out of memory";
  } catch (const std::exception& e) {
    sol = Solution{};
    sol.status = Status::NumericalError;
    sol.message = e.what();
  }
  if (certify && static_cast<int>(sol.y.size()) == model.num_rows && model.num_rows + model.num_cols > 0) {
    PhaseTimer pt("certified_bound");
    sol.certified_bound =
        certified_dual_bound(model, sol.y, within_bound_budget(since(t0), options.time_limit)).bound;
  }
  sol.seconds = since(t0);
  return sol;
}

// Presolve wrapper (solve.cpp:266-467, LP part).
Solution solve_impl(const Model& model, const Options& options) {
  const bool bad_warm = (!options.warm_x.empty() && static_cast<int>(options.warm_x.size()) != model.num_cols) ||
                        (!options.warm_y.empty() && static_cast<int>(options.warm_y.size()) != model.num_rows);
  auto finite = [](const std::vector<double>& v) { return std::all_of(v.begin(), v.end(), [](double a) { return std::isfinite(a); }); };
  const bool bad_warm_values = !finite(options.warm_x) || !finite(options.warm_y);
  if (!options.presolve || bad_warm || bad_warm_values || (!options.model_validated && !model.validate().empty()))
    return solve_direct(model, options);
  if (auto why = model.crossed_bounds(); !why.empty()) return trivially_infeasible(options, why);
  const auto t0 = clock_t_::now();
  // this thread's presolve result, its memory reused from the previous call (host_keep)
  struct PresolveHolder {
    PresolveResult r;
    std::size_t accounted = 0;
    ~PresolveHolder() { host_keep(accounted, 0); }
  };
  static thread_local PresolveHolder t_pr;
  struct KeepResult {
    PresolveHolder& h;
    ~KeepResult() {
      const PresolveResult& r = h.r;
      const std::size_t bytes = capacity_bytes(r.reduced) + 4 * (r.row_map.capacity() + r.col_map.capacity()) +
                                8 * r.fixed_value.capacity() + sizeof(PresolveResult::Singleton) * r.singletons.capacity();
      if (!host_keep(h.accounted, bytes)) h.r = PresolveResult{};
    }
  } keep_result{t_pr};
  PresolveResult& pr = t_pr.r;
  presolve_into(model, pr);
  const double presolve_s = since(t0);
  phase_note("presolve", presolve_s);
  if (pr.outcome == PresolveResult::Outcome::Unchanged) {
    Solution s = solve_direct(model, options);
    s.presolve_seconds = presolve_s;
    return s;
  }
  Options inner = options;
  inner.presolve = false;
  inner.model_validated = false;  // the reduced model is checked before it reaches the device
  {
    // the two sequential sums (the reference's order) are independent: one task each
    double b2 = 0, c2 = 0;
    parallel_tasks(model.num_rows + model.num_cols >= 65536 ? 2 : 1, [&](int t) {
      if (t == 0 || model.num_rows + model.num_cols < 65536) {
        for (int i = 0; i < model.num_rows; ++i) {
          const double lo = std::isfinite(model.row_lower[i]) ? std::fabs(model.row_lower[i]) : 0.0;
          const double up = std::isfinite(model.row_upper[i]) ? std::fabs(model.row_upper[i]) : 0.0;
          b2 += std::max(lo, up) * std::max(lo, up);
        }
      }
      if (t == 1 || model.num_rows + model.num_cols < 65536)
        for (double c : model.obj) c2 += c * c;
    });
    inner.kkt_b_norm = std::sqrt(b2);
    inner.kkt_c_norm = std::sqrt(c2);
    inner.kkt_obj_shift = model.sense * (pr.reduced.obj_offset - model.obj_offset);
  }
  auto budget = [&](Options o, long long used) {
    o.time_limit = std::max(0.0, options.time_limit - since(t0));
    o.iteration_limit = std::max<long long>(0, options.iteration_limit - used);
    return o;
  };
  auto on_original = [&](const Solution& why, const std::string& what) {
    Options direct = budget(options, why.iterations);
    direct.presolve = false;
    Solution d = solve_direct(model, direct);
    d.iterations += why.iterations;
    d.seconds = since(t0);
    note(d, "presolve: " + what + "; re-solved the original model for an original-space certificate");
    return d;
  };
  if (pr.outcome == PresolveResult::Outcome::Infeasible) {
    Solution none;
    return on_original(none, "reduction found infeasibility (" + pr.message + ")");
  }
  if (!options.warm_x.empty()) {
    inner.warm_x.clear();
    for (int j : pr.col_map) inner.warm_x.push_back(options.warm_x[j]);
  }
  if (!options.warm_y.empty()) {
    inner.warm_y.clear();
    for (int i : pr.row_map) inner.warm_y.push_back(options.warm_y[i]);
  }
  Solution red;
  struct PoolAtExit {  // the reduced solution's vectors go back to this thread's pool
    Solution& s;
    ~PoolAtExit() {
      pool_vector(std::move(s.x)), pool_vector(std::move(s.y)), pool_vector(std::move(s.z));
    }
  } pool_red{red};
  if (pr.reduced.num_cols == 0 && pr.reduced.num_rows == 0) {
    red.status = Status::Optimal;
    red.engine = "presolve";
  } else {
    red = solve_direct(pr.reduced, budget(inner, 0), /*certify=*/false);
  }
  const std::string removed = "presolve removed " + std::to_string(pr.removed_rows) + " rows, " +
                              std::to_string(pr.removed_cols) + " cols";
  if (red.status == Status::Infeasible && red.dual_ray.size() == static_cast<std::size_t>(pr.reduced.num_rows)) {
    // cheaper than a re-solve: the reduced Farkas vector mapped to the original rows and checked
    // there (solve.cpp:346-364); only if that fails is the original re-solved
    std::vector<double> r = postsolve_farkas(model, pr, red.dual_ray);
    if (!r.empty() && check_infeasibility_certificate(model, r).passed) {
      Solution s = red;
      s.x.clear(), s.y.clear(), s.z.clear();
      s.dual_ray = std::move(r);
      note(s, removed + "; reduced-model Farkas certificate postsolved to the original rows");
      s.presolve_seconds = presolve_s;
      s.seconds = since(t0);
      return s;
    }
  }
  if (red.status == Status::Unbounded && red.primal_ray.size() == static_cast<std::size_t>(pr.reduced.num_cols) &&
      red.x.size() == static_cast<std::size_t>(pr.reduced.num_cols)) {
    // the same for a primal ray: fixed columns get d = 0, kept columns keep d_j; the point is the
    // ordinary primal postsolve (solve.cpp:365-391)
    std::vector<double> d(static_cast<std::size_t>(model.num_cols), 0.0);
    for (int j = 0; j < pr.reduced.num_cols; ++j) d[pr.col_map[j]] = red.primal_ray[j];
    Solution s = postsolve(model, pr, red);
    if (check_unboundedness_certificate(model, s.x, d).passed) {
      s.status = Status::Unbounded;
      s.primal_ray = std::move(d);
      s.dual_ray.clear(), s.y.clear(), s.z.clear();
      s.objective = s.dual_objective = kNaN;
      note(s, removed + "; reduced-model ray and point postsolved to the original model");
      s.presolve_seconds = presolve_s;
      s.seconds = since(t0);
      return s;
    }
  }
  if (red.status == Status::Infeasible || red.status == Status::Unbounded)
    return on_original(red, std::string("reduced model ") + status_name(red.status));
  Solution post;
  {
    PhaseTimer pt("postsolve");
    post = postsolve(model, pr, red);
  }
  const std::string pnote = "presolve removed " + std::to_string(pr.removed_rows) + " rows, " +
                            std::to_string(pr.removed_cols) + " cols";
  post.message = post.message.empty() ? pnote : post.message + "; " + pnote;
  auto passes = [&](const Solution& s) {
    if (static_cast<int>(s.x.size()) != model.num_cols || static_cast<int>(s.y.size()) != model.num_rows) return false;
    return original_kkt(model, s.x, s.y).converged(options.tolerance);  // solve.cpp:77-84, 414
  };
  bool passed = true;
  if (post.status == Status::Optimal) {
    PhaseTimer pt("original_kkt");
    passed = passes(post);
  }
  if (post.status == Status::Optimal && !passed) {  // solve.cpp:414-450
    Options tight = inner;
    tight.tolerance = std::max(options.tolerance * 1e-2, 1e-13);
    tight.warm_x = red.x;
    tight.warm_y = red.y;
    const Solution red2 = solve_direct(pr.reduced, budget(tight, red.iterations), /*certify=*/false);
    Solution post2 = postsolve(model, pr, red2);
    post2.iterations += red.iterations;
    if (post2.status == Status::Optimal && passes(post2)) {
      char buf[64];
      std::snprintf(buf, sizeof buf, "%.0e", tight.tolerance);
      post2.message = pnote + "; reduced model re-solved to " + buf + " to pass on the original";
      post = post2;
    } else {
      Solution cold = solve_direct(model, budget(inner, red.iterations + red2.iterations));
      cold.iterations += red.iterations + red2.iterations;
      note(cold, pnote + "; postsolved point missed the tolerance, fell back to solving the original");
      post = cold;
    }
  } else if (post.status == Status::Optimal && static_cast<int>(post.x.size()) != model.num_cols) {
    post.status = Status::NumericalError;
  }
  if (static_cast<int>(post.y.size()) == model.num_rows && model.num_rows + model.num_cols > 0) {
    PhaseTimer pt("certified_bound");
    post.certified_bound =
        certified_dual_bound(model, post.y, within_bound_budget(since(t0), options.time_limit)).bound;
  }
  post.presolve_seconds = presolve_s;
  post.seconds = since(t0);
  return post;
}

// The verification gate (solve.cpp:119-185, LP part).
void gate(const Model& model, const Options& options, Solution& s) {
  if (s.status == Status::Infeasible || s.status == Status::Unbounded) {
    s.objective = s.dual_objective = kNaN;
    if (s.status == Status::Infeasible && !model.crossed_bounds().empty()) {
      s.check = "PASS";
      return;
    }
    // claims other than Optimal are verified too (certificates.cpp)
    const CertificateCheck c = s.status == Status::Infeasible ? check_infeasibility_certificate(model, s.dual_ray)
                                                              : check_unboundedness_certificate(model, s.x, s.primal_ray);
    if (!c.present) {
      s.check.clear();
      note(s, "not certified (the engine returned no certificate)");
    } else if (c.passed) {
      s.check = "PASS";
      note(s, c.detail);
    } else {
      s.check = "FAIL";
      note(s, std::string(status_name(s.status)) + " withdrawn, " + c.detail);
      s.status = Status::NumericalError;
    }
    return;
  }
  if (s.status != Status::Optimal) return;
  if (static_cast<int>(s.x.size()) != model.num_cols || static_cast<int>(s.y.size()) != model.num_rows) {
    s.status = Status::NumericalError;
    note(s, "engine reported Optimal without primal and dual vectors");
    return;
  }
  const CheckReport rep = check_solution(model, s.x, s.y);
  s.check = rep.passed() ? "PASS" : "FAIL";
  s.check_primal = rep.max_primal_violation;
  s.check_dual = rep.max_dual_violation;
  s.check_gap = rep.relative_gap;
  if (std::isnan(s.dual_objective)) s.dual_objective = rep.dual_objective;
  if (rep.passed()) return;
  const bool claims_verifier_grade = options.tolerance < 1e-6;
  const std::string what = "in-process check on the original model: " + rep.summary();
  if (claims_verifier_grade) {
    s.status = Status::NumericalError;
    note(s, "Optimal withdrawn, " + what);
  } else {
    note(s, what + " (requested tolerance is looser than the verifier's)");
  }
}

Solution solve_unguarded(const Model& model, const Options& options) {  // solve.cpp:213-259
  Options resolved = options;
  std::string prefix;
  if (options.algorithm == Algorithm::Auto) {
    const double work = static_cast<double>(std::max(model.num_rows, 1)) * static_cast<double>(model.nnz());
    bool first_order_request = options.use_gpu || !options.warm_x.empty() || !options.warm_y.empty() ||
                               options.warm_primal_weight > 0;
    resolved.algorithm = !first_order_request && work <= 2e8 ? Algorithm::Simplex : Algorithm::R2hpdhg;
    char buf[96];
    std::snprintf(buf, sizeof buf, "auto: %s (rows*nnz = %.2g)", alg_name(resolved.algorithm), work);
    prefix = buf;
  }
  Solution s;
  if (resolved.algorithm != Algorithm::R2hpdhg && resolved.algorithm != Algorithm::Pdlp) {
    s.status = Status::NotSolved;
    s.engine = alg_name(resolved.algorithm);
    s.message = std::string("algorithm '") + alg_name(resolved.algorithm) +
                "' is not provided by this library: it runs r2hpdhg and pdlp on the GPU (use_gpu = 1)";
  } else if (!options.use_gpu) {
    s.status = Status::NotSolved;
    s.message = "this library runs r2hpdhg and pdlp on the GPU only: set use_gpu = 1 (there is no CPU fallback)";
  } else {
    bool device = true;
    try {
      require_device();
    } catch (const std::runtime_error& e) {  // cpu_backend.cpp:300-305
      device = false;
      s.status = Status::NotSolved;
      s.message = std::string("CUDA backend unavailable: ") + e.what();
    }
    if (device) {
      s = solve_impl(model, resolved);
      PhaseTimer pt("gate");
      gate(model, resolved, s);
    }
  }
  if (!prefix.empty()) s.message = s.message.empty() ? prefix : prefix + "; " + s.message;
  return s;
}

}  // namespace

void phase_log_begin(bool on) {
  delete g_phases;
  g_phases = on ? new std::vector<std::pair<const char*, double>>() : nullptr;
}
void phase_note(const char* name, double seconds) {
  if (g_phases) g_phases->emplace_back(name, seconds);
}
void phase_log_end(const char* what) {
  if (!g_phases) return;
  std::string line = std::string("ps26119-b200 ") + what + " phases:";
  char buf[96];
  for (const auto& [name, sec] : *g_phases) {
    std::snprintf(buf, sizeof buf, " %s %.1f ms", name, 1e3 * sec);
    line += buf;
  }
  std::fprintf(stderr, "%s\n", line.c_str());
  delete g_phases;
  g_phases = nullptr;
}

Solution solve(const Model& model, const Options& options) {  // solve.cpp:194-210
  try {
    return solve_unguarded(model, options);
  } catch (const std::bad_alloc&) {
    Solution s;
    s.status = Status::NotSolved;
    s.message = "out of memory";
    return s;
  } catch (const std::exception& e) {
    Solution s;
    s.status = Status::NumericalError;
    s.message = std::string("internal error: ") + e.what();
    return s;
  }
}

// ============================================================ batch (batch.cpp:129-441)
std::vector<Solution> solve_batch(const Model& base, const std::vector<Scenario>& scenarios, const Options& options) {
  const auto t0 = clock_t_::now();
  const int K = static_cast<int>(scenarios.size());
  std::vector<Solution> out(K);
  {  // fingerprints of the scenario models (batch.cpp:113-127): the base with the scenario's vectors
    const std::vector<std::uint64_t> fp = scenario_fingerprints(base, scenarios);
    for (int k = 0; k < K; ++k) {
      char buf[17];
      std::snprintf(buf, sizeof buf, "%016llx", static_cast<unsigned long long>(fp[k]));
      out[k].model_fingerprint = buf;
      out[k].engine = "r2hpdhg-batch";
      out[k].precision = "fp64";
    }
  }
  auto fail_all = [&](const std::string& why) {
    for (auto& s : out) s.status = Status::NotSolved, s.message = why;
    return out;
  };
  if (K == 0) return out;
  try {
    if (auto err = base.validate(); !err.empty()) return fail_all("invalid base model: " + err);
    const int m = base.num_rows, n = base.num_cols;
    std::vector<BatchScenarioView> views(K);
    std::vector<int> slots;
    for (int k = 0; k < K; ++k) {  // per-scenario validation (batch.cpp:154-181)
      const Scenario& s = scenarios[k];
      bool ok = true;
      auto pick = [&](const std::vector<double>& v, const std::vector<double>& dflt, std::size_t len) {
        if (v.empty()) return dflt.data();
        ok = ok && v.size() == len;
        return v.data();
      };
      BatchScenarioView& vw = views[k];
      vw.c = pick(s.obj, base.obj, n);
      vw.col_lower = pick(s.col_lower, base.col_lower, n);
      vw.col_upper = pick(s.col_upper, base.col_upper, n);
      vw.row_lower = pick(s.row_lower, base.row_lower, m);
      vw.row_upper = pick(s.row_upper, base.row_upper, m);
      for (int j = 0; ok && j < n; ++j)
        ok = std::isfinite(vw.c[j]) && !std::isnan(vw.col_lower[j]) && !std::isnan(vw.col_upper[j]);
      for (int i = 0; ok && i < m; ++i) ok = !std::isnan(vw.row_lower[i]) && !std::isnan(vw.row_upper[i]);
      bool crossed = false;
      for (int j = 0; ok && !crossed && j < n; ++j) crossed = vw.col_lower[j] > vw.col_upper[j];
      for (int i = 0; ok && !crossed && i < m; ++i) crossed = vw.row_lower[i] > vw.row_upper[i];
      if (!ok) {
        out[k].status = Status::NotSolved;
        out[k].message = "scenario has wrong vector sizes or non-finite data";
      } else if (crossed) {
        out[k].status = Status::Infeasible;
        out[k].message = "bounds cross: scenario has a lower bound above its upper bound";
      } else {
        slots.push_back(k);
      }
    }
    if (slots.empty()) return out;
    require_device();
    EngineOptions eo = engine_options(options);
    // The reference's batch is fp64 only (batch.cpp:136); precision = mixed runs this engine's
    // mixed form (fp32 until every slot reaches the switch, then fp64 to the target).
    std::vector<BatchOutcome> res = run_batch_host(base.view(), views, slots, eo, t0);
    for (int k : slots) {
      BatchOutcome& r = res[k];
      Solution& s = out[k];
      s.status = r.status;
      s.message = r.message;
      s.x = std::move(r.x), s.y = std::move(r.y), s.z = std::move(r.z);
      s.objective = r.objective, s.dual_objective = r.dual_objective;
      s.primal_residual = r.primal_residual, s.dual_residual = r.dual_residual, s.gap = r.gap;
      s.iterations = r.iterations, s.seconds = r.seconds, s.setup_seconds = r.setup_seconds;
      s.iterations_to_fast = r.iterations_to_fast;
      s.primal_weight = r.primal_weight;
      s.engine_result.kernel_launches = r.kernel_launches;
      s.engine_result.iter_kernel_ms = r.spmm_kernel_ms;
      s.engine_result.iter_kernel_launches = r.spmm_launches;
    }
  } catch (const std::bad_alloc&) {
    return fail_all("out of memory");
  } catch (const std::exception& e) {
    const std::string what = e.what();
    return fail_all(what.rfind("no CUDA device", 0) == 0 ? "CUDA backend unavailable: " + what : what);
  }
  return out;
}

}  // namespace b200
