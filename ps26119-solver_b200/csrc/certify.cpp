// certify.cpp — see certify.hpp. Reference files restated: src/core/safe_bound.cpp:1-197,
// src/core/implied_bounds.cpp:1-114, src/core/certificates.cpp:1-138; the double-double
// arithmetic follows the published algorithms cited below (the reference's src/la/dd.h uses the
// same ones, so the results agree bit for bit).
//
// Double-double (value = hi + lo, |lo| ≤ ulp(hi)/2):
//   two_sum        Knuth, TAOCP vol. 2 §4.2.2 (error-free sum)
//   exact product  fma(a, b, −a·b) is the rounding error of a·b (exact unless it underflows)
//   dd + dd        Hida, Li & Bailey, "Library for double-double and quad-double arithmetic"
//                  (the "IEEE" accurate addition: two_sum of both halves, two renormalisations)
//   dd / dd        long division with three partial quotients (same library)
//   expansions     Shewchuk, "Adaptive precision floating-point arithmetic" (1997), GROW-EXPANSION
//                  with zero elimination
#include "certify.hpp"
#include "parallel.hpp"
#include "solver.hpp"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <limits>
#include <memory>
#include <thread>

namespace b200 {
namespace {

constexpr double kVerifyRay = 1e-8;  // tolerances.h:43

// ------------------------------------------------------------------ double-double
struct DD {
  double hi = 0.0, lo = 0.0;
};
inline void two_sum(double a, double b, double& s, double& e) {
  s = a + b;
  const double bb = s - a;
  e = (a - (s - bb)) + (b - bb);
}
inline void fast_two_sum(double a, double b, double& s, double& e) {  // |a| ≥ |b| or a = 0
  s = a + b;
  e = b - (s - a);
}
inline DD exact_product(double a, double b) {
  DD r;
  r.hi = a * b;
  r.lo = std::fma(a, b, -r.hi);
  return r;
}
inline DD operator+(const DD& a, const DD& b) {
  double s1, s2, t1, t2;
  two_sum(a.hi, b.hi, s1, s2);
  two_sum(a.lo, b.lo, t1, t2);
  s2 += t1;
  fast_two_sum(s1, s2, s1, s2);
  s2 += t2;
  DD r;
  fast_two_sum(s1, s2, r.hi, r.lo);
  return r;
}
inline DD operator+(const DD& a, double b) {
  double s1, s2;
  two_sum(a.hi, b, s1, s2);
  s2 += a.lo;
  DD r;
  fast_two_sum(s1, s2, r.hi, r.lo);
  return r;
}
inline DD operator-(const DD& a) { return {-a.hi, -a.lo}; }
inline DD operator-(const DD& a, const DD& b) { return a + (-b); }
inline DD operator*(const DD& a, double b) {
  double p1 = a.hi * b;
  double p2 = std::fma(a.hi, b, -p1);
  p2 += a.lo * b;
  DD r;
  fast_two_sum(p1, p2, r.hi, r.lo);
  return r;
}
inline DD operator/(const DD& a, const DD& b) {
  const double q1 = a.hi / b.hi;
  if (!std::isfinite(q1)) return {q1, 0.0};
  DD r = a - b * q1;
  const double q2 = r.hi / b.hi;
  r = r - b * q2;
  const double q3 = r.hi / b.hi;
  DD q;
  fast_two_sum(q1, q2, q.hi, q.lo);
  return q + q3;
}
inline DD dd_of(double v) { return {v, 0.0}; }
inline double value(const DD& a) { return a.hi + a.lo; }
inline bool operator<(const DD& a, const DD& b) { return a.hi < b.hi || (a.hi == b.hi && a.lo < b.lo); }

// ------------------------------------------------------------------ rigorous rounding
// A dd addition has relative error ≤ 2⁻¹⁰⁴ of its result; products are exact unless they
// underflow (an absolute slack per term covers that). Both are doubled for margin.
constexpr double kRel = 2.0 * 4.930380657631324e-32;  // 2 · 2⁻¹⁰⁴
constexpr double kAbs = 2.0 * 1.0e-289;               // ≥ 2 · 2⁻⁹⁶⁰

double round_down(const DD& v, double err) {  // a double ≤ v − err (exact values pass through)
  if (err == 0.0 && v.lo == 0.0) return v.hi;
  return std::nextafter(value(v - dd_of(err)), -std::numeric_limits<double>::infinity());
}
double round_up(const DD& v, double err) {
  if (err == 0.0 && v.lo == 0.0) return v.hi;
  return std::nextafter(value(v + dd_of(err)), std::numeric_limits<double>::infinity());
}
bool may_underflow(const DD& p) { return p.hi != 0.0 && std::fabs(p.hi) < 1e-280; }

// Exact sum as a nonoverlapping expansion (GROW-EXPANSION, zero elimination), in a fixed array
// updated in place (component k is read before any write at an index ≤ k). grow() returns
// false on a non-finite value or an expansion longer than 64 components (the caller then keeps
// its interval).
struct Expansion {
  double c[66];
  int n = 0;
  bool grow(double b) {
    if (b == 0.0) return true;
    if (!std::isfinite(b)) return false;
    double q = b;
    int w = 0;
    for (int k = 0; k < n; ++k) {
      const double ei = c[k];
      const double sum = q + ei;
      const double bv = sum - q;
      const double av = sum - bv;
      const double err = (q - av) + (ei - bv);
      q = sum;
      c[w] = err;  // kept only when nonzero; stored either way (no branch on the data)
      w += err != 0.0;
    }
    n = w;
    if (!std::isfinite(q)) return false;
    c[n] = q;  // n ≤ 64 here: the array has room
    n += q != 0.0;
    return n <= 64;
  }
};

// min over x ∈ [lo, hi] of z·x as an exact product; `inf` when it is −∞.
DD min_term(double z, double lo, double hi, bool& inf) {
  if (z > 0) {
    if (!std::isfinite(lo)) return inf = true, DD{};
    return exact_product(z, lo);
  }
  if (z < 0) {
    if (!std::isfinite(hi)) return inf = true, DD{};
    return exact_product(z, hi);
  }
  return DD{};
}

// Accumulates dd terms with a running bound on the rounding error.
struct SafeSum {
  DD sum;
  double abs_sum = 0.0;
  long long count = 0;
  void add(const DD& t) {
    sum = sum + t;
    abs_sum += std::fabs(value(t));
    ++count;
  }
  double error() const { return static_cast<double>(count + 2) * (kRel * abs_sum * 1.0000001 + kAbs); }
};

// The bound for multipliers y (already cleared where they point at an infinite row bound) and
// column bounds [col_lo, col_up] (safe_bound.cpp:92-173).
// The per-column term arrays and the cleared multipliers of this thread, kept between calls
// within the host reuse limit (host_keep in solver.hpp).
struct CertifyScratch {
  std::vector<DD> col_term;
  std::vector<char> col_inf;
  std::vector<double> y;
  std::size_t accounted = 0;
  std::size_t bytes() const { return sizeof(DD) * col_term.capacity() + col_inf.capacity() + 8 * y.capacity(); }
  void release() {
    std::vector<DD>().swap(col_term);
    std::vector<char>().swap(col_inf);
    std::vector<double>().swap(y);
  }
  ~CertifyScratch() { host_keep(accounted, 0); }
};
thread_local CertifyScratch t_certify;

SafeBound bound_with(const Model& M, const std::vector<double>& y, const std::vector<double>& col_lo,
                     const std::vector<double>& col_up) {
  SafeBound r;
  const int m = M.num_rows, n = M.num_cols;
  const double sense = M.sense;
  if (static_cast<int>(y.size()) != m) return r;
  // per-column terms min over the enclosure [z_lo, z_hi] of z_j x_j, independent per column
  std::vector<DD>& col_term = t_certify.col_term;
  std::vector<char>& col_inf = t_certify.col_inf;
  size_for_copy(col_term, static_cast<std::size_t>(n));  // every entry is written below before it is read
  size_for_copy(col_inf, static_cast<std::size_t>(n));
  auto columns = [&](long long jb, long long je, Expansion& ex) {
    for (long long jj = jb; jj < je; ++jj) {
      const int j = static_cast<int>(jj);
      if (jj + 2 < je)  // the multipliers of the column after next: random reads, started early
        for (int p = M.col_start[j + 2]; p < M.col_start[j + 3]; ++p) __builtin_prefetch(&y[M.row_index[p]]);
      DD z = dd_of(sense * M.obj[j]);
      double mag = 0.0;  // Σ|terms| after the first (exact) assignment
      int cnt = 0;
      bool uf = false;
      for (int p = M.col_start[j]; p < M.col_start[j + 1]; ++p) {
        const DD prod = exact_product(M.value[p], sense * y[M.row_index[p]]);
        if (prod.hi == 0.0 && prod.lo == 0.0 && M.value[p] * y[M.row_index[p]] == 0.0) continue;  // exact zero
        z = z - prod;
        mag += std::fabs(value(prod)) + std::fabs(value(z));
        uf = uf || may_underflow(prod);
        ++cnt;
      }
      const double ez = cnt == 0 ? 0.0 : (cnt + 2) * (kRel * mag * 1.0000001 + (uf ? kAbs : 0.0));
      double zlo = round_down(z, ez), zhi = round_up(z, ez);
      if (cnt > 0 && !uf) {
        // tighter, still rigorous: z exactly as an expansion (exact cancellation gives exactly 0,
        // a one-component expansion is an exact double, otherwise enclose its dd sum)
        ex.n = 0;
        bool ok = ex.grow(sense * M.obj[j]);
        for (int p = M.col_start[j]; ok && p < M.col_start[j + 1]; ++p) {
          const DD prod = exact_product(M.value[p], sense * y[M.row_index[p]]);
          ok = ex.grow(-prod.hi) && ex.grow(-prod.lo);
        }
        if (ok) {
          if (ex.n == 0) {
            zlo = zhi = 0.0;
          } else if (ex.n == 1) {
            zlo = zhi = ex.c[0];
          } else {
            DD v;
            for (int k = 0; k < ex.n; ++k) v = v + ex.c[k];  // smallest component first
            const double ev = static_cast<double>(ex.n + 2) * kRel * std::fabs(value(v)) * 1.0000001;
            zlo = std::max(zlo, round_down(v, ev));
            zhi = std::min(zhi, round_up(v, ev));
          }
        }
      }
      bool inf_lo = false, inf_hi = false;
      const DD tlo = min_term(zlo, col_lo[j], col_up[j], inf_lo);
      const DD thi = min_term(zhi, col_lo[j], col_up[j], inf_hi);
      col_inf[j] = (inf_lo || inf_hi) ? 1 : 0;
      if (col_inf[j]) continue;
      col_term[j] = tlo < thi ? tlo : thi;
    }
  };
  // The sum in the reference's order: rows, then columns. The columns are cut into chunks taken
  // in index order from a shared counter by every task; task 0 first sums the rows, then sums
  // each chunk's terms in order as soon as the chunk is done, taking chunks itself while the one
  // it needs is not started, so the sequential sum runs beside the column pass instead of after
  // it. The operations and their order are those of a column pass followed by the sum.
  constexpr long long kChunkCols = 8192;
  const long long nchunks = (static_cast<long long>(n) + kChunkCols - 1) / kChunkCols;
  std::unique_ptr<std::atomic<int>[]> done(new std::atomic<int>[static_cast<std::size_t>(std::max(1LL, nchunks))]);
  for (long long k = 0; k < nchunks; ++k) done[k].store(0, std::memory_order_relaxed);
  std::atomic<long long> next{0};
  std::atomic<bool> failed{false};
  auto take_one = [&](Expansion& ex) {  // false: no chunk left to take
    const long long k = next.fetch_add(1, std::memory_order_relaxed);
    if (k >= nchunks) return false;
    try {
      columns(k * kChunkCols, std::min<long long>(n, (k + 1) * kChunkCols), ex);
    } catch (...) {
      failed.store(true);
      done[k].store(1, std::memory_order_release);
      throw;
    }
    done[k].store(1, std::memory_order_release);
    return true;
  };
  SafeSum L;
  const int T = n < 65536 ? 1 : static_cast<int>(std::min<long long>(nchunks, host_thread_limit()));
  parallel_tasks(T, [&](int t) {
    Expansion ex;
    if (t != 0) {
      while (!failed.load(std::memory_order_relaxed) && take_one(ex)) {
      }
      return;
    }
    for (int i = 0; i < m; ++i) {
      bool inf = false;
      const DD tr = min_term(sense * y[i], M.row_lower[i], M.row_upper[i], inf);
      if (inf) ++r.unbounded_row_terms;
      else L.add(tr);
    }
    for (long long k = 0; k < nchunks; ++k) {
      while (done[k].load(std::memory_order_acquire) == 0) {
        if (failed.load()) return;
        if (!take_one(ex)) std::this_thread::yield();  // chunk k is being computed by another task
      }
      if (failed.load()) return;
      const long long je = std::min<long long>(n, (k + 1) * kChunkCols);
      for (long long j = k * kChunkCols; j < je; ++j) {
        if (col_inf[j]) ++r.unbounded_col_terms;
        else L.add(col_term[j]);
      }
    }
  });
  if (r.unbounded_row_terms > 0 || r.unbounded_col_terms > 0) {
    r.finite = false;
    r.bound = sense > 0 ? -std::numeric_limits<double>::infinity() : std::numeric_limits<double>::infinity();
    return r;
  }
  // L bounds min c̃ᵀx from below: MIN optimum ≥ L + offset; MAX optimum = −min(−cᵀx) ≤ −L + offset
  const double err = L.error() + kAbs;
  r.finite = true;
  if (sense > 0) r.bound = round_down(L.sum + dd_of(M.obj_offset), err + kRel * std::fabs(M.obj_offset) * 4);
  else r.bound = round_up(-L.sum + dd_of(M.obj_offset), err + kRel * std::fabs(M.obj_offset) * 4);
  return r;
}

}  // namespace

SafeBound certified_dual_bound(const Model& M, const std::vector<double>& y_in, bool use_implied_bounds) {
  if (static_cast<int>(y_in.size()) != M.num_rows) return SafeBound{};
  // valid for ANY multipliers: clear those that point at an infinite row bound (safe_bound.cpp:178-187)
  struct KeepScratch {
    ~KeepScratch() {
      if (!host_keep(t_certify.accounted, t_certify.bytes())) t_certify.release();
    }
  } keep;
  std::vector<double>& y = t_certify.y;
  size_for_copy(y, y_in.size());
  parallel_ranges(M.num_rows, [&](long long ib, long long ie) {  // element-wise, on the host threads
    for (long long i = ib; i < ie; ++i) {
      const double ym = M.sense * y_in[i];
      const bool clear = (ym > 0 && !std::isfinite(M.row_lower[i])) || (ym < 0 && !std::isfinite(M.row_upper[i]));
      y[i] = clear ? 0.0 : y_in[i];
    }
  });
  SafeBound r = bound_with(M, y, M.col_lower, M.col_upper);
  if (use_implied_bounds && r.unbounded_col_terms > 0 && r.unbounded_row_terms == 0) {
    const ImpliedBounds ib = implied_bounds(M);
    r = bound_with(M, y, ib.lower, ib.upper);
  }
  return r;
}

ImpliedBounds implied_bounds(const Model& M, int max_passes) {  // implied_bounds.cpp:23-112
  constexpr double kSlack = 1e-9;
  const double kInfD = std::numeric_limits<double>::infinity();
  auto loosen_up = [&](double v, double scale) { return std::nextafter(v + kSlack * (scale + std::fabs(v)), kInfD); };
  auto loosen_down = [&](double v, double scale) { return std::nextafter(v - kSlack * (scale + std::fabs(v)), -kInfD); };
  ImpliedBounds r;
  r.lower = M.col_lower;
  r.upper = M.col_upper;
  auto& lo = r.lower;
  auto& up = r.upper;
  const int m = M.num_rows, n = M.num_cols;
  // row access: CSR of A with columns increasing inside each row (la::csr_from_model)
  std::vector<int> rp(static_cast<std::size_t>(m) + 1, 0), rc(M.nnz());
  std::vector<double> rv(M.nnz());
  for (std::size_t k = 0; k < M.nnz(); ++k) ++rp[M.row_index[k] + 1];
  for (int i = 0; i < m; ++i) rp[i + 1] += rp[i];
  {
    std::vector<int> next(rp.begin(), rp.end() - 1);
    for (int j = 0; j < n; ++j)
      for (int k = M.col_start[j]; k < M.col_start[j + 1]; ++k) {
        const int p = next[M.row_index[k]]++;
        rc[p] = j;
        rv[p] = M.value[k];
      }
  }
  // worklist: a row is re-examined only after one of its columns' bounds changed
  std::vector<char> dirty(static_cast<std::size_t>(m), 1);
  auto touch = [&](int j) {
    for (int k = M.col_start[j]; k < M.col_start[j + 1]; ++k) dirty[M.row_index[k]] = 1;
  };
  for (int pass = 0; pass < max_passes; ++pass) {
    bool changed = false;
    for (int i = 0; i < m; ++i) {
      if (!dirty[i]) continue;
      dirty[i] = 0;
      const bool has_up = std::isfinite(M.row_upper[i]), has_lo = std::isfinite(M.row_lower[i]);
      if (!has_up && !has_lo) continue;
      DD amin, amax;
      double mag = 0.0;
      int ninf_min = 0, ninf_max = 0, jinf_min = -1, jinf_max = -1;
      for (int p = rp[i]; p < rp[i + 1]; ++p) {
        const int j = rc[p];
        const double a = rv[p];
        const double bmin = a > 0 ? lo[j] : up[j], bmax = a > 0 ? up[j] : lo[j];
        if (std::isfinite(bmin)) {
          const DD t = exact_product(a, bmin);
          amin = amin + t;
          mag += std::fabs(value(t));
        } else {
          ++ninf_min, jinf_min = j;
        }
        if (std::isfinite(bmax)) {
          const DD t = exact_product(a, bmax);
          amax = amax + t;
          mag += std::fabs(value(t));
        } else {
          ++ninf_max, jinf_max = j;
        }
      }
      for (int p = rp[i]; p < rp[i + 1]; ++p) {
        const int j = rc[p];
        const double a = rv[p];
        const double scale = mag / std::fabs(a);
        if (has_up && (ninf_min == 0 || (ninf_min == 1 && jinf_min == j))) {  // a x_j ≤ ru − rest
          const double bmin = a > 0 ? lo[j] : up[j];
          DD rest = amin;
          if (ninf_min == 0) rest = rest - exact_product(a, bmin);
          const double v = value((dd_of(M.row_upper[i]) - rest) / dd_of(a));
          if (a > 0) {
            const double nb = loosen_up(v, scale);
            if (nb < up[j] - 1e-7 * (1 + std::fabs(nb))) up[j] = nb, changed = true, touch(j);
          } else {
            const double nb = loosen_down(v, scale);
            if (nb > lo[j] + 1e-7 * (1 + std::fabs(nb))) lo[j] = nb, changed = true, touch(j);
          }
        }
        if (has_lo && (ninf_max == 0 || (ninf_max == 1 && jinf_max == j))) {  // a x_j ≥ rl − rest
          const double bmax = a > 0 ? up[j] : lo[j];
          DD rest = amax;
          if (ninf_max == 0) rest = rest - exact_product(a, bmax);
          const double v = value((dd_of(M.row_lower[i]) - rest) / dd_of(a));
          if (a > 0) {
            const double nb = loosen_down(v, scale);
            if (nb > lo[j] + 1e-7 * (1 + std::fabs(nb))) lo[j] = nb, changed = true, touch(j);
          } else {
            const double nb = loosen_up(v, scale);
            if (nb < up[j] - 1e-7 * (1 + std::fabs(nb))) up[j] = nb, changed = true, touch(j);
          }
        }
      }
    }
    if (!changed) break;
  }
  for (int j = 0; j < n; ++j) {
    if (!std::isfinite(M.col_lower[j]) && std::isfinite(lo[j])) ++r.tightened;
    if (!std::isfinite(M.col_upper[j]) && std::isfinite(up[j])) ++r.tightened;
  }
  return r;
}

namespace {

// The interval part of the Farkas tolerance test. A multiplier t on a row (t = r_i) or a column
// (t = −(Aᵀr)_j) picks the lower bound when positive and the upper bound when negative; a
// picked bound that is finite adds t·bound to the certificate's objective and a magnitude term
// to its scale, an infinite one is a violation of size |t|. Zero (and NaN) multipliers pick
// nothing. Terms are taken in the order the caller offers them.
struct FarkasTally {
  double obj = 0.0, mag = 0.0, viol = 0.0;
  template <class Magnitude>
  void take(double t, double lo, double hi, Magnitude&& magnitude) {
    if (!(t > 0) && !(t < 0)) return;
    const double bound = t > 0 ? lo : hi;
    if (std::isfinite(bound)) {
      obj += t * bound;
      mag += magnitude(bound);
    } else {
      viol = std::max(viol, t > 0 ? t : -t);
    }
  }
};

// Largest step a direction value v takes outside the finite sides of an interval: −v past a
// finite lower side, then v past a finite upper side (in that order).
inline double widen(double viol, double v, double lo, double hi) {
  if (std::isfinite(lo)) viol = std::max(viol, -v);
  if (std::isfinite(hi)) viol = std::max(viol, v);
  return viol;
}

std::string format_detail(const char* fmt, ...) {
  char buf[200];
  va_list ap;
  va_start(ap, fmt);
  std::vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  return buf;
}

}  // namespace

// A Farkas vector r proves infeasibility when the best objective of the zero-cost model bounded
// through r is positive. First the rounding-proof way: the certified bound of the model with its
// objective set to zero, from multipliers r. Failing that, the fp64 tolerance test: the tally of
// r over the row intervals, then of −Aᵀr over the column intervals, scaled by max(‖r‖∞,
// violation) (reference src/core/certificates.cpp:14-86; the same terms in the same order).
CertificateCheck check_infeasibility_certificate(const Model& model, const std::vector<double>& r) {
  CertificateCheck c;
  const int m = model.num_rows, n = model.num_cols;
  if (static_cast<int>(r.size()) != m || m == 0) {
    c.detail = "no dual ray";
    return c;
  }
  c.present = true;
  if (!std::all_of(r.begin(), r.end(), [](double v) { return std::isfinite(v); })) {
    c.detail = "dual ray is not finite";
    return c;
  }
  Model zero = model;
  zero.sense = 1;
  zero.obj_offset = 0.0;
  std::fill(zero.obj.begin(), zero.obj.end(), 0.0);
  const SafeBound sb = certified_dual_bound(zero, r);
  if (sb.finite && sb.bound > 0.0) {
    c.passed = c.rigorous = true;
    c.measure = sb.bound;
    c.detail = format_detail("Farkas certificate: certified L0(r) = %.3g > 0 (rounding-proof)", sb.bound);
    return c;
  }
  FarkasTally tally;
  double rmax = 0.0;
  for (int i = 0; i < m; ++i) {
    rmax = std::max(rmax, std::fabs(r[i]));
    tally.take(r[i], model.row_lower[i], model.row_upper[i], [&](double bound) { return std::fabs(r[i] * bound); });
  }
  for (int j = 0; j < n; ++j) {
    double atr = 0.0, atr_abs = 0.0;  // (Aᵀr)_j and Σ|a_ij r_i|, in the column's entry order
    for (int k = model.col_start[j]; k < model.col_start[j + 1]; ++k) {
      const double p = model.value[k] * r[model.row_index[k]];
      atr += p;
      atr_abs += std::fabs(p);
    }
    tally.take(-atr, model.col_lower[j], model.col_upper[j], [&](double bound) { return atr_abs * std::fabs(bound); });
  }
  const double scale = std::max(rmax, tally.viol);
  c.measure = scale > 0 ? tally.obj / scale : 0.0;
  c.violation = scale > 0 ? tally.viol / scale : 0.0;
  const bool positive = std::isfinite(c.measure) && c.measure > 0;
  const bool above_noise = tally.obj > kVerifyRay * tally.mag;
  const bool small_violation = c.violation <= kVerifyRay * c.measure;
  c.passed = positive && above_noise && small_violation;
  c.detail = format_detail(
      "Farkas certificate: rigorous L0(r) = %.3g; tolerance test L0/s = %.3g, violation/s = %.3g, "
      "L0/sum|terms| = %.3g (%s)",
      sb.bound, c.measure, c.violation, tally.mag > 0 ? tally.obj / tally.mag : 0.0,
      c.passed ? "infeasibility shown within tolerance, not rounding-proof" : "FAIL");
  return c;
}

// A point x and a ray prove unboundedness when x is feasible (the gate's primal test) and the
// ray, scaled to ‖d‖∞ = 1, lowers the objective by at least the ray tolerance while leaving the
// recession cone by at most that tolerance relative to the decrease (reference
// src/core/certificates.cpp:88-136; the same terms in the same order).
CertificateCheck check_unboundedness_certificate(const Model& model, const std::vector<double>& x,
                                                 const std::vector<double>& ray) {
  CertificateCheck c;
  const int m = model.num_rows, n = model.num_cols;
  if (static_cast<int>(ray.size()) != n || static_cast<int>(x.size()) != n || n == 0) {
    c.detail = "no primal ray / point";
    return c;
  }
  c.present = true;
  double dmax = 0.0, cmax = 0.0;
  for (int j = 0; j < n; ++j) {
    if (!std::isfinite(ray[j]) || !std::isfinite(x[j])) {
      c.detail = "ray or point is not finite";
      return c;
    }
    dmax = std::max(dmax, std::fabs(ray[j]));
    cmax = std::max(cmax, std::fabs(model.obj[j]));
  }
  if (dmax == 0.0) {
    c.detail = "zero ray";
    return c;
  }
  const CheckReport point = check_solution(model, x, std::vector<double>(m, 0.0));
  std::vector<double> d(n);
  double slope = 0.0, cone = 0.0;  // c'd in the model's sense; the largest step out of the cone
  for (int j = 0; j < n; ++j) {
    d[j] = ray[j] / dmax;
    slope += model.sense * model.obj[j] * d[j];
    cone = widen(cone, d[j], model.col_lower[j], model.col_upper[j]);
  }
  const std::vector<double> ad = model.row_activity(d);
  for (int i = 0; i < m; ++i) cone = widen(cone, ad[i], model.row_lower[i], model.row_upper[i]);
  c.measure = -slope;
  c.violation = cone;
  const bool decreases = -slope >= kVerifyRay * std::max(1.0, cmax);
  const bool in_cone = cone <= kVerifyRay * (-slope);
  c.passed = point.primal_ok && decreases && in_cone;
  c.detail = format_detail("unbounded ray: -c'd = %.3g, cone violation %.3g, point primal violation %.3g (%s)",
                           -slope, cone, point.max_primal_violation, c.passed ? "unboundedness proven" : "FAIL");
  return c;
}

}  // namespace b200
