// tune.hpp — the autotuner's host logic: which launch variant of an iteration kernel a matrix
// gets. The engine times every variant on the matrix itself (CUDA events, a few launches each,
// before the iterates are initialised) the first time it meets a matrix of a shape class, and
// keeps the choice for the life of the process: later solves of that class pay nothing. The
// reference picks its SpMV's threads per row from the mean row length
// (src/gpu/cuda_backend.cu:393-394); this measures instead of guessing.
//
// Environment: PS26119_AUTOTUNE=0 keeps the default variant (index 0) everywhere;
// PS26119_SLAB_VARIANT=k forces variant k (tests run every variant this way).
#pragma once

#include <cmath>
#include <cstdlib>
#include <map>
#include <mutex>
#include <tuple>

namespace b200 {

// A shape class: kernel (0 primal Ãᵀy, 1 dual Ãx̄), working precision (0 fp64, 1 fp32), rows
// rounded to a power of two, and nonzeros per row in quarters.
struct TuneKey {
  int kernel = 0, precision = 0, log2_rows = 0, nnz_per_row_x4 = 0;
  bool operator<(const TuneKey& o) const {
    return std::tie(kernel, precision, log2_rows, nnz_per_row_x4) <
           std::tie(o.kernel, o.precision, o.log2_rows, o.nnz_per_row_x4);
  }
};

inline TuneKey tune_key(int kernel, int precision, long long rows, long long nnz) {
  TuneKey k;
  k.kernel = kernel;
  k.precision = precision;
  long long r = rows > 0 ? rows : 1;
  while (r > 1) r >>= 1, ++k.log2_rows;
  const double per = rows > 0 ? static_cast<double>(nnz) / static_cast<double>(rows) : 0.0;
  k.nnz_per_row_x4 = static_cast<int>(std::lround(per * 4.0));
  return k;
}

// The variant to use given each variant's measured time (ms; non-finite = failed): the fastest,
// unless it beats the default (index 0) by no more than `margin` (relative), in which case the
// default — timings within noise keep the tuned default.
inline int pick_variant(const double* ms, int n, double margin = 0.02) {
  if (n <= 0) return 0;
  int best = -1;
  for (int k = 0; k < n; ++k)
    if (std::isfinite(ms[k]) && ms[k] > 0 && (best < 0 || ms[k] < ms[best])) best = k;
  if (best <= 0) return 0;
  if (!(std::isfinite(ms[0]) && ms[0] > 0)) return best;
  return ms[best] < ms[0] * (1.0 - margin) ? best : 0;
}

// -1: no forced variant; else the index from PS26119_SLAB_VARIANT (read at every call).
inline int tune_forced() {
  const char* e = std::getenv("PS26119_SLAB_VARIANT");
  if (!e || !*e) return -1;
  const int v = std::atoi(e);
  return v >= 0 ? v : -1;
}
inline bool tune_enabled() {
  const char* e = std::getenv("PS26119_AUTOTUNE");
  return !(e && e[0] == '0');
}

// The process's choices by shape class (thread-safe).
class TuneCache {
 public:
  static TuneCache& instance() {
    static TuneCache* c = new TuneCache();
    return *c;
  }
  bool get(const TuneKey& k, int& v) {
    std::lock_guard<std::mutex> lk(mu_);
    auto it = map_.find(k);
    if (it == map_.end()) return false;
    v = it->second;
    return true;
  }
  void put(const TuneKey& k, int v) {
    std::lock_guard<std::mutex> lk(mu_);
    map_[k] = v;
  }

 private:
  std::mutex mu_;
  std::map<TuneKey, int> map_;
};

}  // namespace b200
