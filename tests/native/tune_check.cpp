// tune_check.cpp — test driver for csrc/tune.hpp, the autotuner's host logic: the variant picked
// from measured times (fastest, but the default within a 2% margin; failed timings ignored), the
// shape classes (rows by power of two, nonzeros per row by quarters), the forced-variant and
// disable switches, and the process cache. Prints "ok" and exits 0, or names the first failure.
#include <cmath>
#include <cstdio>
#include <cstdlib>

#include "tune.hpp"

using namespace b200;

static int fail(const char* what) {
  std::printf("%s\n", what);
  return 1;
}

int main() {
  const double inf = INFINITY, nan = NAN;
  {
    const double ms[] = {10.0, 9.0, 11.0};
    if (pick_variant(ms, 3) != 1) return fail("fastest variant");
  }
  {
    const double ms[] = {10.0, 9.9, 11.0};  // 1% faster: within the margin, keep the default
    if (pick_variant(ms, 3) != 0) return fail("margin keeps the default");
  }
  {
    const double ms[] = {10.0, nan, 8.0, inf, -1.0};  // failed timings never win
    if (pick_variant(ms, 5) != 2) return fail("non-finite timings ignored");
  }
  {
    const double ms[] = {nan, 5.0, 4.0};  // the default failed: the fastest of the rest
    if (pick_variant(ms, 3) != 2) return fail("failed default");
  }
  {
    const double ms[] = {nan, nan};
    if (pick_variant(ms, 2) != 0 || pick_variant(ms, 0) != 0) return fail("nothing measured");
  }
  const TuneKey a = tune_key(0, 0, 1000000, 6000000), b = tune_key(0, 0, 1048575, 6291450);
  if (a.log2_rows != 19 || a.nnz_per_row_x4 != 24 || a < b || b < a) return fail("shape class of the 1M LP");
  const TuneKey c = tune_key(1, 0, 1000000, 6000000), d = tune_key(0, 1, 1000000, 6000000);
  if (!(a < c || c < a) || !(a < d || d < a)) return fail("kernel and precision separate classes");
  if (tune_key(0, 0, 0, 0).log2_rows != 0) return fail("empty matrix");
  unsetenv("PS26119_SLAB_VARIANT");
  unsetenv("PS26119_AUTOTUNE");
  if (tune_forced() != -1 || !tune_enabled()) return fail("defaults");
  setenv("PS26119_SLAB_VARIANT", "3", 1);
  setenv("PS26119_AUTOTUNE", "0", 1);
  if (tune_forced() != 3 || tune_enabled()) return fail("switches");
  TuneCache& cache = TuneCache::instance();
  int v = -1;
  if (cache.get(a, v)) return fail("empty cache");
  cache.put(a, 2);
  if (!cache.get(b, v) || v != 2 || cache.get(c, v)) return fail("cache by class");
  std::printf("ok\n");
  return 0;
}
