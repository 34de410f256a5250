// parallel.hpp — host-side data parallelism for the dispatcher's O(nnz) passes (presolve,
// postsolve, certification, checks). Work is split into contiguous ranges, one per thread; every
// caller either writes disjoint outputs per range or combines with commutative integer atomics,
// so results do not depend on the thread count.
#pragma once

#include <algorithm>
#include <thread>
#include <vector>

namespace b200 {

// Runs f(begin, end) over [0, n) on up to 32 host threads (inline below `min_parallel`).
template <class F>
void parallel_ranges(long long n, F&& f, long long min_parallel = 65536) {
  const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  const long long T = n < min_parallel ? 1 : std::min<long long>(hw, 32);
  if (T <= 1) {
    f(0LL, n);
    return;
  }
  std::vector<std::thread> th;
  th.reserve(static_cast<std::size_t>(T - 1));
  for (long long t = 1; t < T; ++t) th.emplace_back([&, t] { f(n * t / T, n * (t + 1) / T); });
  f(0LL, n / T);
  for (auto& x : th) x.join();
}

}  // namespace b200
