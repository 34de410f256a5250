// parallel.hpp — host-side data parallelism for the dispatcher's O(nnz) passes (presolve,
// postsolve, certification, checks). Work is split into contiguous ranges, one per thread; every
// caller either writes disjoint outputs per range or combines with commutative integer atomics,
// so results do not depend on the thread count.
#pragma once

#include <algorithm>
#include <cstring>
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

// One host-to-host copy of `bytes` bytes (non-overlapping buffers).
struct CopyJob {
  void* dst;
  const void* src;
  std::size_t bytes;
};

// Runs every job, the bytes of all jobs split evenly over the host threads (one team for the
// whole list, inline below 4 MiB in total). The destination bytes equal the source bytes
// whatever the thread count.
inline void parallel_copy(const CopyJob* jobs, std::size_t count) {
  std::size_t total = 0;
  for (std::size_t k = 0; k < count; ++k) total += jobs[k].bytes;
  parallel_ranges(
      static_cast<long long>(total),
      [&](long long b, long long e) {
        std::size_t off = 0;  // start of job k in the concatenation of all jobs
        for (std::size_t k = 0; k < count && off < static_cast<std::size_t>(e); off += jobs[k].bytes, ++k) {
          const std::size_t lo = std::max<std::size_t>(static_cast<std::size_t>(b), off);
          const std::size_t hi = std::min<std::size_t>(static_cast<std::size_t>(e), off + jobs[k].bytes);
          if (lo < hi)
            std::memcpy(static_cast<char*>(jobs[k].dst) + (lo - off), static_cast<const char*>(jobs[k].src) + (lo - off),
                        hi - lo);
        }
      },
      4LL << 20);
}

// Sets v's size to n without copying the old elements over, ready to be overwritten by a
// parallel_copy: resizing to the size it already has writes nothing.
template <class T>
void size_for_copy(std::vector<T>& v, std::size_t n) {
  if (n > v.capacity()) std::vector<T>().swap(v), v.reserve(n);
  v.resize(n);
}

}  // namespace b200
