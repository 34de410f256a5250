// parallel_copy_check.cpp — test driver for csrc/parallel.hpp: parallel_copy against memcpy on
// random job lists (empty jobs, small ones, and ones above the 4 MiB threading threshold), with
// guard bytes on both sides of every destination; size_for_copy keeps or replaces a buffer as
// documented; parallel_ranges covers every index exactly once when sections run from several
// threads at once (all but one fall back to threads of their own), when a section is started
// inside another, in a child process made by fork() after the pool has started, and when a range
// throws (the exception reaches the caller after every range has run); parallel_tasks runs every
// task once (pool, nested, single), lets a task wait on work items others took, and returns an
// exception after every task has returned. Prints "ok"
// and exits 0, or names the first failure and exits 1.
#include <sys/wait.h>
#include <unistd.h>

#include <atomic>
#include <cstdio>
#include <cstring>
#include <random>
#include <stdexcept>
#include <thread>
#include <vector>

#include "parallel.hpp"

using namespace b200;

int main() {
  std::mt19937_64 rng(5);
  for (int trial = 0; trial < 200; ++trial) {
    const int jobs = 1 + static_cast<int>(rng() % 12);
    std::vector<std::vector<unsigned char>> src(jobs), dst(jobs), want(jobs);
    std::vector<CopyJob> list;
    for (int k = 0; k < jobs; ++k) {
      const std::size_t len = rng() % 4 == 0 ? 0 : (rng() % 3 == 0 ? rng() % (12u << 20) : rng() % 5000);
      src[k].resize(len);
      for (std::size_t q = 0; q < len; q += 8) {  // eight random bytes per draw
        const unsigned long long w = rng();
        std::memcpy(src[k].data() + q, &w, len - q < 8 ? len - q : 8);
      }
      dst[k].assign(len + 64, 0xAB);
      want[k] = dst[k];
      if (len) std::memcpy(want[k].data() + 32, src[k].data(), len);
      list.push_back({dst[k].data() + 32, src[k].data(), len});
    }
    parallel_copy(list.data(), list.size());
    for (int k = 0; k < jobs; ++k)
      if (dst[k] != want[k]) {
        std::printf("mismatch: trial %d job %d\n", trial, k);
        return 1;
      }
  }
  std::vector<double> v(10, 1.0);
  v.reserve(100);
  const double* before = v.data();
  size_for_copy(v, 50);  // fits the capacity: same buffer, old elements kept
  if (v.size() != 50 || v.data() != before || v[9] != 1.0) {
    std::printf("size_for_copy within capacity\n");
    return 1;
  }
  size_for_copy(v, 1000);  // larger: a new buffer of exactly that size
  if (v.size() != 1000) {
    std::printf("size_for_copy beyond capacity\n");
    return 1;
  }
  // every index of [0, n) visited exactly once by a section
  auto covers = [](long long n) {
    std::vector<std::atomic<int>> seen(static_cast<std::size_t>(n));
    for (auto& a : seen) a.store(0);
    parallel_ranges(n, [&](long long b, long long e) {
      for (long long i = b; i < e; ++i) seen[static_cast<std::size_t>(i)].fetch_add(1);
    });
    for (auto& a : seen)
      if (a.load() != 1) return false;
    return true;
  };
  std::atomic<int> bad{0};
  std::vector<std::thread> callers;
  for (int c = 0; c < 4; ++c)
    callers.emplace_back([&] {
      for (int k = 0; k < 50; ++k)
        if (!covers(70000 + 977 * k)) ++bad;
    });
  for (auto& t : callers) t.join();
  if (bad.load()) {
    std::printf("concurrent sections\n");
    return 1;
  }
  std::atomic<long long> inner{0};
  parallel_ranges(100000, [&](long long b, long long e) {  // a section inside a section
    (void)b, (void)e;
    parallel_ranges(70000, [&](long long ib, long long ie) { inner += ie - ib; });
  });
  const long long T = std::min<long long>(std::max(1u, std::thread::hardware_concurrency()), 32);
  if (inner.load() != 70000 * T) {
    std::printf("nested sections: %lld\n", inner.load());
    return 1;
  }
  // an exception thrown in one range reaches the caller (pool path and own-threads path), every
  // range still runs, and the next section covers every index
  for (int nested = 0; nested < 2; ++nested) {
    std::atomic<long long> visited{0};
    bool caught = false;
    auto throwing = [&] {
      parallel_ranges(200000, [&](long long b, long long e) {
        visited += e - b;
        if (b <= 150000 && 150000 < e) throw std::runtime_error("planted");
      });
    };
    try {
      if (nested) parallel_ranges(70000, [&](long long b, long long) { if (b == 0) throwing(); });
      else throwing();
    } catch (const std::runtime_error& e) {
      caught = std::strcmp(e.what(), "planted") == 0;
    }
    if (!caught || visited.load() != 200000 || !covers(90001) || !covers(70000)) {
      std::printf("exception from a range (nested %d): caught %d, visited %lld\n", nested, caught ? 1 : 0,
                  visited.load());
      return 1;
    }
  }
  // parallel_tasks: every task index runs once, on the pool, nested (threads of its own) and as a
  // single task; a task that takes shared work items from a counter and waits only for items
  // another task has taken finishes in every case; an exception reaches the caller after every
  // task has returned
  auto tasks_ok = [](int T) {
    std::vector<std::atomic<int>> ran(static_cast<std::size_t>(T));
    for (auto& a : ran) a.store(0);
    constexpr int kItems = 97;
    std::vector<std::atomic<int>> done(kItems);
    for (auto& a : done) a.store(0);
    std::atomic<int> next{0};
    long long order_sum = 0;  // task 0 consumes the items in index order
    parallel_tasks(T, [&](int t) {
      ran[static_cast<std::size_t>(t)].fetch_add(1);
      auto take = [&] {
        const int k = next.fetch_add(1);
        if (k >= kItems) return false;
        done[static_cast<std::size_t>(k)].store(1, std::memory_order_release);
        return true;
      };
      if (t != 0) {
        while (take()) {
        }
        return;
      }
      for (int k = 0; k < kItems; ++k) {
        while (done[static_cast<std::size_t>(k)].load(std::memory_order_acquire) == 0)
          if (!take()) std::this_thread::yield();
        order_sum += k;
      }
    });
    for (auto& a : ran)
      if (a.load() != 1) return false;
    return order_sum == static_cast<long long>(kItems) * (kItems - 1) / 2;
  };
  if (!tasks_ok(1) || !tasks_ok(8) || !tasks_ok(static_cast<int>(T))) {
    std::printf("parallel_tasks\n");
    return 1;
  }
  std::atomic<int> nested_ok{0};
  parallel_ranges(100000, [&](long long, long long) { nested_ok += tasks_ok(4) ? 1 : 0; });
  if (nested_ok.load() != T) {
    std::printf("parallel_tasks nested: %d\n", nested_ok.load());
    return 1;
  }
  {
    std::atomic<int> returned{0};
    bool caught = false;
    try {
      parallel_tasks(6, [&](int t) {
        ++returned;
        if (t == 3) throw std::runtime_error("planted task");
      });
    } catch (const std::runtime_error& e) {
      caught = std::strcmp(e.what(), "planted task") == 0;
    }
    if (!caught || returned.load() != 6 || !covers(70000)) {
      std::printf("exception from a task: caught %d, returned %d\n", caught ? 1 : 0, returned.load());
      return 1;
    }
  }
  const pid_t pid = fork();
  if (pid == 0) _exit(covers(123457) && covers(70001) ? 0 : 1);  // the child's own pool
  int status = 0;
  if (pid < 0 || waitpid(pid, &status, 0) != pid || !WIFEXITED(status) || WEXITSTATUS(status) != 0) {
    std::printf("sections in a forked child\n");
    return 1;
  }
  std::printf("ok\n");
  return 0;
}
