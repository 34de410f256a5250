// parallel.hpp — host-side data parallelism for the dispatcher's O(nnz) passes (presolve,
// postsolve, certification, checks). Work is split into contiguous ranges, one per thread; every
// caller either writes disjoint outputs per range or combines with commutative integer atomics,
// so results do not depend on the thread count.
#pragma once

#include <pthread.h>

#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <mutex>
#include <system_error>
#include <thread>
#include <vector>

namespace b200 {

// The host threads one parallel section may use: every hardware thread, at most 32, or fewer
// when the environment variable PS26119_HOST_THREADS gives a smaller positive number (read once).
// Results do not depend on it.
inline int host_thread_limit() {
  static const int limit = [] {
    const int hw = static_cast<int>(std::max(1u, std::thread::hardware_concurrency()));
    int t = std::min(hw, 32);
    if (const char* env = std::getenv("PS26119_HOST_THREADS")) {
      const int want = std::atoi(env);
      if (want > 0) t = std::min(t, want);
    }
    return t;
  }();
  return limit;
}

// Worker threads kept for the life of the process, so that a parallel section costs a wake-up
// instead of creating and joining its threads (about 270 µs per section for 8 threads on an
// 8-core host; a solve runs some 40 sections). One section uses the pool at a time: a section
// started while the pool is busy (another thread's), or from inside a pool worker, returns
// false from run() and its caller uses threads of its own. The pool is never destroyed (its
// workers wait for work until the process ends), and a child process made by fork() starts a
// new pool on first use, as the parent's workers do not exist there.
class HostPool {
 public:
  static HostPool& instance() {
    HostPool* p = slot().load(std::memory_order_acquire);
    if (!p) {
      HostPool* fresh = new HostPool();
      if (slot().compare_exchange_strong(p, fresh, std::memory_order_acq_rel)) p = fresh;
      else delete fresh;  // another thread made it first (no worker started yet)
      static std::atomic<bool> registered{false};
      if (!registered.exchange(true)) pthread_atfork(nullptr, nullptr, [] { slot().store(nullptr); });
    }
    return *p;
  }

  // Runs task(t) for every t in [0, T): t = 0 and any task no worker could be started for on the
  // calling thread, the others on workers. Returns when all have finished; false, having run
  // nothing, when the pool is busy or the caller is one of its workers.
  bool run(int T, const std::function<void(int)>& task) {
    if (in_worker() || !use_.try_lock()) return false;
    std::lock_guard<std::mutex> own(use_, std::adopt_lock);
    while (static_cast<int>(workers_.size()) < T - 1) {
      try {
        workers_.emplace_back(&HostPool::worker, this, static_cast<int>(workers_.size()) + 1);
      } catch (const std::system_error&) {
        break;
      }
    }
    const int on_workers = std::min(T - 1, static_cast<int>(workers_.size()));
    {
      std::lock_guard<std::mutex> lk(mu_);
      task_ = &task;
      want_ = on_workers;
      pending_ = on_workers;
      ++gen_;
    }
    wake_.notify_all();
    task(0);
    for (int t = on_workers + 1; t < T; ++t) task(t);
    std::unique_lock<std::mutex> lk(mu_);
    idle_.wait(lk, [&] { return pending_ == 0; });
    task_ = nullptr;
    return true;
  }

 private:
  HostPool() = default;
  static std::atomic<HostPool*>& slot() {
    static std::atomic<HostPool*> p{nullptr};
    return p;
  }
  static bool& in_worker() {
    static thread_local bool w = false;
    return w;
  }
  void worker(int id) {  // id in 1 .. workers_.size()
    in_worker() = true;
    std::uint64_t seen = 0;
    std::unique_lock<std::mutex> lk(mu_);
    for (;;) {
      wake_.wait(lk, [&] { return gen_ != seen; });
      seen = gen_;
      if (id > want_) continue;  // not part of this section
      const std::function<void(int)>* task = task_;
      lk.unlock();
      (*task)(id);
      lk.lock();
      if (--pending_ == 0) idle_.notify_one();
    }
  }
  std::mutex use_;  // held by the section that owns the workers
  std::mutex mu_;
  std::condition_variable wake_, idle_;
  std::uint64_t gen_ = 0;
  const std::function<void(int)>* task_ = nullptr;
  int want_ = 0, pending_ = 0;
  std::vector<std::thread> workers_;
};

// Runs f(begin, end) over [0, n) on host_thread_limit() threads (inline below `min_parallel`).
// The ranges are the same whichever threads run them.
template <class F>
void parallel_ranges(long long n, F&& f, long long min_parallel = 65536) {
  const long long T = n < min_parallel ? 1 : std::min<long long>(n, host_thread_limit());
  if (T <= 1) {
    f(0LL, n);
    return;
  }
  const std::function<void(int)> task = [&](int t) { f(n * t / T, n * (t + 1) / T); };
  if (HostPool::instance().run(static_cast<int>(T), task)) return;
  std::vector<std::thread> th;  // the pool is in use: threads of this section's own
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
