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
#include <exception>
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
// started while the pool is busy (another thread's), from inside a pool worker, or from inside
// a section of the same calling thread returns false from run() and its caller uses threads of
// its own. The pool is never destroyed (its
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
  // nothing, when the pool is busy, the caller is one of its workers, or the caller is already
  // inside a section of its own (a nested section). An exception thrown by a task is caught
  // where it is thrown; run() still waits for every task, then rethrows the first one on the
  // calling thread.
  bool run(int T, const std::function<void(int)>& task) {
    if (in_worker() || in_section() || !use_.try_lock()) return false;
    std::lock_guard<std::mutex> own(use_, std::adopt_lock);
    struct SectionFlag {
      SectionFlag() { in_section() = true; }
      ~SectionFlag() { in_section() = false; }
    } flag;
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
      error_ = nullptr;
      ++gen_;
    }
    wake_.notify_all();
    std::exception_ptr mine;
    try {
      task(0);
    } catch (...) {
      mine = std::current_exception();
    }
    for (int t = on_workers + 1; t < T; ++t) {
      try {
        task(t);
      } catch (...) {
        if (!mine) mine = std::current_exception();
      }
    }
    std::exception_ptr theirs;
    {
      std::unique_lock<std::mutex> lk(mu_);
      idle_.wait(lk, [&] { return pending_ == 0; });
      task_ = nullptr;
      theirs = error_;
      error_ = nullptr;
    }
    if (mine) std::rethrow_exception(mine);
    if (theirs) std::rethrow_exception(theirs);
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
  static bool& in_section() {  // the calling thread owns the pool for a section
    static thread_local bool s = false;
    return s;
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
      std::exception_ptr err;
      try {
        (*task)(id);
      } catch (...) {  // an exception must not leave the worker: it would end the process
        err = std::current_exception();
      }
      lk.lock();
      if (err && !error_) error_ = err;
      if (--pending_ == 0) idle_.notify_one();
    }
  }
  std::mutex use_;  // held by the section that owns the workers
  std::mutex mu_;
  std::condition_variable wake_, idle_;
  std::uint64_t gen_ = 0;
  const std::function<void(int)>* task_ = nullptr;
  std::exception_ptr error_;  // the first exception a worker caught in the current section
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
  // the pool is in use: threads of this section's own. Exceptions are caught where they are
  // thrown; every thread is joined before the first one is rethrown on the calling thread.
  std::mutex err_mu;
  std::exception_ptr err;
  auto guarded = [&](long long t) {
    try {
      f(n * t / T, n * (t + 1) / T);
    } catch (...) {
      std::lock_guard<std::mutex> lk(err_mu);
      if (!err) err = std::current_exception();
    }
  };
  std::vector<std::thread> th;
  th.reserve(static_cast<std::size_t>(T - 1));
  long long started = 1;
  for (; started < T; ++started) {
    try {
      th.emplace_back(guarded, started);
    } catch (const std::system_error&) {
      break;  // no more threads: the calling thread runs the remaining ranges
    }
  }
  guarded(0);
  for (long long t = started; t < T; ++t) guarded(t);
  for (auto& x : th) x.join();
  if (err) std::rethrow_exception(err);
}

// Runs task(t) for t in [0, T) on the pool (task 0 on the calling thread), or, when the pool is
// in use, on threads of this call's own. Tasks may run one after another (T = 1, no thread could
// be started): a task must never wait for work that only another task would do. The first
// exception is rethrown on the calling thread once every task has returned.
template <class F>
void parallel_tasks(int T, F&& task) {
  if (T <= 1) {
    task(0);
    return;
  }
  const std::function<void(int)> fn = [&](int t) { task(t); };
  if (HostPool::instance().run(T, fn)) return;
  std::mutex err_mu;
  std::exception_ptr err;
  auto guarded = [&](int t) {
    try {
      task(t);
    } catch (...) {
      std::lock_guard<std::mutex> lk(err_mu);
      if (!err) err = std::current_exception();
    }
  };
  std::vector<std::thread> th;
  th.reserve(static_cast<std::size_t>(T - 1));
  int started = 1;
  for (; started < T; ++started) {
    try {
      th.emplace_back(guarded, started);
    } catch (const std::system_error&) {
      break;
    }
  }
  guarded(0);
  for (int t = started; t < T; ++t) guarded(t);
  for (auto& x : th) x.join();
  if (err) std::rethrow_exception(err);
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
