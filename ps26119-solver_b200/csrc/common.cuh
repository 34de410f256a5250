// common.cuh — device buffers, error handling and warp helpers shared by every kernel file.
//
// Numerics contract of every kernel in this library: compiled with -fmad=false, so a*b+c is
// evaluated with two roundings exactly as the reference's x86-64 CPU build evaluates it;
// fp64 division and sqrt are the IEEE-rounded ones (-prec-div/-prec-sqrt are nvcc defaults).
// Element-wise kernels and CSR row products therefore reproduce the reference CPU backend
// (src/pdhg/cpu_backend.cpp) bit for bit. Only reductions may reorder sums (fast mode).
#pragma once

#include <atomic>

#include <cuda_runtime.h>

#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <mutex>
#include <new>
#include <map>
#include <set>
#include <shared_mutex>
#include <vector>
#include <stdexcept>
#include <string>
#include <utility>

namespace b200 {

// Thrown for any CUDA runtime failure; the C ABI maps it to PS26119_NUMERICAL_ERROR
// (reference behaviour: src/core/solve.cpp:590-594).
struct CudaError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

#define B200_CHECK(expr)                                                                         \
  do {                                                                                           \
    cudaError_t e_ = (expr);                                                                     \
    if (e_ != cudaSuccess) {                                                                     \
      if (e_ == cudaErrorMemoryAllocation) {                                                     \
        (void)cudaGetLastError();                                                                \
        throw std::bad_alloc();                                                                  \
      }                                                                                          \
      throw ::b200::CudaError(std::string("CUDA error: ") + cudaGetErrorString(e_) + " in " #expr); \
    }                                                                                            \
  } while (0)

#define B200_LAUNCH_CHECK() B200_CHECK(cudaGetLastError())

// Stream capture and device-wide synchronisation exclude each other. CUDA rejects a device
// synchronisation (cudaDeviceSynchronize, and the implicit one in cudaFree / cudaFreeHost) while
// any stream of the device is being captured, and the rejected call invalidates that capture. So
// with solves running on several host threads (the request loop), every capture in this library
// holds this lock shared (CaptureScope) and every device-wide synchronising call holds it
// exclusively (with_device_sync). A thread inside its own capture makes no such call:
// with_device_sync then does nothing and returns false.
inline std::shared_mutex& capture_mutex() {
  static std::shared_mutex* m = new std::shared_mutex();  // never destroyed
  return *m;
}
inline thread_local bool t_capturing = false;
class CaptureScope {
 public:
  CaptureScope() : lk_(capture_mutex()) { t_capturing = true; }
  ~CaptureScope() { t_capturing = false; }
  CaptureScope(const CaptureScope&) = delete;
  CaptureScope& operator=(const CaptureScope&) = delete;

 private:
  std::shared_lock<std::shared_mutex> lk_;
};
template <class F>
inline bool with_device_sync(F&& f) {
  if (t_capturing) return false;
  std::unique_lock<std::shared_mutex> lk(capture_mutex());
  f();
  return true;
}

// A process-wide cache of device blocks. Solves allocate the same large buffers again and
// again; cudaMalloc / cudaFree of gigabytes cost a device-wide synchronisation and, measured on
// B200, from a few ms up to over a second per solve. Released blocks are kept (per device, by
// size class: powers of two up to 1 MiB, multiples of 2 MiB above) and handed out again; at
// most PS26119_DEVICE_CACHE_MB (default 8192) MiB stay cached, the rest is freed. A block
// released while kernels of its releasing thread may still use it (scoped temporaries of a
// setup step) is handed out again only after a device synchronisation that began after the
// release: solves on other threads and streams never see it in use. On an allocation failure
// the device's cached blocks are freed and the allocation is retried.
class DeviceBlockCache {
 public:
  static DeviceBlockCache& instance() {
    static DeviceBlockCache* c = new DeviceBlockCache();  // never destroyed: no CUDA calls at exit
    return *c;
  }
  static std::size_t size_class(std::size_t bytes) {
    if (bytes <= (1u << 20)) {
      std::size_t c = 512;
      while (c < bytes) c <<= 1;
      return c;
    }
    const std::size_t g = 2u << 20;
    return (bytes + g - 1) / g * g;
  }
  // A released block may still be read or written by kernels its releasing thread enqueued
  // (on any stream). Every release gets a generation number; a block is handed out again only
  // once a device synchronisation that started after its release has completed (`synced_`).
  void* acquire(std::size_t bytes) {  // bytes: a size class
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) dev = 0;
    {
      std::unique_lock<std::mutex> lock(mu_);
      const std::uint64_t idle = synced_[dev];
      long long ready = -1, pending = -1;
      for (std::size_t k = 0; k < free_.size(); ++k)
        if (free_[k].device == dev && free_[k].bytes == bytes) {
          if (free_[k].gen <= idle) {
            ready = static_cast<long long>(k);
            break;
          }
          if (pending < 0) pending = static_cast<long long>(k);
        }
      if (ready >= 0) return take(static_cast<std::size_t>(ready));
      if (pending >= 0 && !t_capturing) {  // reuse after one device synchronisation
        void* p = take(static_cast<std::size_t>(pending));
        const std::uint64_t upto = gen_;
        lock.unlock();
        with_device_sync([] { (void)cudaDeviceSynchronize(); });
        lock.lock();
        synced_[dev] = std::max(synced_[dev], upto);
        return p;
      }
    }
    void* p = nullptr;
    cudaError_t e = cudaMalloc(&p, bytes);
    if (e == cudaErrorMemoryAllocation) {
      (void)cudaGetLastError();
      trim(dev);
      e = cudaMalloc(&p, bytes);
    }
    if (e == cudaErrorMemoryAllocation) {
      (void)cudaGetLastError();
      throw std::bad_alloc();
    }
    if (e != cudaSuccess) throw CudaError(std::string("CUDA error: ") + cudaGetErrorString(e) + " in cudaMalloc");
    return p;
  }
  void release(void* p, std::size_t bytes, int dev) {
    {
      std::lock_guard<std::mutex> lock(mu_);
      if (cached_ + bytes <= limit_ || t_capturing) {  // inside a capture: keep it, freeing would sync
        free_.push_back({dev, bytes, p, ++gen_});
        cached_ += bytes;
        return;
      }
    }
    with_device_sync([p] { cudaFree(p); });  // never throws from a destructor
  }
  void trim(int dev) {  // frees this device's cached blocks
    std::vector<Block> drop;
    {
      std::lock_guard<std::mutex> lock(mu_);
      for (std::size_t k = 0; k < free_.size();)
        if (free_[k].device == dev) {
          drop.push_back(free_[k]);
          cached_ -= free_[k].bytes;
          free_[k] = free_.back();
          free_.pop_back();
        } else {
          ++k;
        }
    }
    if (drop.empty()) return;
    const bool done = with_device_sync([&drop] {
      (void)cudaDeviceSynchronize();
      for (const Block& b : drop) cudaFree(b.p);
    });
    if (!done) {  // inside a capture of this thread: keep the blocks cached
      std::lock_guard<std::mutex> lock(mu_);
      for (const Block& b : drop) free_.push_back(b), cached_ += b.bytes;
    }
  }

 private:
  DeviceBlockCache() {
    const char* env = std::getenv("PS26119_DEVICE_CACHE_MB");
    const long long mb = env ? std::atoll(env) : 8192;
    limit_ = mb > 0 ? static_cast<std::size_t>(mb) << 20 : 0;
  }
  struct Block {
    int device;
    std::size_t bytes;
    void* p;
    std::uint64_t gen;  // release generation
  };
  void* take(std::size_t k) {  // with mu_ held
    void* p = free_[k].p;
    cached_ -= free_[k].bytes;
    free_[k] = free_.back();
    free_.pop_back();
    return p;
  }
  std::mutex mu_;
  std::vector<Block> free_;
  std::map<int, std::uint64_t> synced_;  // per device: blocks released at or before this generation are idle
  std::uint64_t gen_ = 0;
  std::size_t cached_ = 0, limit_ = 0;
};

// Device allocation owned by the host object (through DeviceBlockCache). cudaErrorMemoryAllocation
// becomes std::bad_alloc, reported as NOT_SOLVED "out of memory" (reference cuda_backend.cu:74-80).
template <class T>
class DevBuf {
 public:
  DevBuf() = default;
  explicit DevBuf(std::size_t n) { alloc(n); }
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  DevBuf(DevBuf&& o) noexcept : p_(o.p_), n_(o.n_), bytes_(o.bytes_), dev_(o.dev_) {
    o.p_ = nullptr, o.n_ = 0, o.bytes_ = 0;
  }
  DevBuf& operator=(DevBuf&& o) noexcept {
    if (this != &o) {
      release();
      p_ = o.p_, n_ = o.n_, bytes_ = o.bytes_, dev_ = o.dev_;
      o.p_ = nullptr, o.n_ = 0, o.bytes_ = 0;
    }
    return *this;
  }
  ~DevBuf() { release(); }

  // Allocates n elements plus 64 bytes of tail padding: 16-byte-aligned bulk copies of a
  // range [a, b) are widened to 16-byte boundaries and may read up to 15 bytes past the last
  // element; the padding keeps that inside the allocation.
  void alloc(std::size_t n) {
    release();
    const std::size_t bytes = DeviceBlockCache::size_class(n * sizeof(T) + 64);
    if (cudaGetDevice(&dev_) != cudaSuccess) dev_ = 0;
    p_ = static_cast<T*>(DeviceBlockCache::instance().acquire(bytes));
    n_ = n;
    bytes_ = bytes;
  }
  void ensure(std::size_t n) {
    if (n_ < n || !p_) alloc(n);
  }
  void upload(const T* h, std::size_t n, cudaStream_t s) {
    ensure(n);
    if (n) B200_CHECK(cudaMemcpyAsync(p_, h, n * sizeof(T), cudaMemcpyHostToDevice, s));
  }
  void download(T* h, std::size_t n, cudaStream_t s) const {
    if (n) B200_CHECK(cudaMemcpyAsync(h, p_, n * sizeof(T), cudaMemcpyDeviceToHost, s));
  }
  T* get() { return p_; }
  const T* get() const { return p_; }
  std::size_t size() const { return n_; }

 private:
  void release() {
    if (p_) DeviceBlockCache::instance().release(p_, bytes_, dev_);  // never throws
    p_ = nullptr;
    n_ = 0;
    bytes_ = 0;
  }
  T* p_ = nullptr;
  std::size_t n_ = 0, bytes_ = 0;
  int dev_ = 0;
};

// Page-locked host blocks, cached like the device blocks: cudaFreeHost synchronises the device
// and was measured to take from under a millisecond to over ten per call. At most 256 MiB stay
// cached; blocks are reused by exact size class.
class PinnedBlockCache {
 public:
  static PinnedBlockCache& instance() {
    static PinnedBlockCache* c = new PinnedBlockCache();  // never destroyed: no CUDA calls at exit
    return *c;
  }
  void* acquire(std::size_t bytes) {
    {
      std::lock_guard<std::mutex> lock(mu_);
      for (std::size_t k = 0; k < free_.size(); ++k)
        if (free_[k].first == bytes) {
          void* p = free_[k].second;
          free_[k] = free_.back();
          free_.pop_back();
          cached_ -= bytes;
          return p;
        }
    }
    void* p = nullptr;
    B200_CHECK(cudaMallocHost(&p, bytes));
    return p;
  }
  void release(void* p, std::size_t bytes) {
    {
      std::lock_guard<std::mutex> lock(mu_);
      if (cached_ + bytes <= (256u << 20) || t_capturing) {
        free_.push_back({bytes, p});
        cached_ += bytes;
        return;
      }
    }
    with_device_sync([p] { cudaFreeHost(p); });
  }

 private:
  std::mutex mu_;
  std::vector<std::pair<std::size_t, void*>> free_;
  std::size_t cached_ = 0;
};

// Page-locked host memory for the per-check status transfers. The host code syncs the stream
// that used a block before the block goes back to the cache.
template <class T>
class PinnedBuf {
 public:
  PinnedBuf() = default;
  PinnedBuf(const PinnedBuf&) = delete;
  PinnedBuf& operator=(const PinnedBuf&) = delete;
  ~PinnedBuf() {
    if (p_) PinnedBlockCache::instance().release(p_, bytes_);
  }
  void alloc(std::size_t n) {
    if (p_) PinnedBlockCache::instance().release(p_, bytes_);
    p_ = nullptr;
    bytes_ = DeviceBlockCache::size_class((n ? n : 1) * sizeof(T));
    p_ = static_cast<T*>(PinnedBlockCache::instance().acquire(bytes_));
    n_ = n;
  }
  T* get() { return p_; }
  T& operator[](std::size_t i) { return p_[i]; }
  std::size_t size() const { return n_; }

 private:
  T* p_ = nullptr;
  std::size_t n_ = 0, bytes_ = 0;
};

constexpr int kBlock = 256;
constexpr unsigned kFull = 0xffffffffu;

inline int grid_for(std::int64_t n, int block = kBlock) {
  const std::int64_t g = (n + block - 1) / block;
  return static_cast<int>(g < 1 ? 1 : (g > (1LL << 30) ? (1LL << 30) : g));
}

// Streaming multiprocessors of the current device (cached per device).
inline int sm_count() {
  static std::atomic<int> cached[64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
  int v = cached[dev].load(std::memory_order_relaxed);
  if (v == 0) {
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0) v = 148;
    cached[dev].store(v, std::memory_order_relaxed);
  }
  return v;
}

// Grid-stride helper over [0, n).
#define B200_FOR(i, n) \
  for (std::int64_t i = blockIdx.x * static_cast<std::int64_t>(blockDim.x) + threadIdx.x; i < (n); \
       i += static_cast<std::int64_t>(gridDim.x) * blockDim.x)

// clamp exactly as the reference's cpu_backend.cpp:17-20 (NaN passes through).
template <class T>
__host__ __device__ __forceinline__ T ref_clamp(T v, T lo, T hi) {
  return v < lo ? lo : (v > hi ? hi : v);
}
// std::max / std::min semantics (first argument wins on ties and on NaN in the second).
__host__ __device__ __forceinline__ double std_max(double a, double b) { return (a < b) ? b : a; }
__host__ __device__ __forceinline__ double std_min(double a, double b) { return (b < a) ? b : a; }

// Monotone key of a NON-NEGATIVE double for integer atomics (max of non-negative doubles).
__device__ __forceinline__ unsigned long long nonneg_key(double v) {
  return static_cast<unsigned long long>(__double_as_longlong(v));
}
__device__ __forceinline__ void atomic_max_nonneg(unsigned long long* slot, double v) {
  // std::max(acc, v) ignores a NaN v; -0.0 compares equal to 0.0 and never wins.
  if (v > 0.0) atomicMax(slot, nonneg_key(v));
}
__device__ __forceinline__ void atomic_min_pos(unsigned long long* slot, double v) {
  if (v > 0.0) atomicMin(slot, nonneg_key(v));
}

// Maximum of a non-negative candidate over the whole warp (all 32 lanes must call it), then one
// atomic per warp: order-independent like atomic_max_nonneg, without the contention of one
// atomic per element on a single address.
__device__ __forceinline__ void warp_max_atomic(unsigned long long* slot, double v) {
  unsigned long long key = (v > 0.0) ? nonneg_key(v) : 0ULL;  // NaN and -0.0 never win
  for (int off = 16; off > 0; off >>= 1) {
    const unsigned long long o = __shfl_xor_sync(kFull, key, off);
    key = o > key ? o : key;
  }
  if ((threadIdx.x & 31) == 0 && key != 0ULL) atomicMax(slot, key);
}
__device__ __forceinline__ void warp_min_atomic_pos(unsigned long long* slot, double v) {
  unsigned long long key = (v > 0.0) ? nonneg_key(v) : ~0ULL;
  for (int off = 16; off > 0; off >>= 1) {
    const unsigned long long o = __shfl_xor_sync(kFull, key, off);
    key = o < key ? o : key;
  }
  if ((threadIdx.x & 31) == 0 && key != ~0ULL) atomicMin(slot, key);
}

}  // namespace b200
