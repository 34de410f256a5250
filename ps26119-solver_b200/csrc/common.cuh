// common.cuh — device buffers, error handling and warp helpers shared by every kernel file.
//
// Numerics contract of every kernel in this library: compiled with -fmad=false, so a*b+c is
// evaluated with two roundings exactly as the reference's x86-64 CPU build evaluates it;
// fp64 division and sqrt are the IEEE-rounded ones (-prec-div/-prec-sqrt are nvcc defaults).
// Element-wise kernels and CSR row products therefore reproduce the reference CPU backend
// (src/pdhg/cpu_backend.cpp) bit for bit. Only reductions may reorder sums (fast mode).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <new>
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

// Device allocation owned by the host object. cudaErrorMemoryAllocation becomes
// std::bad_alloc, reported as NOT_SOLVED "out of memory" (reference cuda_backend.cu:74-80).
template <class T>
class DevBuf {
 public:
  DevBuf() = default;
  explicit DevBuf(std::size_t n) { alloc(n); }
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  DevBuf(DevBuf&& o) noexcept : p_(o.p_), n_(o.n_) { o.p_ = nullptr, o.n_ = 0; }
  DevBuf& operator=(DevBuf&& o) noexcept {
    if (this != &o) {
      release();
      p_ = o.p_, n_ = o.n_;
      o.p_ = nullptr, o.n_ = 0;
    }
    return *this;
  }
  ~DevBuf() { release(); }

  // Allocates n elements plus 64 bytes of tail padding: 16-byte-aligned bulk copies of a
  // range [a, b) are widened to 16-byte boundaries and may read up to 15 bytes past the last
  // element; the padding keeps that inside the allocation.
  void alloc(std::size_t n) {
    release();
    const std::size_t bytes = n * sizeof(T) + 64;
    void* p = nullptr;
    B200_CHECK(cudaMalloc(&p, bytes));
    p_ = static_cast<T*>(p);
    n_ = n;
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
    if (p_) cudaFree(p_);  // never throws from a destructor
    p_ = nullptr;
    n_ = 0;
  }
  T* p_ = nullptr;
  std::size_t n_ = 0;
};

// Page-locked host memory for the per-check status transfers.
template <class T>
class PinnedBuf {
 public:
  PinnedBuf() = default;
  PinnedBuf(const PinnedBuf&) = delete;
  PinnedBuf& operator=(const PinnedBuf&) = delete;
  ~PinnedBuf() {
    if (p_) cudaFreeHost(p_);
  }
  void alloc(std::size_t n) {
    if (p_) cudaFreeHost(p_);
    p_ = nullptr;
    B200_CHECK(cudaMallocHost(reinterpret_cast<void**>(&p_), (n ? n : 1) * sizeof(T)));
    n_ = n;
  }
  T* get() { return p_; }
  T& operator[](std::size_t i) { return p_[i]; }
  std::size_t size() const { return n_; }

 private:
  T* p_ = nullptr;
  std::size_t n_ = 0;
};

constexpr int kBlock = 256;
constexpr unsigned kFull = 0xffffffffu;

inline int grid_for(std::int64_t n, int block = kBlock) {
  const std::int64_t g = (n + block - 1) / block;
  return static_cast<int>(g < 1 ? 1 : (g > (1LL << 30) ? (1LL << 30) : g));
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
