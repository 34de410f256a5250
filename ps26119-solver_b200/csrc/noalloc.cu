// noalloc.cu — ps26119_dot_noalloc: the fp64 dot product of two device vectors for callers
// that must not allocate device memory.
//
// Who needs it: callers that cannot call cudaMalloc at the point where they need the dot
// product — a caller whose device memory is all handed out by its own pool and budgeted to the
// byte (an allocation behind its back can fail or push it out of memory), or a loop with a
// latency bound that may not wait on the allocator's locks and the driver calls behind them.
// The backend's Backend::dot (ps26119_backend_dot) materialises its per-element terms and
// partial sums in buffers it allocates; this entry point does the same arithmetic with that
// scratch in one file-scope device array instead, so a call allocates nothing.
//
// The scratch: g_noalloc_scratch, kNoAllocMaxN + 256 doubles (16 MiB + 2 KiB) per device,
// reserved when the CUDA runtime loads this library's device code and held until the process
// exits. Its address is taken once per device (cudaGetSymbolAddress, with that device current)
// on the first call made while the device is current, so that first call should come before any
// stream capture. The address is kept for the life of the process: do not call this entry point
// again on a device after cudaDeviceReset (the reset unloads the array the address points to).
// Every call on a device shares the one array: calls whose kernels overlap on the GPU (two
// streams, or two host threads with different streams) race on it and may return wrong sums;
// serialise them on one stream. Nothing in the scratch needs to start at zero: every term and
// partial is written before it is read.
//
// Results: exact = 1 sums in la::parallel_sum's order (64 contiguous chunks, each summed in
// order, then the chunk sums in order) and equals ps26119_backend_dot of an exact-mode backend
// bit for bit; exact = 0 uses the backend's fixed 96-block tree and equals its fast-mode dot.
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>
#include <string>

#include "../../include/ps26119.h"
#include "../../include/ps26119_backend.h"
#include "reduce.cuh"

namespace b200 {
void set_backend_error(const std::string& text);  // c_api.cpp: the thread's last-error text
}

namespace {

using namespace b200;

constexpr long long kNoAllocMaxN = 1LL << 21;  // 2,097,152 elements: 16 MiB of terms
constexpr int kMaxDevices = 64;

// [0, kNoAllocMaxN) terms, then 64 chunk partials, then kTreeBlocks tree partials.
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocMaxN + 256];

std::mutex g_setup_mu;
double* g_scratch_ptr[kMaxDevices] = {};

__global__ void k_na_terms(long long n, const double* __restrict__ a, const double* __restrict__ b,
                           double* __restrict__ t) {
  B200_FOR(i, n) t[i] = a[i] * b[i];
}

// exact: warp c sums chunk c of [0, n) in order (the chunk boundaries of la::parallel_sum)
__global__ void k_na_chunks(long long n, long long chunks, const double* __restrict__ t, double* __restrict__ part) {
  const long long c = (blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (c >= chunks) return;
  const long long lo = n * c / chunks, hi = n * (c + 1) / chunks;
  double s = 0.0;
  long long base = lo;
  double v = (base + lane < hi) ? t[base + lane] : 0.0;
  while (base < hi) {
    const long long nb = base + 32;
    const double vn = (nb + lane < hi) ? t[nb + lane] : 0.0;
    const long long rem = hi - base;
    const int cnt = rem < 32 ? static_cast<int>(rem) : 32;
    for (int j = 0; j < cnt; ++j) s += __shfl_sync(kFull, v, j);
    v = vn;
    base = nb;
  }
  if (lane == 0) part[c] = s;
}
__global__ void k_na_chunks_final(long long chunks, const double* __restrict__ part, double* __restrict__ out) {
  if (threadIdx.x != 0) return;
  double s = 0.0;
  for (long long c = 0; c < chunks; ++c) s += part[c];
  *out = s;
}

// fast: the backend's two-level tree (kTreeBlocks block sums, then one block over them)
__global__ void k_na_tree1(long long n, const double* __restrict__ t, double* __restrict__ part) {
  __shared__ double sh[32];
  const int b = blockIdx.x;
  const long long a = n * b / kTreeBlocks, e = n * (b + 1) / kTreeBlocks;
  double acc = 0.0;
  for (long long i = a + threadIdx.x; i < e; i += blockDim.x) acc += t[i];
  acc = block_sum_fixed(acc, sh);
  if (threadIdx.x == 0) part[b] = acc;
}
__global__ void k_na_tree2(const double* __restrict__ part, double* __restrict__ out) {
  __shared__ double sh[32];
  double acc = 0.0;
  for (int i = threadIdx.x; i < kTreeBlocks; i += blockDim.x) acc += part[i];
  acc = block_sum_fixed(acc, sh);
  if (threadIdx.x == 0) *out = 0.0 + acc;
}

// The scratch address of the current device, looked up once per device.
double* scratch_of_current_device(std::string& err) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    (void)cudaGetLastError();
    err = std::string("CUDA backend unavailable: ") + cudaGetErrorString(e);
    return nullptr;
  }
  if (dev < 0 || dev >= kMaxDevices) {
    err = "device ordinal out of range for the no-alloc scratch table";
    return nullptr;
  }
  std::lock_guard<std::mutex> lock(g_setup_mu);
  if (!g_scratch_ptr[dev]) {
    double* p = nullptr;
    e = cudaGetSymbolAddress(reinterpret_cast<void**>(&p), g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      (void)cudaGetLastError();
      err = std::string("cudaGetSymbolAddress of the no-alloc scratch failed: ") + cudaGetErrorString(e);
      return nullptr;
    }
    g_scratch_ptr[dev] = p;
  }
  return g_scratch_ptr[dev];
}

}  // namespace

extern "C" int ps26119_dot_noalloc(long long n, const double* a, const double* b, int exact, double* out,
                                   void* stream) {
  if (n < 0 || !out || (n > 0 && (!a || !b))) {
    b200::set_backend_error("invalid arguments: n must be >= 0 and a, b, out non-NULL");
    return PS26119_INVALID_ARGUMENT;
  }
  if (n > kNoAllocMaxN) {
    char buf[160];
    std::snprintf(buf, sizeof buf, "n = %lld exceeds the no-alloc scratch maximum of %lld elements", n,
                  kNoAllocMaxN);
    b200::set_backend_error(buf);
    return PS26119_INVALID_ARGUMENT;
  }
  std::string err;
  double* s = scratch_of_current_device(err);
  if (!s) {
    b200::set_backend_error(err);
    return PS26119_NOT_SOLVED;
  }
  double* terms = s;
  double* chunk_part = s + kNoAllocMaxN;
  double* tree_part = s + kNoAllocMaxN + 64;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (n > 0) k_na_terms<<<grid_for(n), kBlock, 0, st>>>(n, a, b, terms);
  if (exact) {
    const long long chunks = n < kChunks ? (n < 1 ? 1 : n) : kChunks;
    k_na_chunks<<<static_cast<unsigned>((chunks + 3) / 4), 128, 0, st>>>(n, chunks, terms, chunk_part);
    k_na_chunks_final<<<1, 32, 0, st>>>(chunks, chunk_part, out);
  } else {
    k_na_tree1<<<kTreeBlocks, kBlock, 0, st>>>(n, terms, tree_part);
    k_na_tree2<<<1, kBlock, 0, st>>>(tree_part, out);
  }
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    b200::set_backend_error(std::string("CUDA error: ") + cudaGetErrorString(e));
    return PS26119_NUMERICAL_ERROR;
  }
  return 0;
}
