// bench_gather_rate — bench.py's probe (not part of the library): the device's rate of random 8-byte gathers from a vector that stays in
// L2, the second ceiling of the iteration kernels besides HBM bandwidth (each nonzero of Ã and
// Ãᵀ gathers one element of x̄ or y: 2·nnz random gathers per iteration).
//
//   bench_gather_rate [n] [count]     (defaults: n = 1,500,000 doubles, count = 6,000,000 gathers)
//
// Prints one JSON line: {"gathers_per_s": G, "n": n, "count": count, "us": T}. The indices are
// drawn on the host in [0, n), so every access is in bounds; the gathered vector is brought into
// L2 by an untimed pass before each timed one, and the best of five timed passes is reported.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <random>
#include <vector>

namespace {

#define GR_CHECK(x)                                                              \
  do {                                                                           \
    const cudaError_t e_ = (x);                                                  \
    if (e_ != cudaSuccess) {                                                     \
      std::fprintf(stderr, "gather_rate: %s (line %d)\n", cudaGetErrorString(e_), __LINE__); \
      return 1;                                                                  \
    }                                                                            \
  } while (0)

// Each thread gathers 4 independent elements per round (the batch the iteration kernels use).
__global__ void k_gather(long long count, const int* __restrict__ idx, const double* __restrict__ x, double* out) {
  const long long t = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
  const long long stride = static_cast<long long>(gridDim.x) * blockDim.x;
  double s = 0.0;
  for (long long k = t; k < count; k += 4 * stride) {
    double p[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const long long kk = k + q * stride;
      p[q] = kk < count ? x[__ldg(idx + kk)] : 0.0;
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) s += p[q];
  }
  out[t] = s;
}

}  // namespace

int main(int argc, char** argv) {
  const long long n = argc > 1 ? std::atoll(argv[1]) : 1500000LL;
  const long long count = argc > 2 ? std::atoll(argv[2]) : 6000000LL;
  if (n <= 0 || count <= 0 || n > (1LL << 31) - 1) {
    std::fprintf(stderr, "usage: gather_rate [n] [count]\n");
    return 2;
  }
  std::vector<int> h(static_cast<std::size_t>(count));
  std::mt19937_64 rng(1);
  for (auto& i : h) i = static_cast<int>(rng() % static_cast<unsigned long long>(n));
  int nsm = 0;
  GR_CHECK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, 0));
  const int grid = nsm * 8, block = 256;
  int* idx = nullptr;
  double *x = nullptr, *out = nullptr;
  GR_CHECK(cudaMalloc(&idx, static_cast<std::size_t>(count) * sizeof(int)));
  GR_CHECK(cudaMalloc(&x, static_cast<std::size_t>(n) * sizeof(double)));
  GR_CHECK(cudaMalloc(&out, static_cast<std::size_t>(grid) * block * sizeof(double)));
  GR_CHECK(cudaMemcpy(idx, h.data(), h.size() * sizeof(int), cudaMemcpyHostToDevice));
  GR_CHECK(cudaMemset(x, 0, static_cast<std::size_t>(n) * sizeof(double)));
  cudaEvent_t a, b;
  GR_CHECK(cudaEventCreate(&a));
  GR_CHECK(cudaEventCreate(&b));
  float best = 1e30f;
  for (int r = 0; r < 6; ++r) {
    k_gather<<<grid, block>>>(count, idx, x, out);  // x into L2
    GR_CHECK(cudaEventRecord(a));
    k_gather<<<grid, block>>>(count, idx, x, out);
    GR_CHECK(cudaEventRecord(b));
    GR_CHECK(cudaEventSynchronize(b));
    float ms = 0;
    GR_CHECK(cudaEventElapsedTime(&ms, a, b));
    if (r > 0 && ms < best) best = ms;
  }
  GR_CHECK(cudaGetLastError());
  std::printf("{\"gathers_per_s\": %.6g, \"n\": %lld, \"count\": %lld, \"us\": %.3f}\n",
              static_cast<double>(count) / (best * 1e-3), n, count, best * 1e3);
  cudaFree(idx);
  cudaFree(x);
  cudaFree(out);
  return 0;
}
