// parallel_copy_check.cpp — test driver for csrc/parallel.hpp: parallel_copy against memcpy on
// random job lists (empty jobs, small ones, and ones above the 4 MiB threading threshold), with
// guard bytes on both sides of every destination; size_for_copy keeps or replaces a buffer as
// documented. Prints "ok" and exits 0, or names the first mismatch and exits 1.
#include <cstdio>
#include <cstring>
#include <random>
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
  std::printf("ok\n");
  return 0;
}
