// reduce.cuh — deterministic fp64 sums over term arrays, in two selectable orders.
//
// Every reduction of the engine first materialises its per-element terms (double), then a
// SumPlan reduces them. Two orders:
//   exact: the reference CPU's own order. kSeq = one sequential chain (the reference's plain
//          host loops, e.g. kkt_general, cpu_backend.cpp:226-284); kChunk64 = 64 contiguous
//          chunks summed sequentially, then the 64 partials in order (la::parallel_sum,
//          parallel.h:169-188, used by Backend::dot / diff_norm2). A chain is walked by one
//          warp: the 32 lanes load 32 consecutive terms, and the running sum takes them one
//          by one through shuffles, so the order is exactly i = lo, lo+1, ….
//   fast:  a fixed two-level tree (kTreeBlocks blocks per sum, block tree, then one block
//          combines the partials) — deterministic run to run, but a different rounding.
// Maxima never go through a SumPlan: they are taken with integer atomics on non-negative
// doubles, which is order-independent and exact.
#pragma once

#include <vector>

#include "common.cuh"

namespace b200 {

enum class SumOrder { kSeq, kChunk64 };

struct ChainSeg {
  const double* t;
  long long lo, hi;
  double init;
  double* out;
};
struct TreeSeg {
  const double* t;
  long long lo, hi;
  double init;
  double* out;
};

constexpr int kTreeBlocks = 96;
constexpr int kChunks = 64;  // la::kReduceChunks

__device__ __forceinline__ double block_sum_fixed(double v, double* sh) {
  for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(kFull, v, off);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) sh[wid] = v;
  __syncthreads();
  if (wid == 0) {
    v = lane < static_cast<int>(blockDim.x >> 5) ? sh[lane] : 0.0;
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(kFull, v, off);
  }
  return v;  // valid in thread 0
}

// One warp per segment; the running sum visits t[lo], t[lo+1], … in order. `gate`, when
// non-null, is read first and a non-zero value skips the work (graph-replayed launches).
static __global__ void k_chain(const ChainSeg* segs, int nseg, const int* skip) {
  if (skip && *skip) return;
  const int warp = static_cast<int>((blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (warp >= nseg) return;
  const ChainSeg g = segs[warp];
  double s = g.init;
  long long base = g.lo;
  double v = (base + lane < g.hi) ? g.t[base + lane] : 0.0;
  while (base < g.hi) {
    const long long nb = base + 32;
    const double vn = (nb + lane < g.hi) ? g.t[nb + lane] : 0.0;
    const long long rem = g.hi - base;
    const int cnt = rem < 32 ? static_cast<int>(rem) : 32;
    for (int j = 0; j < cnt; ++j) s += __shfl_sync(kFull, v, j);
    v = vn;
    base = nb;
  }
  if (lane == 0) *g.out = s;
}

static __global__ void k_tree1(const TreeSeg* segs, int nseg, double* partials, const int* skip) {
  __shared__ double sh[32];
  if (skip && *skip) return;
  const int s = blockIdx.x / kTreeBlocks, b = blockIdx.x % kTreeBlocks;
  if (s >= nseg) return;
  const TreeSeg g = segs[s];
  const long long len = g.hi - g.lo;
  const long long a = g.lo + len * b / kTreeBlocks, e = g.lo + len * (b + 1) / kTreeBlocks;
  double acc = 0.0;
  for (long long i = a + threadIdx.x; i < e; i += blockDim.x) acc += g.t[i];
  acc = block_sum_fixed(acc, sh);
  if (threadIdx.x == 0) partials[static_cast<long long>(s) * kTreeBlocks + b] = acc;
}

static __global__ void k_tree2(const TreeSeg* segs, int nseg, const double* partials, const int* skip) {
  __shared__ double sh[32];
  if (skip && *skip) return;
  const int s = blockIdx.x;
  if (s >= nseg) return;
  double acc = 0.0;
  for (int i = threadIdx.x; i < kTreeBlocks; i += blockDim.x) acc += partials[static_cast<long long>(s) * kTreeBlocks + i];
  acc = block_sum_fixed(acc, sh);
  if (threadIdx.x == 0) *segs[s].out = segs[s].init + acc;
}

// A fixed set of sums over fixed term arrays. Built once (descriptors live on the device),
// launched any number of times, also inside stream capture.
class SumPlan {
 public:
  void add(const double* terms, long long lo, long long hi, double init, SumOrder order, double* out) {
    jobs_.push_back({terms, lo, hi, init, order, out});
  }
  // skip: optional device int; when non-zero at run time every kernel of the plan returns.
  // st: the stream the plan is launched on; the segment descriptors are copied to the device on
  // it, so they are in place before the plan's first launch on that stream.
  void build(bool exact, const int* skip, cudaStream_t st) {
    exact_ = exact;
    skip_ = skip;
    std::vector<ChainSeg> phase1, phase2;
    std::vector<TreeSeg> tree;
    if (exact) {
      long long nchunk_jobs = 0;
      for (const Job& j : jobs_)
        if (j.order == SumOrder::kChunk64) ++nchunk_jobs;
      partials_.alloc(static_cast<std::size_t>(nchunk_jobs > 0 ? nchunk_jobs * kChunks : 1));
      long long slot = 0;
      for (const Job& j : jobs_) {
        const long long n = j.hi - j.lo;
        if (j.order == SumOrder::kSeq) {
          phase1.push_back({j.t, j.lo, j.hi, j.init, j.out});
        } else {
          const long long chunks = n < kChunks ? (n < 1 ? 1 : n) : kChunks;
          double* part = partials_.get() + slot * kChunks;
          for (long long c = 0; c < chunks; ++c)
            phase1.push_back({j.t, j.lo + n * c / chunks, j.lo + n * (c + 1) / chunks, 0.0, part + c});
          // parallel_sum: s = 0; s += part[c] in order — then the caller's init (0 for dots)
          phase2.push_back({part, 0, chunks, j.init, j.out});
          ++slot;
        }
      }
      upload(phase1, seg1_, st);
      upload(phase2, seg2_, st);
      n1_ = static_cast<int>(phase1.size());
      n2_ = static_cast<int>(phase2.size());
    } else {
      for (const Job& j : jobs_) tree.push_back({j.t, j.lo, j.hi, j.init, j.out});
      upload(tree, tseg_, st);
      nt_ = static_cast<int>(tree.size());
      partials_.alloc(static_cast<std::size_t>(nt_ > 0 ? nt_ : 1) * kTreeBlocks);
    }
  }
  void launch(cudaStream_t st) const {
    if (exact_) {
      if (n1_ > 0) {
        const int warps_per_block = 4;
        k_chain<<<(n1_ + warps_per_block - 1) / warps_per_block, 32 * warps_per_block, 0, st>>>(
            reinterpret_cast<const ChainSeg*>(seg1_.get()), n1_, skip_);
        B200_LAUNCH_CHECK();
      }
      if (n2_ > 0) {
        k_chain<<<(n2_ + 3) / 4, 128, 0, st>>>(reinterpret_cast<const ChainSeg*>(seg2_.get()), n2_, skip_);
        B200_LAUNCH_CHECK();
      }
    } else if (nt_ > 0) {
      k_tree1<<<nt_ * kTreeBlocks, kBlock, 0, st>>>(reinterpret_cast<const TreeSeg*>(tseg_.get()), nt_,
                                                    partials_.get(), skip_);
      B200_LAUNCH_CHECK();
      k_tree2<<<nt_, kBlock, 0, st>>>(reinterpret_cast<const TreeSeg*>(tseg_.get()), nt_, partials_.get(), skip_);
      B200_LAUNCH_CHECK();
    }
  }
  int kernel_count() const { return exact_ ? (n1_ > 0) + (n2_ > 0) : (nt_ > 0 ? 2 : 0); }
  bool empty() const { return jobs_.empty(); }

 private:
  struct Job {
    const double* t;
    long long lo, hi;
    double init;
    SumOrder order;
    double* out;
  };
  // Stream-ordered copy from pageable memory: cudaMemcpyAsync stages the source before it
  // returns, and the device copy lands before any later work on `st`. (A plain cudaMemcpy on the
  // legacy stream may return before the copy lands and is not ordered with a non-blocking `st`.)
  template <class S>
  static void upload(const std::vector<S>& v, DevBuf<unsigned char>& dst, cudaStream_t st) {
    dst.alloc(v.size() * sizeof(S) + 1);
    if (!v.empty())
      B200_CHECK(cudaMemcpyAsync(dst.get(), v.data(), v.size() * sizeof(S), cudaMemcpyHostToDevice, st));
  }
  std::vector<Job> jobs_;
  bool exact_ = false;
  const int* skip_ = nullptr;
  DevBuf<unsigned char> seg1_, seg2_, tseg_;
  mutable DevBuf<double> partials_;
  int n1_ = 0, n2_ = 0, nt_ = 0;
};

}  // namespace b200
