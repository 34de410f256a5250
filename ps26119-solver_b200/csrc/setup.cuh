// setup.cuh — device-side problem setup: CSR/CSC structure and diagonal scaling.
//
// Reference: pdhg::make_scaled_problem (src/pdhg/scaling.cpp:37-142) and la::transpose /
// csr_from_model (src/la/csr.cpp:8-36), which the reference runs on the host (9.4 s of a
// 116 s solve at 1M rows). Here everything runs on the device and reproduces the
// reference's values bit for bit:
//   * CSR of A: rows sorted by column (the order la::transpose produces). Built by a
//     counting pass, an exclusive scan, an atomic scatter, and a per-row sort by column;
//     column indices are unique inside a row, so the sorted order is canonical and the
//     result is deterministic whatever the atomic order was.
//   * Ãᵀ in CSR = CSC of Ã with row indices sorted inside each column (la::transpose(Ã)).
//   * Scaling factors: min/max norms are order-free; 1-norms are summed per row in CSR
//     order and per column in increasing row order, as scaling.cpp:18-32 does; products
//     val *= r_i * c_j are applied identically to the CSR and the CSC copy.
#pragma once

#include "common.cuh"

namespace b200 {

// ------------------------------------------------------------------ scan (int, exclusive)
constexpr int kScanItems = 8;
constexpr int kScanTile = kBlock * kScanItems;  // 2048 elements per block

static __global__ void k_scan_tiles(const int* in, int* out, long long n, int* tile_sums) {
  __shared__ int sh[kBlock];
  const long long base = static_cast<long long>(blockIdx.x) * kScanTile + threadIdx.x * kScanItems;
  int v[kScanItems];
  int sum = 0;
#pragma unroll
  for (int q = 0; q < kScanItems; ++q) {
    v[q] = (base + q < n) ? in[base + q] : 0;
    sum += v[q];
  }
  sh[threadIdx.x] = sum;
  __syncthreads();
  for (int off = 1; off < kBlock; off <<= 1) {  // Hillis-Steele inclusive scan of thread sums
    const int t = threadIdx.x >= off ? sh[threadIdx.x - off] : 0;
    __syncthreads();
    sh[threadIdx.x] += t;
    __syncthreads();
  }
  int run = sh[threadIdx.x] - sum;  // exclusive prefix of this thread
#pragma unroll
  for (int q = 0; q < kScanItems; ++q) {
    if (base + q < n) out[base + q] = run;
    run += v[q];
  }
  if (threadIdx.x == kBlock - 1 && tile_sums) tile_sums[blockIdx.x] = sh[kBlock - 1];
}
static __global__ void k_scan_add(int* out, long long n, const int* tile_offsets) {
  const long long i = static_cast<long long>(blockIdx.x) * kScanTile + threadIdx.x;
  const int add = tile_offsets[blockIdx.x];
  for (int q = 0; q < kScanItems; ++q) {
    const long long k = i + static_cast<long long>(q) * kBlock;
    if (k < n) out[k] += add;
  }
}

// Exclusive scan of n ints (out may alias in). Recursive over tile sums.
inline void exclusive_scan(const int* in, int* out, long long n, cudaStream_t st) {
  if (n <= 0) return;
  const long long tiles = (n + kScanTile - 1) / kScanTile;
  if (tiles == 1) {
    k_scan_tiles<<<1, kBlock, 0, st>>>(in, out, n, nullptr);
    B200_LAUNCH_CHECK();
    return;
  }
  DevBuf<int> sums(static_cast<std::size_t>(tiles)), offs(static_cast<std::size_t>(tiles));
  k_scan_tiles<<<static_cast<int>(tiles), kBlock, 0, st>>>(in, out, n, sums.get());
  B200_LAUNCH_CHECK();
  exclusive_scan(sums.get(), offs.get(), tiles, st);
  k_scan_add<<<static_cast<int>(tiles), kBlock, 0, st>>>(out, n, offs.get());
  B200_LAUNCH_CHECK();
  B200_CHECK(cudaStreamSynchronize(st));  // sums/offs are freed on return
}

// ------------------------------------------------------------------ transpose
static __global__ void k_count(long long nnz, const int* idx, int* counts) {
  B200_FOR(k, nnz) atomicAdd(counts + idx[k], 1);
}
// One thread per source row (CSC column j): entries go to their target rows at an atomic
// cursor; the per-row order is fixed afterwards by k_sort_rows.
static __global__ void k_scatter(int src_rows, const int* src_rp, const int* src_idx, const double* src_val,
                          int* cursor, int* dst_idx, double* dst_val) {
  B200_FOR(j, src_rows) {
    for (int k = src_rp[j]; k < src_rp[j + 1]; ++k) {
      const int p = atomicAdd(cursor + src_idx[k], 1);
      dst_idx[p] = static_cast<int>(j);
      dst_val[p] = src_val[k];
    }
  }
}

constexpr int kShortRow = 32;

// Rows of length <= kShortRow: insertion sort by key in registers. Longer rows are queued.
static __global__ void k_sort_short(int rows, const int* rp, int* key, double* val, int* long_rows, int* n_long) {
  B200_FOR(i, rows) {
    const int a = rp[i], b = rp[i + 1], len = b - a;
    if (len > kShortRow) {
      long_rows[atomicAdd(n_long, 1)] = static_cast<int>(i);
      continue;
    }
    int kk[kShortRow];
    double vv[kShortRow];
    for (int q = 0; q < len; ++q) kk[q] = key[a + q], vv[q] = val[a + q];
    for (int q = 1; q < len; ++q) {
      const int k0 = kk[q];
      const double v0 = vv[q];
      int p = q - 1;
      while (p >= 0 && kk[p] > k0) {
        kk[p + 1] = kk[p];
        vv[p + 1] = vv[p];
        --p;
      }
      kk[p + 1] = k0;
      vv[p + 1] = v0;
    }
    for (int q = 0; q < len; ++q) key[a + q] = kk[q], val[a + q] = vv[q];
  }
}

// One block per long row: bitonic network in the all-ascending form (each merge starts by
// comparing mirrored positions), run in place in global memory. Positions >= len act as +inf
// and never need to move, so no padding storage is required.
static __global__ void k_sort_long(const int* rp, const int* long_rows, const int* n_long, int* key, double* val) {
  const int nl = *n_long;
  for (int r = blockIdx.x; r < nl; r += gridDim.x) {
    const int row = long_rows[r];
    const int a = rp[row], len = rp[row + 1] - a;
    int P = 1;
    while (P < len) P <<= 1;
    int* kp = key + a;
    double* vp = val + a;
    for (int k = 2; k <= P; k <<= 1) {
      for (int j = k >> 1; j > 0; j >>= 1) {
        for (int i = threadIdx.x; i < P; i += blockDim.x) {
          const int partner = (j == (k >> 1)) ? (i ^ (k - 1)) : (i ^ j);
          if (partner > i && partner < len) {
            if (kp[i] > kp[partner]) {
              const int tk = kp[i];
              kp[i] = kp[partner];
              kp[partner] = tk;
              const double tv = vp[i];
              vp[i] = vp[partner];
              vp[partner] = tv;
            }
          }
        }
        __syncthreads();
      }
    }
    __syncthreads();
  }
}

// ------------------------------------------------------------------ scaling kernels
static __global__ void k_abs_range(long long nnz, const double* v, unsigned long long* amin_key,
                                   unsigned long long* amax_key) {
  double lo = INFINITY, hi = 0.0;
  B200_FOR(k, nnz) {
    const double a = fabs(v[k]);
    if (v[k] != 0.0) lo = std_min(lo, a), hi = std_max(hi, a);
  }
  warp_min_atomic_pos(amin_key, lo == INFINITY ? 0.0 : lo);
  warp_max_atomic(amax_key, hi);
}

__device__ __forceinline__ double clampf_gm(double v) { return std_min(std_max(v, 1e-20), 1e20); }
__device__ __forceinline__ double safe_inv_sqrt(double v) { return v > 0.0 && isfinite(v) ? 1.0 / sqrt(v) : 1.0; }

// Geometric-mean sweep over rows of a CSR of ORIGINAL values (scaling.cpp:65-74):
// out_i = clampf(1/(sqrt(lo_i) sqrt(hi_i))) over v = |a_ij| * other_j (positive, finite).
static __global__ void k_gm_pass(int rows, const int* rp, const int* idx, const double* val, const double* other,
                          double* out) {
  B200_FOR(i, rows) {
    double lo = INFINITY, hi = 0.0;
    for (int k = rp[i]; k < rp[i + 1]; ++k) {
      const double v = fabs(val[k]) * other[idx[k]];
      if (v > 0 && isfinite(v)) lo = std_min(lo, v), hi = std_max(hi, v);
    }
    if (hi > 0) out[i] = clampf_gm(1.0 / (sqrt(lo) * sqrt(hi)));
  }
}

// Per-row ∞-norm (max |a|) or 1-norm (Σ|a| in storage order) of a CSR (scaling.cpp:18-32).
static __global__ void k_row_norm(int rows, const int* rp, const double* val, int inf_norm, double* out) {
  B200_FOR(i, rows) {
    double s = 0.0;
    for (int k = rp[i]; k < rp[i + 1]; ++k) {
      const double a = fabs(val[k]);
      if (inf_norm) s = std_max(s, a);
      else s += a;
    }
    out[i] = s;
  }
}

static __global__ void k_inv_sqrt_factor(long long n, const double* norm, double* f, double* scale) {
  B200_FOR(i, n) {
    f[i] = safe_inv_sqrt(norm[i]);
    scale[i] *= f[i];
  }
}

// val[k] *= rf[row] * cf[col] on a CSR (rows = rows of A) ...
static __global__ void k_apply_csr(int rows, const int* rp, const int* col, double* val, const double* rf,
                            const double* cf) {
  B200_FOR(i, rows) {
    const double r = rf[i];
    for (int k = rp[i]; k < rp[i + 1]; ++k) val[k] *= r * cf[col[k]];
  }
}
// ... and on the CSC copy (rows of the CSR = columns of A): same product r_i * c_j.
static __global__ void k_apply_csc(int cols, const int* cp, const int* row, double* val, const double* rf,
                            const double* cf) {
  B200_FOR(j, cols) {
    const double c = cf[j];
    for (int k = cp[j]; k < cp[j + 1]; ++k) val[k] *= rf[row[k]] * c;
  }
}

static __global__ void k_copy_scale(long long n, const double* src, double* dst) {
  B200_FOR(i, n) dst[i] = src[i];
}

// Scaled vectors before the bound/objective scalars (scaling.cpp:111-124).
static __global__ void k_scaled_cols(int n, int sense, const double* c, const double* cl, const double* cu,
                              const double* col_scale, double* sc, double* scl, double* scu) {
  B200_FOR(j, n) {
    sc[j] = col_scale[j] * static_cast<double>(sense) * c[j];
    scl[j] = cl[j] / col_scale[j];
    scu[j] = cu[j] / col_scale[j];
  }
}
static __global__ void k_scaled_rows(int m, const double* rl, const double* ru, const double* row_scale, double* srl,
                              double* sru) {
  B200_FOR(i, m) {
    srl[i] = row_scale[i] * rl[i];
    sru[i] = row_scale[i] * ru[i];
  }
}
// Terms of ‖b̃‖² (max of |finite bounds| per row) and ‖c̃‖² (scaling.cpp:127-135).
static __global__ void k_b2_terms(int m, const double* rl, const double* ru, double* t) {
  B200_FOR(i, m) {
    const double lo = isfinite(rl[i]) ? fabs(rl[i]) : 0.0;
    const double up = isfinite(ru[i]) ? fabs(ru[i]) : 0.0;
    const double b = std_max(lo, up);
    t[i] = b * b;
  }
}
static __global__ void k_sq_terms(long long n, const double* v, double* t) {
  B200_FOR(i, n) t[i] = v[i] * v[i];
}
static __global__ void k_scale_vec(long long n, double* v, double s) {
  B200_FOR(i, n) v[i] *= s;
}
template <class D, class S>
static __global__ void k_convert(long long n, const S* src, D* dst) {
  B200_FOR(i, n) dst[i] = static_cast<D>(src[i]);
}

}  // namespace b200
