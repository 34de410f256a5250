/* ps26119_backend.h — C ABI of the GPU backend plugin (libps26119.so).
 *
 * The reference's internal plugin boundary is the C++ class pdhg::Backend
 * (src/pdhg/backend.h:36-69) with make_backend(use_gpu, error) (backend.h:87): vector handles,
 * spmv / spmv_t, fused r²HPDHG steps, fp64 reductions and the KKT evaluation. This header
 * exposes the same operations over the GPU implementation with plain C types, so a reference
 * maintainer (or a test) can drive the GPU op by op exactly as tests/unit/test_gpu.cpp:33-95
 * drives the CUDA backend against the CPU one.
 *
 * Every function returns 0 on success and a non-zero PS26119_* status on failure (with the
 * reason in the thread's last-error text, ps26119_backend_last_error). Nothing throws.
 */
#ifndef PS26119_B200_BACKEND_H
#define PS26119_B200_BACKEND_H

#ifndef PS26119_API
#if defined(__GNUC__)
#define PS26119_API __attribute__((visibility("default")))
#else
#define PS26119_API
#endif
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ps26119_backend ps26119_backend;

/* Scaling options (reference src/pdhg/scaling.h:32-46); NULL = defaults
 * (12 geometric-mean sweeps when the entries span 10^4.5, Ruiz 10, Pock–Chambolle, bound and
 * objective rescaling). */
typedef struct {
  int geometric_mean_iterations;
  double geometric_mean_min_log10_range;
  int ruiz_iterations;
  int pock_chambolle;
  int bound_objective_rescaling;
} ps26119_scaling_options;

/* Creates the backend and runs Backend::setup on the GPU: uploads the CSC model (host arrays,
 * same layout as ps26119_solve_lp) and builds the scaled problem on the device
 * (make_scaled_problem, reference src/pdhg/scaling.cpp:37-142). exact = 1 takes every
 * reduction in the reference's summation order. Replaces make_backend(true, error)
 * (reference src/pdhg/cpu_backend.cpp:293-310) + Backend::setup. */
PS26119_API int ps26119_backend_new(ps26119_backend** out, int num_rows, int num_cols, int sense, double obj_offset,
                        const double* c, const double* col_lower, const double* col_upper,
                        const double* row_lower, const double* row_upper, const int* col_start,
                        const int* row_index, const double* value, const ps26119_scaling_options* so,
                        int exact);
PS26119_API void ps26119_backend_free(ps26119_backend* b);
PS26119_API const char* ps26119_backend_last_error(void);

/* Backend::set_precision / create / upload / download / fill / copy / axpby (backend.h:43-51) */
PS26119_API int ps26119_backend_set_precision(ps26119_backend* b, int mixed);
PS26119_API int ps26119_backend_create(ps26119_backend* b, int dual); /* returns the handle (>= 0), or -1 */
PS26119_API int ps26119_backend_upload(ps26119_backend* b, int v, const double* src);
PS26119_API int ps26119_backend_download(ps26119_backend* b, int v, double* dst);
PS26119_API int ps26119_backend_fill(ps26119_backend* b, int v, double a);
PS26119_API int ps26119_backend_copy(ps26119_backend* b, int dst, int src);
PS26119_API int ps26119_backend_axpby(ps26119_backend* b, double a, int x, double bb, int y);
/* Backend::spmv / spmv_t (backend.h:52-53) */
PS26119_API int ps26119_backend_spmv(ps26119_backend* b, int x, int out);
PS26119_API int ps26119_backend_spmv_t(ps26119_backend* b, int y, int out);
/* Backend::dot / norm2 / diff_norm2 (backend.h:54-56), result in *out */
PS26119_API int ps26119_backend_dot(ps26119_backend* b, int x, int y, double* out);
PS26119_API int ps26119_backend_norm2(ps26119_backend* b, int x, double* out);
PS26119_API int ps26119_backend_diff_norm2(ps26119_backend* b, int x, int y, double* out);
/* Backend::primal_step / dual_step / r2h_primal / r2h_dual (backend.h:58-61); yb = -1 skips ȳ */
PS26119_API int ps26119_backend_primal_step(ps26119_backend* b, int x, int aty, double tau, int xh);
PS26119_API int ps26119_backend_dual_step(ps26119_backend* b, int y, int ax, double sigma, int yh);
PS26119_API int ps26119_backend_r2h_primal(ps26119_backend* b, int x, int x0, int aty, double tau, double w, double rho,
                               int xh, int xb);
PS26119_API int ps26119_backend_r2h_dual(ps26119_backend* b, int y, int y0, int ax, double sigma, double w, double rho,
                             int yh, int yb);
/* The engine's fused kernels: Ãᵀy + r2h_primal in one launch, Ãx̄ + r2h_dual in one launch
 * (no reference counterpart as single calls; equal to spmv_t + r2h_primal, spmv + r2h_dual). */
PS26119_API int ps26119_backend_fused_primal(ps26119_backend* b, int y, int x, int x0, double tau, double w, double rho,
                                 int xh, int xb);
PS26119_API int ps26119_backend_fused_dual(ps26119_backend* b, int xb, int y, int y0, double sigma, double w, double rho,
                               int yh, int yb);
/* Backend::kkt (backend.h:65): out[8] = primal_residual, dual_residual, primal_obj, dual_obj,
 * b_norm, c_norm, primal_max_rel, dual_max_rel (termination.h:35-60) */
PS26119_API int ps26119_backend_kkt(ps26119_backend* b, int xs, int ys, double* out);
PS26119_API int ps26119_backend_sync(ps26119_backend* b);
/* Scaled problem introspection: which = 0 Ã values (CSR), 1 Ãᵀ values (CSR), 2 c̃, 3 l̃, 4 ũ,
 * 5 r̃l, 6 r̃u, 7 row scale, 8 column scale (the ScaledProblem fields, scaling.h:48-67).
 * Returns the element count (dst may be NULL to query it), or -1. */
PS26119_API long long ps26119_backend_scaled_get(ps26119_backend* b, int which, double* dst);
/* Structure of Ã (which = 0, m+1 row pointers) or Ãᵀ (which = 1, n+1); returns nnz. */
PS26119_API long long ps26119_backend_scaled_structure(ps26119_backend* b, int which, int* row_ptr, int* col);
/* out[4] = bound_scale, obj_scale, log10_range, geometric_mean_applied */
PS26119_API int ps26119_backend_scalars(ps26119_backend* b, double* out);
/* ‖Ã‖₂ estimate (la::estimate_norm2, reference src/la/csr.cpp:86-132) */
PS26119_API int ps26119_backend_norm2_estimate(ps26119_backend* b, double* out);

/* fp64 dot product Σ a_i·b_i of two DEVICE vectors of length n, written to the device double
 * *out on `stream` (a cudaStream_t; NULL = the legacy default stream). No counterpart in the
 * reference: it is for callers that cannot allocate device memory when they need the sum (a
 * caller whose device memory all belongs to its own pool, a loop that may not wait on the
 * allocator). It calls no cudaMalloc or cudaFree; its scratch is one fixed array in this
 * library's device code, at most n = 2,097,152 elements (16 MiB), held by every device that
 * loads the library until exit; larger n is rejected with PS26119_INVALID_ARGUMENT. The first
 * call on a device looks up that array's address (make it before any stream capture) and keeps
 * it: not for use after cudaDeviceReset. All calls on a device share the array, so calls that
 * overlap on the GPU race: serialise them on one stream.
 * exact = 1 sums in the reference's la::parallel_sum order and equals ps26119_backend_dot of an
 * exact backend bit for bit; exact = 0 equals the fast-mode ps26119_backend_dot.
 * Returns 0, or a PS26119_* status with the reason in ps26119_backend_last_error(). */
PS26119_API int ps26119_dot_noalloc(long long n, const double* a, const double* b, int exact, double* out,
                                    void* stream);

/* Σ of the DEVICE vector t[0, n) in fp64, written to the host double *out (synchronises
 * `stream`, a cudaStream_t; NULL = the legacy default stream).
 *   order 0: one sequential chain, init + t[0] + t[1] + … — the order of the reference's host
 *            loops (e.g. pdhg::kkt_general, src/pdhg/cpu_backend.cpp:226-284);
 *   order 1: la::parallel_sum (src/la/parallel.h:169-188): 64 contiguous chunks, each summed in
 *            order from 0, then init + part[0] + part[1] + … in order.
 * exact = 1 returns exactly what that sequential evaluation returns, bit for bit (ties, signed
 * zeros, infinities and NaN included); exact = 0 uses the engine's fixed-order tree (same result
 * run to run, different rounding). No reference counterpart: it exposes the engine's reduction
 * kernels to tests and to callers that need reference-order sums of device data.
 * Returns 0, or a PS26119_* status with the reason in ps26119_backend_last_error(). */
PS26119_API int ps26119_ordered_sum(long long n, const double* t, double init, int order, int exact, double* out,
                                    void* stream);

#ifdef __cplusplus
}
#endif

#endif /* PS26119_B200_BACKEND_H */
