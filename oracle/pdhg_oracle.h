/* pdhg_oracle.h — TEST ORACLE (checker only; never linked into the product).
 *
 * A single-threaded C restatement of the reference's first-order r²HPDHG path
 * (JaiVerma20/ps26119-solver), written so that every floating-point operation happens in the
 * reference's order: row-sequential CSR products, 64-chunk ordered partial sums for dot
 * products (src/la/parallel.h:169-188), fully sequential host loops where the reference uses
 * them, no FMA contraction (compiled with -ffp-contract=off). Its results are therefore
 * bit-identical to the reference CPU engine for any reference thread count.
 *
 * Pinning: tests/test_oracle_vs_reference.py compares it bit-for-bit against the reference
 * built from its own sources (oracle/_ref) and against the reference's known answers
 * (tests/golden/).
 *
 * Reference files restated (file:line in the reference project):
 *   scaling            src/pdhg/scaling.cpp:37-155, scaling.h:32-46
 *   CSR / transpose    src/la/csr.h:30-43, src/la/csr.cpp:19-36
 *   ‖A‖₂ (Lanczos)     src/la/csr.cpp:54-132
 *   backend ops        src/pdhg/cpu_backend.cpp:113-215
 *   KKT                src/pdhg/cpu_backend.cpp:226-284, src/pdhg/termination.h:35-60
 *   ray test           src/pdhg/engine.cpp:82-184
 *   precision policy   src/pdhg/engine.cpp:56-79, 186-192
 *   context / finish   src/pdhg/engine.cpp:195-307
 *   r²HPDHG loop       src/pdhg/r2hpdhg.cpp:11-162
 */
#ifndef PDHG_ORACLE_H
#define PDHG_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  int m, n, sense;
  double offset;
  const double *c, *col_lower, *col_upper, *row_lower, *row_upper;
  const int *col_start, *row_index;
  const double* value;
} orc_model;

typedef struct {
  int ruiz_iterations;           /* 10 */
  int pock_chambolle;            /* 1 */
  int bound_objective_rescaling; /* 1 */
  int geometric_mean_iterations; /* 12 */
  double geometric_mean_min_log10_range; /* 4.5 */
} orc_scaling_options;

typedef struct {
  double tolerance;         /* 1e-8 */
  long long iteration_limit;/* 100,000,000 */
  int check_every;          /* 64 */
  int mixed;                /* 0 fp64, 1 mixed */
  orc_scaling_options scaling;
  double reflection, restart_sufficient, restart_necessary, restart_artificial;
  double pid_kp, pid_ki, pid_kd, pid_integral_decay, pid_max_log_step;
  const double* warm_x; /* n or NULL */
  const double* warm_y; /* m or NULL */
  double warm_primal_weight;
} orc_options;

typedef struct {
  int status; /* 0 Optimal .. 6 NotSolved (reference Status order) */
  long long iterations;
  double objective, dual_objective, primal_residual, dual_residual, gap;
  double primal_weight, eta, initial_primal_weight;
  long long iterations_to_fast, switch_iteration;
  long long restarts, checks;
  char message[256];
} orc_result;

void orc_default_options(orc_options* o);

/* Full r²HPDHG solve (no presolve, no gate): the reference's
 * ps26119::solve(model, {algorithm=R2hpdhg, presolve=false}) engine result. x, z (n), y (m),
 * dual_ray (m), primal_ray (n) may be NULL. Returns status. */
int orc_solve_r2hpdhg(const orc_model* M, const orc_options* o, orc_result* r, double* x, double* y, double* z,
                      double* dual_ray, double* primal_ray);

/* Scaled problem (make_scaled_problem) and its ‖Ã‖₂ estimate. */
typedef struct orc_scaled orc_scaled;
orc_scaled* orc_scale(const orc_model* M, const orc_scaling_options* so);
void orc_scaled_free(orc_scaled* sp);
/* which: 0 Ã vals (CSR), 1 Ãᵀ vals (CSR), 2 c̃, 3 l̃, 4 ũ, 5 r̃l, 6 r̃u, 7 row_scale, 8 col_scale */
long long orc_scaled_get(const orc_scaled* sp, int which, double* dst);
/* out = [bound_scale, obj_scale, log10_range, geometric_mean_applied] */
void orc_scaled_scalars(const orc_scaled* sp, double* out);
double orc_norm2(const orc_scaled* sp);

/* The CPU backend (cpu_backend.cpp) over an orc_scaled problem: the op-by-op checker. */
typedef struct orc_backend orc_backend;
orc_backend* orc_backend_new(const orc_scaled* sp);
void orc_backend_free(orc_backend* b);
void orc_backend_set_precision(orc_backend* b, int mixed);
int orc_backend_create(orc_backend* b, int dual);
void orc_backend_upload(orc_backend* b, int v, const double* src);
void orc_backend_download(orc_backend* b, int v, double* dst);
void orc_backend_fill(orc_backend* b, int v, double a);
void orc_backend_copy(orc_backend* b, int dst, int src);
void orc_backend_axpby(orc_backend* b, double a, int x, double bb, int y);
void orc_backend_spmv(orc_backend* b, int x, int out);
void orc_backend_spmv_t(orc_backend* b, int y, int out);
double orc_backend_dot(orc_backend* b, int x, int y);
double orc_backend_norm2(orc_backend* b, int x);
double orc_backend_diff_norm2(orc_backend* b, int x, int y);
void orc_backend_primal_step(orc_backend* b, int x, int aty, double tau, int xh);
void orc_backend_dual_step(orc_backend* b, int y, int ax, double sigma, int yh);
void orc_backend_r2h_primal(orc_backend* b, int x, int x0, int aty, double tau, double w, double rho, int xh, int xb);
void orc_backend_r2h_dual(orc_backend* b, int y, int y0, int ax, double sigma, double w, double rho, int yh, int yb);
/* out = [primal_residual, dual_residual, primal_obj, dual_obj, b_norm, c_norm, primal_max_rel, dual_max_rel] */
void orc_backend_kkt(orc_backend* b, int xs, int ys, double* out);

#ifdef __cplusplus
}
#endif
#endif
