/* ps26119.h — C ABI of the B200 r²HPDHG engine (libps26119.so).
 *
 * Drop-in for the reference's C API (JaiVerma20/ps26119-solver include/ps26119/ps26119.h):
 * the same five symbols, the same struct layouts, status codes, argument meaning and error
 * behaviour. The model is
 *     minimise / maximise   cᵀx + obj_offset
 *     subject to            row_lower ≤ A x ≤ row_upper,   col_lower ≤ x ≤ col_upper
 * with A in CSC: col_start[n+1], row_index[nnz], value[nnz]. Infinity = HUGE_VAL. Duals follow
 * z = c − Aᵀy (HiGHS signs).
 *
 * This library runs the first-order r²HPDHG engine on the GPU. A request for another
 * algorithm, or with use_gpu = 0, returns PS26119_NOT_SOLVED with the reason in
 * result->message: there is no CPU fallback.
 *
 * No function throws or aborts: every error is returned as a status code.
 */
#ifndef PS26119_B200_C_API_H
#define PS26119_B200_C_API_H

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

/* Status codes (same meaning and order as the reference ps26119::Status;
 * reference include/ps26119/ps26119.h:19-28). */
enum {
  PS26119_OPTIMAL = 0,
  PS26119_INFEASIBLE = 1,
  PS26119_UNBOUNDED = 2,
  PS26119_ITERATION_LIMIT = 3,
  PS26119_TIME_LIMIT = 4,
  PS26119_NUMERICAL_ERROR = 5,
  PS26119_NOT_SOLVED = 6,
  PS26119_INVALID_ARGUMENT = 7
};

/* reference include/ps26119/ps26119.h:30-31 */
enum { PS26119_ALG_AUTO = 0, PS26119_ALG_ORACLE = 1, PS26119_ALG_PDLP = 2, PS26119_ALG_R2HPDHG = 3, PS26119_ALG_SIMPLEX = 4 };
enum { PS26119_PREC_FP64 = 0, PS26119_PREC_MIXED = 1 };

/* reference include/ps26119/ps26119.h:33-45 (identical layout) */
typedef struct {
  int algorithm;             /* PS26119_ALG_* (AUTO and R2HPDHG run r²HPDHG on the GPU) */
  int precision;             /* PS26119_PREC_* */
  int use_gpu;               /* must be 1 for this library */
  double tolerance;          /* relative KKT target (0 = default 1e-8) */
  double time_limit;         /* seconds (0 = default 3600); negative or NaN -> INVALID_ARGUMENT */
  long long iteration_limit; /* 0 = default; negative -> INVALID_ARGUMENT */
  int verbosity;
  int threads;               /* host threads for presolve/verification; results never depend on it */
  const double* warm_x;      /* warm start x (num_cols) or NULL */
  const double* warm_y;      /* warm start y (num_rows) or NULL */
} ps26119_options;

/* reference include/ps26119/ps26119.h:47-63 (identical layout) */
typedef struct {
  int status;
  double objective;
  double dual_objective;
  double primal_residual;
  double dual_residual;
  double gap;
  double certified_bound; /* rounding-proof bound from y; NaN when not computed */
  long long iterations;
  double seconds;
  char engine[16];
  char message[160];
  int check;              /* 1 PASS, 0 FAIL, -1 not applicable */
} ps26119_result;

/* Replaces reference ps26119_version (ps26119.h:66; c_api.cpp:177). */
PS26119_API const char* ps26119_version(void);

/* Replaces reference ps26119_default_options (ps26119.h:69; c_api.cpp:179-192). The defaults
 * are the reference's (AUTO, fp64, use_gpu = 0, 1e-8, 3600 s): set use_gpu = 1. */
PS26119_API void ps26119_default_options(ps26119_options* opt);

/* Replaces reference ps26119_solve_lp (ps26119.h:74-78; c_api.cpp:194-200). */
PS26119_API int ps26119_solve_lp(int num_rows, int num_cols, int sense, double obj_offset, const double* c,
                     const double* col_lower, const double* col_upper, const double* row_lower,
                     const double* row_upper, const int* col_start, const int* row_index,
                     const double* value, const ps26119_options* opt, ps26119_result* result,
                     double* x, double* y, double* z);

/* Replaces reference ps26119_solve_lp_ex (ps26119.h:84-88; c_api.cpp:202-259). Presolve runs
 * on the host as in the reference (always on behind the C API), the engine on the GPU, the
 * in-process check on the original model fills result->check. */
PS26119_API int ps26119_solve_lp_ex(int num_rows, int num_cols, int sense, double obj_offset, const double* c,
                        const double* col_lower, const double* col_upper, const double* row_lower,
                        const double* row_upper, const int* col_start, const int* row_index,
                        const double* value, const ps26119_options* opt, ps26119_result* result,
                        double* x, double* y, double* z, double* dual_ray, double* primal_ray);

/* Replaces reference ps26119_solve_mps (ps26119.h:90-94; c_api.cpp:161-202): reads an MPS file
 * (free or fixed format), solves it, and writes the solution file (the reference's .sol format)
 * when solution_path is non-NULL. Read errors return PS26119_INVALID_ARGUMENT with the reason and
 * line in result->message. Integer markers are read but the LP relaxation is solved (this library
 * has no MILP engine); the message then starts with "LP relaxation (integrality ignored)". */
PS26119_API int ps26119_solve_mps(const char* path, const ps26119_options* opt, ps26119_result* result,
                      const char* solution_path);

/* ------------------------------------------------------------------ additions
 * Engine-level controls that the reference keeps in its C++ Options (include/ps26119/
 * options.h:37-82) and EngineOptions (src/pdhg/engine.h:27-48) but not in the C struct. */
typedef struct {
  int presolve;              /* 1 = reference default (host presolve + postsolve), 0 = engine only */
  int check_every;           /* K, iterations between checks (0 = 64) */
  int exact_reductions;      /* 1 = every reduction in the reference's summation order (bit-identical
                                trajectory to the reference CPU engine; for modest sizes); 0 = fixed-order
                                tree reductions (deterministic, fast) */
  int ruiz_iterations;       /* -1 = default 10 */
  int pock_chambolle;        /* -1 = default 1 */
  int bound_objective_rescaling; /* -1 = default 1 */
  double reflection;         /* 0 = default 1.0 */
  double warm_primal_weight; /* > 0: start from this primal weight */
  int mixed_stall_checks;    /* precision = mixed: checks without a 10% gain of the best relative KKT
                                before the switch to fp64 (0 = the reference's 10; the switch at
                                relative KKT 1e-6 applies either way) */
  int reserved;              /* 0 */
} ps26119_engine_options;

PS26119_API void ps26119_default_engine_options(ps26119_engine_options* eo);

/* As ps26119_solve_lp_ex with engine options (NULL = defaults). Host arrays. */
PS26119_API int ps26119_solve_lp_engine(int num_rows, int num_cols, int sense, double obj_offset, const double* c,
                            const double* col_lower, const double* col_upper, const double* row_lower,
                            const double* row_upper, const int* col_start, const int* row_index,
                            const double* value, const ps26119_options* opt,
                            const ps26119_engine_options* eo, ps26119_result* result, double* x,
                            double* y, double* z, double* dual_ray, double* primal_ray);

/* Device-resident solve: every array argument (model and outputs) is a DEVICE pointer on the
 * current device; stream is a cudaStream_t (NULL = a stream of the library's own). No presolve
 * (the model must be valid: the caller owns validation), no host copies of the model. Outputs
 * x, z (n) and y (m) are written on the device when non-NULL; result is host memory.
 * Engine options as above (NULL = defaults). result->check is the in-process check computed
 * on the device; result->certified_bound is NaN. */
PS26119_API int ps26119_solve_lp_device(int num_rows, int num_cols, int sense, double obj_offset, const double* d_c,
                            const double* d_col_lower, const double* d_col_upper, const double* d_row_lower,
                            const double* d_row_upper, const int* d_col_start, const int* d_row_index,
                            const double* d_value, const ps26119_options* opt,
                            const ps26119_engine_options* eo, ps26119_result* result, double* d_x,
                            double* d_y, double* d_z, void* stream);

/* Extra statistics of the last solve on the calling thread (host memory, filled by every
 * solve entry point). */
typedef struct {
  double setup_seconds;      /* scaling, ‖A‖₂, uploads */
  double loop_seconds;       /* iterations + checks */
  double finish_seconds;
  double presolve_seconds;
  double primal_weight;
  double eta;
  long long checks, restarts;
  long long iterations_to_fast;
  long long switch_iteration;  /* mixed precision: iteration of the fp32 -> fp64 promotion, -1 if none */
  long long kernel_launches;   /* kernels launched by the solve (graph nodes counted per replay) */
  long long m, n, nnz;         /* size of the problem the engine ran on (after presolve) */
  double spmv_kernel_ms;       /* total device time of the fused iteration kernels (CUDA events) */
  long long spmv_kernel_launches;
  double teardown_seconds;     /* releasing the engine's device state after the loop */
  double call_seconds;         /* the whole entry-point call, host wall clock */
  int slab_variant_primal;     /* launch variants of the fused iteration kernels picked by the */
  int slab_variant_dual;       /*   autotuner for this matrix (indices of the library's variant list) */
  int tuned;                   /* 1: this solve timed the variants itself (first of its shape class) */
  int reserved;
} ps26119_stats;

PS26119_API void ps26119_last_stats(ps26119_stats* out);

/* certified_dual_bound (reference src/core/safe_bound.h:37-43, C++ only there): a
 * rounding-error-proof bound on the model's optimum from ANY row multipliers y (the model's
 * sense, as ps26119_result's y): at most the optimum for a minimisation, at least for a
 * maximisation, infinite when a multiplier or reduced cost points at an infinite bound.
 * use_implied_bounds = 1 lets columns bounded on one side take rigorous implied bounds.
 * Host computation (no GPU). out[4] = finite (0/1), bound, unbounded row terms, unbounded
 * column terms. Returns 0, or PS26119_INVALID_ARGUMENT for an invalid model. */
PS26119_API int ps26119_certified_bound(int num_rows, int num_cols, int sense, double obj_offset, const double* c,
                                        const double* col_lower, const double* col_upper, const double* row_lower,
                                        const double* row_upper, const int* col_start, const int* row_index,
                                        const double* value, const double* y, int use_implied_bounds, double* out);

/* check_infeasibility_certificate / check_unboundedness_certificate (reference
 * src/core/certificates.h:41-43): kind 0 checks a Farkas vector `ray` (num_rows values; x is
 * ignored), kind 1 a feasible point x and a recession ray (num_cols values each). Host
 * computation. out[5] = present, passed, rigorous (Farkas stage 1), measure, violation. Returns 0,
 * or PS26119_INVALID_ARGUMENT. */
PS26119_API int ps26119_check_certificate(int kind, int num_rows, int num_cols, int sense, double obj_offset,
                                          const double* c, const double* col_lower, const double* col_upper,
                                          const double* row_lower, const double* row_upper, const int* col_start,
                                          const int* row_index, const double* value, const double* x,
                                          const double* ray, double* out);

/* One scenario of a batch: host arrays of the base model's sizes (a pointer carries no length:
 * each array must hold n or m values); NULL keeps the base's vector (an empty vector in the
 * reference's ps26119::Scenario, include/ps26119/batch.h:22-28). */
typedef struct {
  const double* obj;
  const double* col_lower;
  const double* col_upper;
  const double* row_lower;
  const double* row_upper;
} ps26119_scenario;

/* ps26119::solve_batch (reference include/ps26119/batch.h:32-33, src/pdhg/batch.cpp:129-441,
 * which the reference offers in C++ and through its CLI `batch` command): K LPs that share the
 * base model's matrix, solved by r²HPDHG in lockstep on the GPU, fp64, no presolve, no
 * infeasibility detection (as the reference). results[k] receives scenario k's outcome (status,
 * objective, residuals, iterations, engine "r2hpdhg-batch"); x (K×n), y (K×m), z (K×n),
 * scenario-major, may be NULL. engine may be NULL; its presolve and warm_primal_weight fields are
 * ignored. opt->use_gpu is ignored (the batch always runs on the GPU). Returns 0 when the batch
 * ran (per-scenario status in results), or PS26119_INVALID_ARGUMENT / PS26119_NOT_SOLVED with the
 * reason in every results[k].message. */
PS26119_API int ps26119_solve_batch(int num_rows, int num_cols, int sense, double obj_offset, const double* c,
                                    const double* col_lower, const double* col_upper, const double* row_lower,
                                    const double* row_upper, const int* col_start, const int* row_index,
                                    const double* value, int num_scenarios, const ps26119_scenario* scenarios,
                                    const ps26119_options* opt, const ps26119_engine_options* engine,
                                    ps26119_result* results, double* x, double* y, double* z);

/* ---- Serving: a request loop for independent LPs on one GPU (continuous batching).
 * No reference counterpart: the reference solves one LP per call. Requests are admitted in
 * arrival order when one of `slots` is free and the device memory the request needs fits in the
 * HBM budget left by the requests running (the first request in flight is always admitted). Each
 * slot runs the same solve as ps26119_solve_lp_ex (presolve, the GPU engine on the slot's own
 * stream, the gate), so a request's result equals that call's result; requests that arrive while
 * others run start as slots and memory free up, and their work overlaps on the device. */
typedef struct ps26119_server ps26119_server;

typedef struct {
  int slots;               /* requests solved at the same time (0 = 8) */
  double hbm_budget_bytes; /* device memory for the running requests (0 = 80% of free memory) */
  double dry_run_seconds;  /* > 0: requests are admitted and timed but not solved (each holds its
                              slot and memory this long); status NOT_SOLVED, engine "dry-run" */
  int solo_engines;        /* 0 (default): the r²HPDHG epochs of all running requests are launched
                              together, one grouped kernel per half-step over every request's
                              slabs; 1: each request's engine launches its own kernels */
} ps26119_server_options;

typedef struct {
  double submitted, started, finished; /* seconds on the server's steady clock */
} ps26119_request_times;

/* A server on the current device; NULL if opt has a negative field (opt NULL = defaults). */
PS26119_API ps26119_server* ps26119_server_create(const ps26119_server_options* opt);

/* Queues one LP (the arguments of ps26119_solve_lp_ex; the library copies them). Returns the
 * request id (>= 0), or -PS26119_INVALID_ARGUMENT with the reason in error->message (error may
 * be NULL) when the model or the options are invalid. */
PS26119_API long long ps26119_server_submit(ps26119_server* server, int num_rows, int num_cols, int sense,
                                            double obj_offset, const double* c, const double* col_lower,
                                            const double* col_upper, const double* row_lower,
                                            const double* row_upper, const int* col_start,
                                            const int* row_index, const double* value,
                                            const ps26119_options* opt, ps26119_result* error);

/* Request `id`: 1 when it has finished (waiting for it if wait != 0) — result, x, y, z (each
 * may be NULL) and times are written and the request is forgotten; 0 while it is pending; -1
 * for an unknown id. */
PS26119_API int ps26119_server_poll(ps26119_server* server, long long id, int wait, ps26119_result* result,
                                    double* x, double* y, double* z, ps26119_request_times* times);

/* Finishes every request already submitted, then releases the server. */
PS26119_API void ps26119_server_destroy(ps26119_server* server);

#ifdef __cplusplus
}
#endif

#endif /* PS26119_B200_C_API_H */
