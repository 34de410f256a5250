"""ps26119 — Python interface to the B200 r²HPDHG engine (ctypes over libps26119.so).

Same call shape as the reference's ctypes package (python/ps26119/__init__.py of
JaiVerma20/ps26119-solver):

    import numpy as np, ps26119
    res = ps26119.solve_lp(c, A, row_lower, row_upper, col_lower, col_upper, sense=-1)
    res.status, res.objective, res.x, res.y, res.z

A may be a dense 2-D array, a (col_start, row_index, value) CSC triple, or a scipy.sparse
matrix. Infinity = numpy.inf. The engine runs on the GPU: ``gpu`` defaults to True here
(the reference's default CPU engine is not part of this library; gpu=False returns
NOT_SOLVED with the reason, as the C API does).

Beyond the reference's API: ``engine`` (presolve switch, check interval, exact-order
reductions), :func:`solve_lp_device` (device-resident arrays), :func:`last_stats`, and
:class:`Backend` (the pdhg::Backend plugin operations on the GPU).

The library is looked up in $PS26119_LIB, then ../lib next to this package (the in-tree
build of ps26119-solver_b200/build.py). Nothing here falls back to a CPU implementation:
a missing library raises OSError.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass, field

import numpy as np

__all__ = ["solve_lp", "solve_lp_device", "solve_mps", "Result", "version", "last_stats", "Backend", "load",
           "OPTIMAL", "INFEASIBLE", "UNBOUNDED", "ITERATION_LIMIT", "TIME_LIMIT", "NUMERICAL_ERROR", "NOT_SOLVED",
           "INVALID_ARGUMENT", "LIB_PATH"]

OPTIMAL, INFEASIBLE, UNBOUNDED, ITERATION_LIMIT, TIME_LIMIT, NUMERICAL_ERROR, NOT_SOLVED, INVALID_ARGUMENT = range(8)
_STATUS = ["Optimal", "Infeasible", "Unbounded", "IterationLimit", "TimeLimit", "NumericalError", "NotSolved",
           "InvalidArgument"]
_ALG = {"auto": 0, "oracle": 1, "pdlp": 2, "r2hpdhg": 3, "simplex": 4}
_PREC = {"fp64": 0, "mixed": 1}
_CHECK = {1: "PASS", 0: "FAIL", -1: ""}

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(HERE), "lib", "libps26119.so")

_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int)


class _Options(ctypes.Structure):  # ps26119_options
    _fields_ = [("algorithm", ctypes.c_int), ("precision", ctypes.c_int), ("use_gpu", ctypes.c_int),
                ("tolerance", ctypes.c_double), ("time_limit", ctypes.c_double),
                ("iteration_limit", ctypes.c_longlong), ("verbosity", ctypes.c_int), ("threads", ctypes.c_int),
                ("warm_x", _D), ("warm_y", _D)]


class _Result(ctypes.Structure):  # ps26119_result
    _fields_ = [("status", ctypes.c_int), ("objective", ctypes.c_double), ("dual_objective", ctypes.c_double),
                ("primal_residual", ctypes.c_double), ("dual_residual", ctypes.c_double), ("gap", ctypes.c_double),
                ("certified_bound", ctypes.c_double), ("iterations", ctypes.c_longlong),
                ("seconds", ctypes.c_double), ("engine", ctypes.c_char * 16), ("message", ctypes.c_char * 160),
                ("check", ctypes.c_int)]


class _EngineOptions(ctypes.Structure):  # ps26119_engine_options
    _fields_ = [("presolve", ctypes.c_int), ("check_every", ctypes.c_int), ("exact_reductions", ctypes.c_int),
                ("ruiz_iterations", ctypes.c_int), ("pock_chambolle", ctypes.c_int),
                ("bound_objective_rescaling", ctypes.c_int), ("reflection", ctypes.c_double),
                ("warm_primal_weight", ctypes.c_double), ("mixed_stall_checks", ctypes.c_int),
                ("reserved", ctypes.c_int)]


class _Stats(ctypes.Structure):  # ps26119_stats
    _fields_ = [("setup_seconds", ctypes.c_double), ("loop_seconds", ctypes.c_double),
                ("finish_seconds", ctypes.c_double), ("presolve_seconds", ctypes.c_double),
                ("primal_weight", ctypes.c_double), ("eta", ctypes.c_double), ("checks", ctypes.c_longlong),
                ("restarts", ctypes.c_longlong), ("iterations_to_fast", ctypes.c_longlong),
                ("switch_iteration", ctypes.c_longlong), ("kernel_launches", ctypes.c_longlong),
                ("m", ctypes.c_longlong), ("n", ctypes.c_longlong), ("nnz", ctypes.c_longlong),
                ("spmv_kernel_ms", ctypes.c_double), ("spmv_kernel_launches", ctypes.c_longlong),
                ("teardown_seconds", ctypes.c_double), ("call_seconds", ctypes.c_double),
                ("slab_variant_primal", ctypes.c_int), ("slab_variant_dual", ctypes.c_int), ("tuned", ctypes.c_int),
                ("reserved", ctypes.c_int)]


class _Scenario(ctypes.Structure):  # ps26119_scenario
    _fields_ = [("obj", _D), ("col_lower", _D), ("col_upper", _D), ("row_lower", _D), ("row_upper", _D)]


class _ServerOptions(ctypes.Structure):  # ps26119_server_options
    _fields_ = [("slots", ctypes.c_int), ("hbm_budget_bytes", ctypes.c_double), ("dry_run_seconds", ctypes.c_double),
                ("solo_engines", ctypes.c_int)]


class _RequestTimes(ctypes.Structure):  # ps26119_request_times
    _fields_ = [("submitted", ctypes.c_double), ("started", ctypes.c_double), ("finished", ctypes.c_double)]


class _ScalingOptions(ctypes.Structure):  # ps26119_scaling_options
    _fields_ = [("geometric_mean_iterations", ctypes.c_int), ("geometric_mean_min_log10_range", ctypes.c_double),
                ("ruiz_iterations", ctypes.c_int), ("pock_chambolle", ctypes.c_int),
                ("bound_objective_rescaling", ctypes.c_int)]


_MODEL = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double, _D, _D, _D, _D, _D, _I, _I, _D]

# Every symbol the C headers declare (include/ps26119.h, include/ps26119_backend.h).
EXPORTS = ["ps26119_version", "ps26119_default_options", "ps26119_solve_lp", "ps26119_solve_lp_ex",
           "ps26119_solve_mps", "ps26119_default_engine_options", "ps26119_solve_lp_engine",
           "ps26119_solve_lp_device", "ps26119_last_stats", "ps26119_solve_batch",
           "ps26119_certified_bound", "ps26119_check_certificate", "ps26119_backend_new", "ps26119_backend_free",
           "ps26119_backend_last_error", "ps26119_backend_set_precision", "ps26119_backend_create",
           "ps26119_backend_upload", "ps26119_backend_download", "ps26119_backend_fill", "ps26119_backend_copy",
           "ps26119_backend_axpby", "ps26119_backend_spmv", "ps26119_backend_spmv_t", "ps26119_backend_dot",
           "ps26119_backend_norm2", "ps26119_backend_diff_norm2", "ps26119_backend_primal_step",
           "ps26119_backend_dual_step", "ps26119_backend_r2h_primal", "ps26119_backend_r2h_dual",
           "ps26119_backend_fused_primal", "ps26119_backend_fused_dual", "ps26119_backend_kkt",
           "ps26119_backend_sync", "ps26119_backend_scaled_get", "ps26119_backend_scaled_structure",
           "ps26119_backend_scalars", "ps26119_backend_norm2_estimate", "ps26119_dot_noalloc",
           "ps26119_ordered_sum",
           "ps26119_server_create", "ps26119_server_submit", "ps26119_server_poll", "ps26119_server_destroy"]

_lib = None


def load(path: str | None = None):
    """Loads libps26119.so (raises OSError when it is missing) and declares every signature."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or os.environ.get("PS26119_LIB") or LIB_PATH
    L = ctypes.CDLL(p)
    P = ctypes.POINTER
    L.ps26119_version.restype = ctypes.c_char_p
    L.ps26119_default_options.argtypes = [P(_Options)]
    L.ps26119_default_engine_options.argtypes = [P(_EngineOptions)]
    L.ps26119_solve_lp.argtypes = _MODEL + [P(_Options), P(_Result), _D, _D, _D]
    L.ps26119_solve_lp_ex.argtypes = _MODEL + [P(_Options), P(_Result), _D, _D, _D, _D, _D]
    L.ps26119_solve_lp_engine.argtypes = _MODEL + [P(_Options), P(_EngineOptions), P(_Result), _D, _D, _D, _D, _D]
    L.ps26119_solve_lp_device.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double] + \
        [ctypes.c_void_p] * 8 + [P(_Options), P(_EngineOptions), P(_Result)] + [ctypes.c_void_p] * 4
    L.ps26119_solve_mps.argtypes = [ctypes.c_char_p, P(_Options), P(_Result), ctypes.c_char_p]
    L.ps26119_last_stats.argtypes = [P(_Stats)]
    L.ps26119_solve_batch.argtypes = _MODEL + [ctypes.c_int, P(_Scenario), P(_Options), P(_EngineOptions),
                                               P(_Result), _D, _D, _D]
    L.ps26119_certified_bound.argtypes = _MODEL + [_D, ctypes.c_int, _D]
    L.ps26119_check_certificate.argtypes = [ctypes.c_int] + _MODEL + [_D, _D, _D]
    B = ctypes.c_void_p
    L.ps26119_backend_new.argtypes = [P(B)] + _MODEL + [P(_ScalingOptions), ctypes.c_int]
    L.ps26119_backend_free.argtypes = [B]
    L.ps26119_backend_last_error.restype = ctypes.c_char_p
    ii = [B, ctypes.c_int, ctypes.c_int]
    L.ps26119_backend_set_precision.argtypes = [B, ctypes.c_int]
    L.ps26119_backend_create.argtypes = [B, ctypes.c_int]
    L.ps26119_backend_upload.argtypes = [B, ctypes.c_int, _D]
    L.ps26119_backend_download.argtypes = [B, ctypes.c_int, _D]
    L.ps26119_backend_fill.argtypes = [B, ctypes.c_int, ctypes.c_double]
    L.ps26119_backend_copy.argtypes = ii
    L.ps26119_backend_axpby.argtypes = [B, ctypes.c_double, ctypes.c_int, ctypes.c_double, ctypes.c_int]
    L.ps26119_backend_spmv.argtypes = ii
    L.ps26119_backend_spmv_t.argtypes = ii
    L.ps26119_backend_dot.argtypes = ii + [_D]
    L.ps26119_backend_norm2.argtypes = [B, ctypes.c_int, _D]
    L.ps26119_backend_diff_norm2.argtypes = ii + [_D]
    L.ps26119_backend_primal_step.argtypes = [B, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_int]
    L.ps26119_backend_dual_step.argtypes = L.ps26119_backend_primal_step.argtypes
    step = [B, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double,
            ctypes.c_int, ctypes.c_int]
    for f in ("r2h_primal", "r2h_dual", "fused_primal", "fused_dual"):
        getattr(L, "ps26119_backend_" + f).argtypes = step
    L.ps26119_backend_kkt.argtypes = [B, ctypes.c_int, ctypes.c_int, _D]
    L.ps26119_backend_sync.argtypes = [B]
    L.ps26119_backend_scaled_get.argtypes = [B, ctypes.c_int, _D]
    L.ps26119_backend_scaled_get.restype = ctypes.c_longlong
    L.ps26119_backend_scaled_structure.argtypes = [B, ctypes.c_int, _I, _I]
    L.ps26119_backend_scaled_structure.restype = ctypes.c_longlong
    L.ps26119_backend_scalars.argtypes = [B, _D]
    L.ps26119_backend_norm2_estimate.argtypes = [B, _D]
    L.ps26119_dot_noalloc.argtypes = [ctypes.c_longlong, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                      ctypes.c_void_p, ctypes.c_void_p]
    L.ps26119_ordered_sum.argtypes = [ctypes.c_longlong, ctypes.c_void_p, ctypes.c_double, ctypes.c_int,
                                      ctypes.c_int, _D, ctypes.c_void_p]
    L.ps26119_server_create.restype = ctypes.c_void_p
    L.ps26119_server_create.argtypes = [P(_ServerOptions)]
    L.ps26119_server_submit.restype = ctypes.c_longlong
    L.ps26119_server_submit.argtypes = [ctypes.c_void_p] + _MODEL + [P(_Options), P(_Result)]
    L.ps26119_server_poll.argtypes = [ctypes.c_void_p, ctypes.c_longlong, ctypes.c_int, P(_Result), _D, _D, _D,
                                      P(_RequestTimes)]
    L.ps26119_server_destroy.argtypes = [ctypes.c_void_p]
    if path is None:
        _lib = L
    return L


def version() -> str:
    return load().ps26119_version().decode()


def ordered_sum(t_ptr: int, n: int, init: float = 0.0, order: str = "seq", exact: bool = True,
                stream: int | None = None) -> float:
    """Σ of a device vector of n doubles at address t_ptr, in the reference's order: "seq" (one
    chain init + t[0] + t[1] + …) or "chunk64" (la::parallel_sum); exact=False takes the
    engine's fast tree instead (ps26119_ordered_sum)."""
    L = load()
    out = ctypes.c_double(float("nan"))
    rc = L.ps26119_ordered_sum(int(n), ctypes.c_void_p(t_ptr), float(init), 1 if order == "chunk64" else 0,
                               int(bool(exact)), ctypes.byref(out), ctypes.c_void_p(stream) if stream else None)
    if rc != 0:
        raise RuntimeError(f"ps26119_ordered_sum: {L.ps26119_backend_last_error().decode()}")
    return out.value


@dataclass
class Result:
    status: int
    status_name: str
    objective: float
    dual_objective: float
    primal_residual: float
    dual_residual: float
    gap: float
    certified_bound: float
    iterations: int
    seconds: float
    engine: str
    message: str
    check: str = ""
    x: np.ndarray = field(repr=False, default=None)
    y: np.ndarray = field(repr=False, default=None)
    z: np.ndarray = field(repr=False, default=None)
    dual_ray: np.ndarray = field(repr=False, default=None)
    primal_ray: np.ndarray = field(repr=False, default=None)


def _lookup(table, key, what):
    if key not in table:
        raise ValueError(f"unknown {what} {key!r}; expected one of {sorted(table)}")
    return table[key]


def _csc(A, m, n):
    if isinstance(A, tuple):
        cs, ri, v = A
        return (np.ascontiguousarray(cs, dtype=np.int32), np.ascontiguousarray(ri, dtype=np.int32),
                np.ascontiguousarray(v, dtype=np.float64))
    if hasattr(A, "tocsc"):
        A = A.tocsc()
        A.sort_indices()
        return A.indptr.astype(np.int32), A.indices.astype(np.int32), A.data.astype(np.float64)
    A = np.asarray(A, dtype=np.float64)
    if A.shape != (m, n):
        raise ValueError(f"A has shape {A.shape}, expected {(m, n)}")
    r, k = np.nonzero(A.T)  # column-major order
    cs = np.zeros(n + 1, dtype=np.int32)
    np.cumsum(np.bincount(r, minlength=n), out=cs[1:])
    return cs, k.astype(np.int32), A.T[r, k].astype(np.float64)


def _ptr(a, ctype=ctypes.c_double):
    return a.ctypes.data_as(ctypes.POINTER(ctype)) if a is not None else None


def _options(algorithm, precision, gpu, tolerance, time_limit, iteration_limit, verbosity, threads):
    opt = _Options()
    load().ps26119_default_options(ctypes.byref(opt))
    opt.algorithm = _lookup(_ALG, algorithm, "algorithm")
    opt.precision = _lookup(_PREC, precision, "precision")
    opt.use_gpu = int(bool(gpu))
    opt.tolerance = tolerance
    opt.time_limit = time_limit
    opt.iteration_limit = iteration_limit
    opt.verbosity = verbosity
    opt.threads = threads
    return opt


def engine_options(presolve=True, check_every=64, exact=False, ruiz_iterations=-1, pock_chambolle=-1,
                   bound_objective_rescaling=-1, reflection=0.0, warm_primal_weight=0.0,
                   mixed_stall_checks=0) -> _EngineOptions:
    eo = _EngineOptions()
    load().ps26119_default_engine_options(ctypes.byref(eo))
    eo.presolve = int(bool(presolve))
    eo.check_every = int(check_every)
    eo.exact_reductions = int(bool(exact))
    eo.ruiz_iterations = int(ruiz_iterations)
    eo.pock_chambolle = int(pock_chambolle)
    eo.bound_objective_rescaling = int(bound_objective_rescaling)
    eo.reflection = float(reflection)
    eo.warm_primal_weight = float(warm_primal_weight)
    eo.mixed_stall_checks = int(mixed_stall_checks)
    return eo


def _result(st, res, x=None, y=None, z=None, dr=None, pr=None):
    return Result(st, _STATUS[st] if 0 <= st < len(_STATUS) else str(st), res.objective, res.dual_objective,
                  res.primal_residual, res.dual_residual, res.gap, res.certified_bound, res.iterations, res.seconds,
                  res.engine.decode(), res.message.decode(errors="replace"), _CHECK.get(res.check, ""), x, y, z, dr,
                  pr)


def solve_lp(c, A, row_lower, row_upper, col_lower=None, col_upper=None, sense=1, offset=0.0, algorithm="auto",
             precision="fp64", gpu=True, tolerance=1e-8, time_limit=3600.0, iteration_limit=0, warm_x=None,
             warm_y=None, verbosity=0, threads=1, engine=None) -> Result:
    """min (sense=+1) or max (sense=−1) cᵀx + offset  s.t. row_lower ≤ A x ≤ row_upper, bounds.

    ``engine``: None for the reference C API behaviour (ps26119_solve_lp_ex: presolve on), or a
    dict of :func:`engine_options` arguments (ps26119_solve_lp_engine)."""
    c = np.ascontiguousarray(c, dtype=np.float64)
    n = c.size
    rl = np.ascontiguousarray(row_lower, dtype=np.float64)
    ru = np.ascontiguousarray(row_upper, dtype=np.float64)
    m = rl.size
    cl = np.zeros(n) if col_lower is None else np.ascontiguousarray(col_lower, dtype=np.float64)
    cu = np.full(n, np.inf) if col_upper is None else np.ascontiguousarray(col_upper, dtype=np.float64)
    cs, ri, v = _csc(A, m, n)
    L = load()
    opt = _options(algorithm, precision, gpu, tolerance, time_limit, iteration_limit, verbosity, threads)
    wx = None if warm_x is None else np.ascontiguousarray(warm_x, dtype=np.float64)
    wy = None if warm_y is None else np.ascontiguousarray(warm_y, dtype=np.float64)
    opt.warm_x = _ptr(wx)
    opt.warm_y = _ptr(wy)
    res = _Result()
    x, y, z = np.full(n, np.nan), np.empty(m), np.empty(n)
    dr, pr = np.full(m, np.nan), np.full(n, np.nan)
    args = [m, n, int(sense), float(offset), _ptr(c), _ptr(cl), _ptr(cu), _ptr(rl), _ptr(ru),
            _ptr(cs, ctypes.c_int), _ptr(ri, ctypes.c_int), _ptr(v), ctypes.byref(opt)]
    if engine is None:
        st = L.ps26119_solve_lp_ex(*args, ctypes.byref(res), _ptr(x), _ptr(y), _ptr(z), _ptr(dr), _ptr(pr))
    else:
        eo = engine_options(**engine)
        st = L.ps26119_solve_lp_engine(*args, ctypes.byref(eo), ctypes.byref(res), _ptr(x), _ptr(y), _ptr(z),
                                       _ptr(dr), _ptr(pr))
    have = st in (OPTIMAL, ITERATION_LIMIT, TIME_LIMIT)
    ray_d = dr if st == INFEASIBLE and m > 0 and not np.isnan(dr).any() else None
    ray_p = pr if st == UNBOUNDED and n > 0 and not np.isnan(pr).any() else None
    return _result(st, res, x if have or ray_p is not None else None, y if have else None, z if have else None,
                   ray_d, ray_p)


class Server:
    """The request loop (ps26119_server_*): independent LPs admitted by slots and HBM budget,
    solved concurrently on the GPU, each exactly as :func:`solve_lp` would solve it.

    >>> with Server(slots=8) as srv:
    ...     rid = srv.submit(lp)          # an object with the generators.Lp fields
    ...     res, times = srv.result(rid)  # waits; times = (submitted, started, finished) seconds
    """

    def __init__(self, slots=8, hbm_budget_bytes=0.0, dry_run_seconds=0.0, grouped=True):
        self.L = load()
        o = _ServerOptions(int(slots), float(hbm_budget_bytes), float(dry_run_seconds), 0 if grouped else 1)
        self.h = self.L.ps26119_server_create(ctypes.byref(o))
        if not self.h:
            raise ValueError("ps26119_server_create refused the options")
        self.shapes = {}

    def submit(self, lp, algorithm="r2hpdhg", precision="fp64", tolerance=1e-8, time_limit=3600.0,
               iteration_limit=0) -> int:
        args, keep = _model_args(lp)
        opt = _options(algorithm, precision, True, tolerance, time_limit, iteration_limit, 0, 1)
        err = _Result()
        rid = self.L.ps26119_server_submit(self.h, *args, ctypes.byref(opt), ctypes.byref(err))
        del keep
        if rid < 0:
            raise ValueError(err.message.decode(errors="replace"))
        self.shapes[rid] = (lp.num_rows, lp.num_cols)
        return rid

    def poll(self, rid, wait=False):
        """(Result, (submitted, started, finished)) once request ``rid`` has finished, else None."""
        m, n = self.shapes[rid]
        res, t = _Result(), _RequestTimes()
        x, y, z = np.full(n, np.nan), np.full(m, np.nan), np.full(n, np.nan)
        r = self.L.ps26119_server_poll(self.h, rid, int(bool(wait)), ctypes.byref(res), _ptr(x), _ptr(y), _ptr(z),
                                       ctypes.byref(t))
        if r == 0:
            return None
        if r < 0:
            raise KeyError(rid)
        del self.shapes[rid]
        have = res.status in (OPTIMAL, ITERATION_LIMIT, TIME_LIMIT)
        return (_result(res.status, res, x if have else None, y if have else None, z if have else None),
                (t.submitted, t.started, t.finished))

    def result(self, rid):
        return self.poll(rid, wait=True)

    def close(self):
        if self.h:
            self.L.ps26119_server_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def solve_lp_device(m, n, sense, offset, ptrs, precision="fp64", tolerance=1e-8, time_limit=3600.0,
                    iteration_limit=0, engine=None, out=(None, None, None), stream=None, verbosity=0) -> Result:
    """Device-resident solve: ``ptrs`` = device addresses (ints) of c, col_lower, col_upper,
    row_lower, row_upper, col_start, row_index, value; ``out`` = device addresses of x, y, z
    (or None); ``stream`` = a cudaStream_t address (or None)."""
    L = load()
    opt = _options("r2hpdhg", precision, True, tolerance, time_limit, iteration_limit, verbosity, 1)
    eo = engine_options(**(engine or {}))
    res = _Result()
    st = L.ps26119_solve_lp_device(int(m), int(n), int(sense), float(offset), *[ctypes.c_void_p(p) for p in ptrs],
                                   ctypes.byref(opt), ctypes.byref(eo), ctypes.byref(res),
                                   *[ctypes.c_void_p(p) if p else None for p in out],
                                   ctypes.c_void_p(stream) if stream else None)
    return _result(st, res)


def solve_batch(c, A, row_lower, row_upper, col_lower=None, col_upper=None, scenarios=(), sense=1, offset=0.0,
                tolerance=1e-8, time_limit=3600.0, iteration_limit=0, engine=None, verbosity=0,
                precision="fp64") -> list[Result]:
    """ps26119::solve_batch on the GPU: the base LP (as :func:`solve_lp`) and a list of scenarios,
    each a dict with any of obj, col_lower, col_upper, row_lower, row_upper (missing = the
    base's). Returns one :class:`Result` per scenario (x, y, z set when the scenario has a point)."""
    c = np.ascontiguousarray(c, dtype=np.float64)
    n = c.size
    rl = np.ascontiguousarray(row_lower, dtype=np.float64)
    ru = np.ascontiguousarray(row_upper, dtype=np.float64)
    m = rl.size
    cl = np.zeros(n) if col_lower is None else np.ascontiguousarray(col_lower, dtype=np.float64)
    cu = np.full(n, np.inf) if col_upper is None else np.ascontiguousarray(col_upper, dtype=np.float64)
    cs, ri, v = _csc(A, m, n)
    # A C pointer carries no length: a scenario vector of the wrong size is rejected here, alone,
    # as the reference's solve_batch rejects it (batch.cpp:154-177); the others still run.
    sizes = {"obj": n, "col_lower": n, "col_upper": n, "row_lower": m, "row_upper": m}
    bad = [any(s.get(key) is not None and np.size(s[key]) != ln for key, ln in sizes.items()) for s in scenarios]
    run = [k for k in range(len(scenarios)) if not bad[k]]
    K = len(run)
    keep = []
    sc = (_Scenario * max(1, K))()
    for t, k in enumerate(run):
        for key in sizes:
            if scenarios[k].get(key) is not None:
                a = np.ascontiguousarray(scenarios[k][key], dtype=np.float64)
                keep.append(a)
                setattr(sc[t], key, _ptr(a))
    opt = _options("r2hpdhg", precision, True, tolerance, time_limit, iteration_limit, verbosity, 1)
    eo = engine_options(**(engine or {}))
    res = (_Result * max(1, K))()
    x, y, z = np.full((K, n), np.nan), np.full((K, m), np.nan), np.full((K, n), np.nan)
    L = load()
    L.ps26119_solve_batch(m, n, int(sense), float(offset), _ptr(c), _ptr(cl), _ptr(cu), _ptr(rl), _ptr(ru),
                          _ptr(cs, ctypes.c_int), _ptr(ri, ctypes.c_int), _ptr(v), K, sc, ctypes.byref(opt),
                          ctypes.byref(eo), res, _ptr(x), _ptr(y), _ptr(z))
    out = [None] * len(scenarios)
    for t, k in enumerate(run):
        st = res[t].status
        have = st in (OPTIMAL, ITERATION_LIMIT, TIME_LIMIT)
        out[k] = _result(st, res[t], x[t] if have else None, y[t] if have else None, z[t] if have else None)
    for k in range(len(scenarios)):
        if bad[k]:
            out[k] = Result(NOT_SOLVED, _STATUS[NOT_SOLVED], np.nan, np.nan, np.nan, np.nan, np.nan, np.nan, 0, 0.0,
                            "r2hpdhg-batch", "scenario has wrong vector sizes or non-finite data")
    return out


def _model_args(lp):
    f = lambda a: np.ascontiguousarray(a, dtype=np.float64)
    g = lambda a: np.ascontiguousarray(a, dtype=np.int32)
    arrs = [f(lp.c), f(lp.col_lower), f(lp.col_upper), f(lp.row_lower), f(lp.row_upper), g(lp.col_start),
            g(lp.row_index), f(lp.value)]
    args = [lp.num_rows, lp.num_cols, int(lp.sense), float(lp.offset)] + \
        [_ptr(a) for a in arrs[:5]] + [_ptr(arrs[5], ctypes.c_int), _ptr(arrs[6], ctypes.c_int), _ptr(arrs[7])]
    return args, arrs


def certified_bound(lp, y, use_implied_bounds=True) -> dict:
    """Rounding-error-proof bound on the optimum of ``lp`` (an object with the generators.Lp
    fields) from row multipliers ``y`` (host computation)."""
    args, keep = _model_args(lp)
    yy = np.ascontiguousarray(y, dtype=np.float64)
    out = np.zeros(4)
    rc = load().ps26119_certified_bound(*args, _ptr(yy), int(bool(use_implied_bounds)), _ptr(out))
    if rc != 0:
        raise ValueError(f"ps26119_certified_bound failed ({rc})")
    return {"finite": bool(out[0]), "bound": out[1], "unbounded_row_terms": int(out[2]),
            "unbounded_col_terms": int(out[3])}


def check_certificate(lp, ray, x=None) -> dict:
    """Farkas (x None: ray has num_rows values) or unboundedness (x and ray: num_cols values) check."""
    args, keep = _model_args(lp)
    r = np.ascontiguousarray(ray, dtype=np.float64)
    xx = None if x is None else np.ascontiguousarray(x, dtype=np.float64)
    out = np.zeros(5)
    rc = load().ps26119_check_certificate(0 if x is None else 1, *args, _ptr(xx), _ptr(r), _ptr(out))
    if rc != 0:
        raise ValueError(f"ps26119_check_certificate failed ({rc})")
    return {"present": bool(out[0]), "passed": bool(out[1]), "rigorous": bool(out[2]), "measure": out[3],
            "violation": out[4]}


def solve_mps(path, algorithm="auto", precision="fp64", gpu=True, tolerance=1e-8, time_limit=3600.0,
              iteration_limit=0, verbosity=0, threads=1, out=None) -> Result:
    opt = _options(algorithm, precision, gpu, tolerance, time_limit, iteration_limit, verbosity, threads)
    res = _Result()
    st = load().ps26119_solve_mps(os.fsencode(path) if path is not None else None, ctypes.byref(opt),
                                  ctypes.byref(res), None if out is None else os.fsencode(out))
    return _result(st, res)


def last_stats() -> dict:
    s = _Stats()
    load().ps26119_last_stats(ctypes.byref(s))
    return {k: getattr(s, k) for k, _ in _Stats._fields_}


class Backend:
    """The pdhg::Backend operations on the GPU (include/ps26119_backend.h)."""

    def __init__(self, lp, exact=False, ruiz_iterations=10, pock_chambolle=True, bound_objective_rescaling=True,
                 geometric_mean_iterations=12, geometric_mean_min_log10_range=4.5):
        self.L = load()
        f = lambda a: np.ascontiguousarray(a, dtype=np.float64)
        g = lambda a: np.ascontiguousarray(a, dtype=np.int32)
        a = [f(lp.c), f(lp.col_lower), f(lp.col_upper), f(lp.row_lower), f(lp.row_upper), g(lp.col_start),
             g(lp.row_index), f(lp.value)]
        so = _ScalingOptions(geometric_mean_iterations, geometric_mean_min_log10_range, ruiz_iterations,
                             int(pock_chambolle), int(bound_objective_rescaling))
        self.h = ctypes.c_void_p()
        rc = self.L.ps26119_backend_new(ctypes.byref(self.h), lp.num_rows, lp.num_cols, lp.sense, lp.offset,
                                        _ptr(a[0]), _ptr(a[1]), _ptr(a[2]), _ptr(a[3]), _ptr(a[4]),
                                        _ptr(a[5], ctypes.c_int), _ptr(a[6], ctypes.c_int), _ptr(a[7]),
                                        ctypes.byref(so), int(bool(exact)))
        if rc != 0:
            raise RuntimeError(f"ps26119_backend_new failed ({rc}): {self.L.ps26119_backend_last_error().decode()}")
        self.m, self.n = lp.num_rows, lp.num_cols
        self.sizes = []

    def __del__(self):
        if getattr(self, "h", None):
            self.L.ps26119_backend_free(self.h)
            self.h = None

    def _ok(self, rc):
        if rc != 0:
            raise RuntimeError(f"backend op failed ({rc}): {self.L.ps26119_backend_last_error().decode()}")

    def set_precision(self, mixed):
        self._ok(self.L.ps26119_backend_set_precision(self.h, int(bool(mixed))))

    def create(self, dual):
        v = self.L.ps26119_backend_create(self.h, int(bool(dual)))
        if v < 0:
            raise RuntimeError(self.L.ps26119_backend_last_error().decode())
        self.sizes.append(self.m if dual else self.n)
        return v

    def upload(self, v, a):
        a = np.ascontiguousarray(a, dtype=np.float64)
        self._ok(self.L.ps26119_backend_upload(self.h, v, _ptr(a)))

    def download(self, v):
        out = np.empty(self.sizes[v])
        self._ok(self.L.ps26119_backend_download(self.h, v, _ptr(out)))
        return out

    def _scalar(self, fn, *a):
        out = ctypes.c_double()
        self._ok(fn(self.h, *a, ctypes.byref(out)))
        return out.value

    def dot(self, a, b):
        return self._scalar(self.L.ps26119_backend_dot, a, b)

    def norm2(self, a):
        return self._scalar(self.L.ps26119_backend_norm2, a)

    def diff_norm2(self, a, b):
        return self._scalar(self.L.ps26119_backend_diff_norm2, a, b)

    def norm2_estimate(self):
        return self._scalar(self.L.ps26119_backend_norm2_estimate)

    def kkt(self, xs, ys):
        out = np.zeros(8)
        self._ok(self.L.ps26119_backend_kkt(self.h, xs, ys, _ptr(out)))
        return dict(zip(["primal_residual", "dual_residual", "primal_obj", "dual_obj", "b_norm", "c_norm",
                         "primal_max_rel", "dual_max_rel"], out))

    def scaled(self, which):
        cnt = self.L.ps26119_backend_scaled_get(self.h, which, None)
        out = np.empty(cnt)
        self.L.ps26119_backend_scaled_get(self.h, which, _ptr(out))
        return out

    def structure(self, which):
        rows = self.m if which == 0 else self.n
        nnz = self.L.ps26119_backend_scaled_structure(self.h, which, None, None)
        rp, col = np.empty(rows + 1, dtype=np.int32), np.empty(nnz, dtype=np.int32)
        self.L.ps26119_backend_scaled_structure(self.h, which, _ptr(rp, ctypes.c_int), _ptr(col, ctypes.c_int))
        return rp, col

    def scalars(self):
        out = np.zeros(4)
        self._ok(self.L.ps26119_backend_scalars(self.h, _ptr(out)))
        return {"bound_scale": out[0], "obj_scale": out[1], "log10_range": out[2],
                "geometric_mean_applied": bool(out[3])}

    def __getattr__(self, name):
        fn = getattr(self.L, "ps26119_backend_" + name)
        return lambda *a: self._ok(fn(self.h, *a))
