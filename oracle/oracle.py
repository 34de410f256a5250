"""ctypes access to the C restatement of the reference r²HPDHG path (oracle/pdhg_oracle.c).

TEST ORACLE: only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it,
and only as the checker. Built by ``make -C oracle oracle`` (also run by
__graft_entry__.build()).
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
STATUS = ["Optimal", "Infeasible", "Unbounded", "IterationLimit", "TimeLimit", "NumericalError", "NotSolved"]

_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int)


class Model(ctypes.Structure):
    _fields_ = [("m", ctypes.c_int), ("n", ctypes.c_int), ("sense", ctypes.c_int), ("offset", ctypes.c_double),
                ("c", _D), ("col_lower", _D), ("col_upper", _D), ("row_lower", _D), ("row_upper", _D),
                ("col_start", _I), ("row_index", _I), ("value", _D)]


class ScalingOptions(ctypes.Structure):
    _fields_ = [("ruiz_iterations", ctypes.c_int), ("pock_chambolle", ctypes.c_int),
                ("bound_objective_rescaling", ctypes.c_int), ("geometric_mean_iterations", ctypes.c_int),
                ("geometric_mean_min_log10_range", ctypes.c_double)]


class Options(ctypes.Structure):
    _fields_ = [("tolerance", ctypes.c_double), ("iteration_limit", ctypes.c_longlong),
                ("check_every", ctypes.c_int), ("mixed", ctypes.c_int), ("scaling", ScalingOptions),
                ("reflection", ctypes.c_double), ("restart_sufficient", ctypes.c_double),
                ("restart_necessary", ctypes.c_double), ("restart_artificial", ctypes.c_double),
                ("pid_kp", ctypes.c_double), ("pid_ki", ctypes.c_double), ("pid_kd", ctypes.c_double),
                ("pid_integral_decay", ctypes.c_double), ("pid_max_log_step", ctypes.c_double),
                ("warm_x", _D), ("warm_y", _D), ("warm_primal_weight", ctypes.c_double)]


class Result(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int), ("iterations", ctypes.c_longlong), ("objective", ctypes.c_double),
                ("dual_objective", ctypes.c_double), ("primal_residual", ctypes.c_double),
                ("dual_residual", ctypes.c_double), ("gap", ctypes.c_double), ("primal_weight", ctypes.c_double),
                ("eta", ctypes.c_double), ("initial_primal_weight", ctypes.c_double),
                ("iterations_to_fast", ctypes.c_longlong), ("switch_iteration", ctypes.c_longlong),
                ("restarts", ctypes.c_longlong), ("checks", ctypes.c_longlong), ("message", ctypes.c_char * 256)]


_lib = None


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise FileNotFoundError(f"{LIB_PATH} not built (make -C oracle oracle)")
        L = ctypes.CDLL(LIB_PATH)
        L.orc_default_options.argtypes = [ctypes.POINTER(Options)]
        L.orc_solve_r2hpdhg.argtypes = [ctypes.POINTER(Model), ctypes.POINTER(Options), ctypes.POINTER(Result), _D, _D,
                                        _D, _D, _D]
        L.orc_solve_r2hpdhg.restype = ctypes.c_int
        L.orc_scale.argtypes = [ctypes.POINTER(Model), ctypes.POINTER(ScalingOptions)]
        L.orc_scale.restype = ctypes.c_void_p
        L.orc_scaled_free.argtypes = [ctypes.c_void_p]
        L.orc_scaled_get.argtypes = [ctypes.c_void_p, ctypes.c_int, _D]
        L.orc_scaled_get.restype = ctypes.c_longlong
        L.orc_scaled_scalars.argtypes = [ctypes.c_void_p, _D]
        L.orc_norm2.argtypes = [ctypes.c_void_p]
        L.orc_norm2.restype = ctypes.c_double
        L.orc_backend_new.argtypes = [ctypes.c_void_p]
        L.orc_backend_new.restype = ctypes.c_void_p
        L.orc_backend_free.argtypes = [ctypes.c_void_p]
        L.orc_backend_set_precision.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.orc_backend_create.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.orc_backend_create.restype = ctypes.c_int
        L.orc_backend_upload.argtypes = [ctypes.c_void_p, ctypes.c_int, _D]
        L.orc_backend_download.argtypes = [ctypes.c_void_p, ctypes.c_int, _D]
        L.orc_backend_fill.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double]
        L.orc_backend_copy.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
        L.orc_backend_axpby.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_int, ctypes.c_double,
                                        ctypes.c_int]
        L.orc_backend_spmv.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
        L.orc_backend_spmv_t.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
        for f in ("orc_backend_dot", "orc_backend_diff_norm2"):
            getattr(L, f).argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
            getattr(L, f).restype = ctypes.c_double
        L.orc_backend_norm2.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.orc_backend_norm2.restype = ctypes.c_double
        L.orc_backend_primal_step.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                              ctypes.c_int]
        L.orc_backend_dual_step.argtypes = L.orc_backend_primal_step.argtypes
        L.orc_backend_r2h_primal.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                             ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                             ctypes.c_int]
        L.orc_backend_r2h_dual.argtypes = L.orc_backend_r2h_primal.argtypes
        L.orc_backend_kkt.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _D]
        _lib = L
    return _lib


class _ModelRef:
    """Keeps numpy copies alive for the lifetime of the ctypes Model."""

    def __init__(self, lp):
        f = lambda a: np.ascontiguousarray(a, dtype=np.float64)
        g = lambda a: np.ascontiguousarray(a, dtype=np.int32)
        self.arrays = [f(lp.c), f(lp.col_lower), f(lp.col_upper), f(lp.row_lower), f(lp.row_upper),
                       g(lp.col_start), g(lp.row_index), f(lp.value)]
        a = self.arrays
        d = lambda x: x.ctypes.data_as(_D)
        i = lambda x: x.ctypes.data_as(_I)
        self.model = Model(lp.num_rows, lp.num_cols, lp.sense, lp.offset, d(a[0]), d(a[1]), d(a[2]), d(a[3]),
                           d(a[4]), i(a[5]), i(a[6]), d(a[7]))


@dataclass
class OracleSolution:
    status: str
    iterations: int
    objective: float
    dual_objective: float
    primal_residual: float
    dual_residual: float
    gap: float
    primal_weight: float
    eta: float
    iterations_to_fast: int
    switch_iteration: int
    restarts: int
    checks: int
    message: str
    x: np.ndarray
    y: np.ndarray
    z: np.ndarray


def default_options() -> Options:
    o = Options()
    lib().orc_default_options(ctypes.byref(o))
    return o


def solve(lp, precision="fp64", tol=0.0, iteration_limit=0, check_every=0, params=None, warm_x=None,
          warm_y=None) -> OracleSolution:
    L = lib()
    mr = _ModelRef(lp)
    o = default_options()
    o.mixed = 1 if precision == "mixed" else 0
    if tol > 0:
        o.tolerance = tol
    if iteration_limit > 0:
        o.iteration_limit = iteration_limit
    if check_every > 0:
        o.check_every = check_every
    for k, v in (params or {}).items():
        if hasattr(o.scaling, k) and k in dict(ScalingOptions._fields_):
            setattr(o.scaling, k, type(getattr(o.scaling, k))(v))
        else:
            setattr(o, k, v)
    keep = []
    if warm_x is not None:
        keep.append(np.ascontiguousarray(warm_x, dtype=np.float64))
        o.warm_x = keep[-1].ctypes.data_as(_D)
    if warm_y is not None:
        keep.append(np.ascontiguousarray(warm_y, dtype=np.float64))
        o.warm_y = keep[-1].ctypes.data_as(_D)
    m, n = lp.num_rows, lp.num_cols
    x, y, z = np.full(n, np.nan), np.full(m, np.nan), np.full(n, np.nan)
    r = Result()
    L.orc_solve_r2hpdhg(ctypes.byref(mr.model), ctypes.byref(o), ctypes.byref(r), x.ctypes.data_as(_D),
                        y.ctypes.data_as(_D), z.ctypes.data_as(_D), None, None)
    return OracleSolution(STATUS[r.status], r.iterations, r.objective, r.dual_objective, r.primal_residual,
                          r.dual_residual, r.gap, r.primal_weight, r.eta, r.iterations_to_fast, r.switch_iteration,
                          r.restarts, r.checks, r.message.decode(errors="replace"), x, y, z)


class Scaled:
    """make_scaled_problem restated (scaling.cpp:37-142) plus the ‖Ã‖₂ estimate."""

    def __init__(self, lp, ruiz_iterations=10, pock_chambolle=True, bound_objective_rescaling=True,
                 geometric_mean_iterations=12, geometric_mean_min_log10_range=4.5):
        self.L = lib()
        self._mr = _ModelRef(lp)
        so = ScalingOptions(ruiz_iterations, int(pock_chambolle), int(bound_objective_rescaling),
                            geometric_mean_iterations, geometric_mean_min_log10_range)
        self.h = self.L.orc_scale(ctypes.byref(self._mr.model), ctypes.byref(so))

    def __del__(self):
        if getattr(self, "h", None):
            self.L.orc_scaled_free(self.h)
            self.h = None

    def get(self, which: int) -> np.ndarray:
        cnt = self.L.orc_scaled_get(self.h, which, None)
        out = np.empty(cnt)
        self.L.orc_scaled_get(self.h, which, out.ctypes.data_as(_D))
        return out

    def scalars(self):
        out = np.zeros(4)
        self.L.orc_scaled_scalars(self.h, out.ctypes.data_as(_D))
        return {"bound_scale": out[0], "obj_scale": out[1], "log10_range": out[2],
                "geometric_mean_applied": bool(out[3])}

    def norm2(self) -> float:
        return self.L.orc_norm2(self.h)


class Backend:
    """The reference CpuBackend restated (cpu_backend.cpp:31-215) over a Scaled problem."""

    def __init__(self, scaled: Scaled):
        self.L = lib()
        self.scaled = scaled
        self.h = self.L.orc_backend_new(scaled.h)
        self.sizes = []
        self.m = scaled._mr.model.m
        self.n = scaled._mr.model.n

    def __del__(self):
        if getattr(self, "h", None):
            self.L.orc_backend_free(self.h)
            self.h = None

    def set_precision(self, mixed: bool):
        self.L.orc_backend_set_precision(self.h, int(mixed))

    def create(self, dual: bool) -> int:
        self.sizes.append(self.m if dual else self.n)
        return self.L.orc_backend_create(self.h, int(dual))

    def upload(self, v, a):
        a = np.ascontiguousarray(a, dtype=np.float64)
        self.L.orc_backend_upload(self.h, v, a.ctypes.data_as(_D))

    def download(self, v):
        out = np.empty(self.sizes[v])
        self.L.orc_backend_download(self.h, v, out.ctypes.data_as(_D))
        return out

    def __getattr__(self, name):
        f = getattr(self.L, "orc_backend_" + name)
        return lambda *a: f(self.h, *a)

    def kkt(self, xs, ys):
        out = np.zeros(8)
        self.L.orc_backend_kkt(self.h, xs, ys, out.ctypes.data_as(_D))
        return dict(zip(["primal_residual", "dual_residual", "primal_obj", "dual_obj", "b_norm", "c_norm",
                         "primal_max_rel", "dual_max_rel"], out))
