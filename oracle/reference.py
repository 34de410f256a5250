"""ctypes access to the REFERENCE solver built from its own sources (oracle/_ref).

Test infrastructure only: the checker in tests/, the CPU baseline in bench.py. The library
is built by ``make -C oracle ref`` (see oracle/Makefile) where the reference sources are
present; the built ``.so`` travels with the repository snapshot, so this module works on a
machine without the reference sources as long as the library was built beforehand.

Functions mirror the shim in oracle/ref_shim.cpp, which drives:
  ps26119::solve (reference src/core/solve.cpp:194), solve_batch (src/pdhg/batch.cpp:129),
  make_scaled_problem (src/pdhg/scaling.cpp:37), estimate_norm2 (src/la/csr.cpp:86),
  the CpuBackend ops (src/pdhg/cpu_backend.cpp:31-215), check_solution
  (src/core/solution_checker.cpp:61) and certified_dual_bound (src/core/safe_bound.cpp:178).
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libps26119_ref.so")
# the same reference built with its own CUDA backend (src/gpu/cuda_backend.cu, sm_100a)
LIB_GPU_PATH = os.path.join(HERE, "_ref", "libps26119_refgpu.so")

STATUS = ["Optimal", "Infeasible", "Unbounded", "IterationLimit", "TimeLimit", "NumericalError", "NotSolved"]
INFO = ["status", "objective", "dual_objective", "primal_residual", "dual_residual", "gap", "iterations", "seconds",
        "setup_seconds", "primal_weight", "certified_bound", "check", "iterations_to_fast"]

_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int)
_libs = {}


def available() -> bool:
    return os.path.exists(LIB_PATH)


def available_gpu() -> bool:
    return os.path.exists(LIB_GPU_PATH)


def lib(gpu: bool = False):
    key = bool(gpu)
    if key not in _libs:
        path = LIB_GPU_PATH if gpu else LIB_PATH
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} not built (make -C oracle {'ref_gpu' if gpu else 'ref'})")
        L = ctypes.CDLL(path)
        model = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double, _D, _D, _D, _D, _D, _I, _I, _D]
        L.ref_solve.argtypes = model + [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                        ctypes.c_longlong, ctypes.c_double, ctypes.c_int, ctypes.c_int,
                                        ctypes.POINTER(ctypes.c_char_p), _D, _D, _D, _D, _D, _D, _D, _D, _D,
                                        ctypes.c_char_p, ctypes.c_int]
        L.ref_solve.restype = ctypes.c_int
        L.ref_batch.argtypes = model + [ctypes.c_int, _D, _D, _D, _D, _D, ctypes.c_int, ctypes.c_double,
                                        ctypes.c_longlong, _D, _D, _D]
        L.ref_batch.restype = ctypes.c_int
        L.ref_backend_new.argtypes = model + [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                              ctypes.c_double]
        L.ref_backend_new.restype = ctypes.c_void_p
        L.ref_backend_free.argtypes = [ctypes.c_void_p]
        L.ref_scaled_get.argtypes = [ctypes.c_void_p, ctypes.c_int, _D]
        L.ref_scaled_get.restype = ctypes.c_longlong
        L.ref_scaled_structure.argtypes = [ctypes.c_void_p, ctypes.c_int, _I, _I]
        L.ref_scaled_structure.restype = ctypes.c_longlong
        L.ref_scaled_scalars.argtypes = [ctypes.c_void_p, _D]
        L.ref_norm2.argtypes = [ctypes.c_void_p]
        L.ref_norm2.restype = ctypes.c_double
        L.ref_backend_set_precision.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.ref_backend_create.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.ref_backend_create.restype = ctypes.c_int
        L.ref_backend_upload.argtypes = [ctypes.c_void_p, ctypes.c_int, _D, ctypes.c_longlong]
        L.ref_backend_download.argtypes = [ctypes.c_void_p, ctypes.c_int, _D, ctypes.c_longlong]
        L.ref_backend_fill.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double]
        L.ref_backend_copy.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
        L.ref_backend_axpby.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_int, ctypes.c_double,
                                        ctypes.c_int]
        L.ref_backend_spmv.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
        L.ref_backend_spmv_t.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
        for f in ("ref_backend_dot", "ref_backend_diff_norm2"):
            getattr(L, f).argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
            getattr(L, f).restype = ctypes.c_double
        L.ref_backend_norm2.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.ref_backend_norm2.restype = ctypes.c_double
        L.ref_backend_primal_step.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                              ctypes.c_int]
        L.ref_backend_dual_step.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                            ctypes.c_int]
        L.ref_backend_r2h_primal.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                             ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                             ctypes.c_int]
        L.ref_backend_r2h_dual.argtypes = L.ref_backend_r2h_primal.argtypes
        L.ref_backend_kkt.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _D]
        L.ref_check.argtypes = model + [_D, _D, _D]
        L.ref_bound.argtypes = model + [_D, ctypes.c_int, _D]
        L.ref_read_fingerprint.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int,
                                           ctypes.POINTER(ctypes.c_longlong)]
        L.ref_presolve_file.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int,
                                        ctypes.POINTER(ctypes.c_longlong)]
        L.ref_check_file.argtypes = [ctypes.c_char_p, _D, _D, _D]
        L.ref_kkt_file.argtypes = [ctypes.c_char_p, _D, _D, ctypes.c_double, _D]
        L.ref_postsolve_file.argtypes = [ctypes.c_char_p, _D, ctypes.c_longlong, _D, ctypes.c_longlong, _D, _D, _D,
                                         _D, ctypes.POINTER(ctypes.c_longlong)]
        L.ref_certificate.argtypes = [ctypes.c_int] + model + [_D, _D, _D]
        L.ps26119_solve_lp.argtypes = None  # the reference's own C API, used by bench.py
        _libs[key] = L
    return _libs[key]


def _d(a):
    return a.ctypes.data_as(_D) if a is not None else None


def _i(a):
    return a.ctypes.data_as(_I)


def _model_args(lp):
    f = lambda a: np.ascontiguousarray(a, dtype=np.float64)
    g = lambda a: np.ascontiguousarray(a, dtype=np.int32)
    keep = [f(lp.c), f(lp.col_lower), f(lp.col_upper), f(lp.row_lower), f(lp.row_upper), g(lp.col_start),
            g(lp.row_index), f(lp.value)]
    args = [lp.num_rows, lp.num_cols, lp.sense, lp.offset, _d(keep[0]), _d(keep[1]), _d(keep[2]), _d(keep[3]),
            _d(keep[4]), _i(keep[5]), _i(keep[6]), _d(keep[7])]
    return args, keep


@dataclass
class RefSolution:
    status: str
    objective: float
    dual_objective: float
    primal_residual: float
    dual_residual: float
    gap: float
    iterations: int
    seconds: float
    setup_seconds: float
    primal_weight: float
    certified_bound: float
    check: int
    iterations_to_fast: int
    x: np.ndarray
    y: np.ndarray
    z: np.ndarray
    dual_ray: np.ndarray
    primal_ray: np.ndarray
    message: str


def solve(lp, presolve=False, precision="fp64", threads=1, tol=0.0, iteration_limit=0, time_limit=0.0,
          check_every=0, params=None, warm_x=None, warm_y=None, algorithm="r2hpdhg", gpu=False) -> RefSolution:
    """ps26119::solve with algorithm r2hpdhg (or pdlp) on the CPU (reference src/core/solve.cpp:194);
    gpu=True: the reference's own CUDA backend (Options::use_gpu, its library built with
    src/gpu/cuda_backend.cu)."""
    L = lib(gpu)
    args, keep = _model_args(lp)
    m, n = lp.num_rows, lp.num_cols
    params = list((params or {}).items())
    if algorithm == "pdlp":
        params.append(("algorithm", 2.0))
    if gpu:
        params.append(("use_gpu", 1.0))
    names = (ctypes.c_char_p * max(1, len(params)))(*[k.encode() for k, _ in params])
    vals = np.array([v for _, v in params] or [0.0], dtype=np.float64)
    wx = None if warm_x is None else np.ascontiguousarray(warm_x, dtype=np.float64)
    wy = None if warm_y is None else np.ascontiguousarray(warm_y, dtype=np.float64)
    x, y, z = np.full(n, np.nan), np.full(m, np.nan), np.full(n, np.nan)
    dr, pr = np.full(m, np.nan), np.full(n, np.nan)
    info = np.zeros(len(INFO))
    msg = ctypes.create_string_buffer(512)
    L.ref_solve(*args, int(presolve), 1 if precision == "mixed" else 0, int(threads), float(tol),
                int(iteration_limit), float(time_limit), int(check_every), len(params), names, _d(vals), _d(wx),
                _d(wy), _d(x), _d(y), _d(z), _d(dr), _d(pr), _d(info), msg, 512)
    del keep
    i = dict(zip(INFO, info))
    return RefSolution(STATUS[int(i["status"])], i["objective"], i["dual_objective"], i["primal_residual"],
                       i["dual_residual"], i["gap"], int(i["iterations"]), i["seconds"], i["setup_seconds"],
                       i["primal_weight"], i["certified_bound"], int(i["check"]), int(i["iterations_to_fast"]), x, y,
                       z, dr, pr, msg.value.decode(errors="replace"))


def batch(lp, scen, threads=1, tol=0.0, iteration_limit=0):
    """solve_batch (reference src/pdhg/batch.cpp:129); scen = list of dicts (generators.scenarios)."""
    L = lib()
    args, keep = _model_args(lp)
    K, m, n = len(scen), lp.num_rows, lp.num_cols

    def stack(key, length):
        if not any(key in s for s in scen):
            return None
        return np.ascontiguousarray(np.stack([s.get(key, None) if s.get(key) is not None else
                                              getattr(lp, {"obj": "c"}.get(key, key)) for s in scen]),
                                    dtype=np.float64)
    arrs = [stack("obj", n), stack("col_lower", n), stack("col_upper", n), stack("row_lower", m),
            stack("row_upper", m)]
    x, y, info = np.full((K, n), np.nan), np.full((K, m), np.nan), np.zeros((K, len(INFO)))
    L.ref_batch(*args, K, *[_d(a) for a in arrs], int(threads), float(tol), int(iteration_limit), _d(x), _d(y),
                _d(info))
    del keep
    out = []
    for k in range(K):
        i = dict(zip(INFO, info[k]))
        out.append({"status": STATUS[int(i["status"])], "objective": i["objective"],
                    "iterations": int(i["iterations"]), "x": x[k], "y": y[k], **{kk: i[kk] for kk in INFO[3:6]}})
    return out


def check(lp, x, y):
    """check_solution + certified_dual_bound on the original model."""
    L = lib()
    args, keep = _model_args(lp)
    out = np.zeros(7)
    L.ref_check(*args, _d(np.ascontiguousarray(x, dtype=np.float64)),
                _d(np.ascontiguousarray(y, dtype=np.float64)), _d(out))
    del keep
    return {"passed": bool(out[0]), "primal": out[1], "dual": out[2], "gap": out[3], "primal_objective": out[4],
            "dual_objective": out[5], "certified_bound": out[6]}


def check_file(path, x, y):
    """check() on the model read from a file by the reference's readers: the 7 values
    (passed, primal, dual, gap, primal objective, dual objective, certified bound) as an array,
    or None when the file does not read."""
    L = lib()
    out = np.zeros(7)
    ok = L.ref_check_file(os.fsencode(path), _d(np.ascontiguousarray(x, dtype=np.float64)),
                          _d(np.ascontiguousarray(y, dtype=np.float64)), _d(out))
    return out if ok else None


def kkt_file(path, x, y, eps):
    """original_kkt (reference src/core/solve.cpp:77-84) of (x, y) on the model read from a
    file: the 8 KktStats values and converged(eps) as an array of 9, or None when the file does
    not read."""
    L = lib()
    out = np.zeros(9)
    ok = L.ref_kkt_file(os.fsencode(path), _d(np.ascontiguousarray(x, dtype=np.float64)),
                        _d(np.ascontiguousarray(y, dtype=np.float64)), float(eps), _d(out))
    return out if ok else None


def read_fingerprint(path):
    """The reference reader's view of a model file: (fingerprint hex, (rows, cols, nnz)) or
    (None, error text)."""
    L = lib()
    buf = ctypes.create_string_buffer(512)
    dims = (ctypes.c_longlong * 3)()
    ok = L.ref_read_fingerprint(os.fsencode(path), buf, 512, dims)
    return (buf.value.decode(), tuple(dims)) if ok else (None, buf.value.decode())


def presolve_file(path):
    """The reference reader and ps26119::presolve on a model file: (digest hex, (outcome,
    removed rows, removed cols, tightened bounds)) with outcome 0 reduced, 1 infeasible,
    2 unchanged; or (None, error text)."""
    L = lib()
    buf = ctypes.create_string_buffer(512)
    counts = (ctypes.c_longlong * 4)()
    ok = L.ref_presolve_file(os.fsencode(path), buf, 512, counts)
    return (buf.value.decode(), tuple(counts)) if ok else (None, buf.value.decode())


def postsolve_file(path, num_rows, num_cols, red_x, red_y):
    """The reference reader, presolve and postsolve (reference src/core/presolve.cpp:158-193) of
    the reduced point (red_x, red_y) on a model file with num_rows × num_cols: (x, y, z,
    objective), each vector empty when postsolve cleared it; None when presolve does not reduce."""
    L = lib()
    red_x = np.ascontiguousarray(red_x, dtype=np.float64)
    red_y = np.ascontiguousarray(red_y, dtype=np.float64)
    x, y, z = np.zeros(num_cols), np.zeros(num_rows), np.zeros(num_cols)
    obj = np.zeros(1)
    sizes = (ctypes.c_longlong * 3)()
    if not L.ref_postsolve_file(os.fsencode(path), _d(red_x), len(red_x), _d(red_y), len(red_y), _d(x), _d(y), _d(z),
                                _d(obj), sizes):
        return None
    return x[:sizes[0]], y[:sizes[1]], z[:sizes[2]], float(obj[0])


def bound(lp, y, use_implied=True):
    """certified_dual_bound (reference src/core/safe_bound.cpp:178)."""
    L = lib()
    args, keep = _model_args(lp)
    out = np.zeros(4)
    L.ref_bound(*args, _d(np.ascontiguousarray(y, dtype=np.float64)), int(bool(use_implied)), _d(out))
    del keep
    return {"finite": bool(out[0]), "bound": out[1], "unbounded_row_terms": int(out[2]),
            "unbounded_col_terms": int(out[3])}


def certificate(lp, ray, x=None):
    """check_infeasibility_certificate (x None) / check_unboundedness_certificate
    (reference src/core/certificates.cpp:14, 88)."""
    L = lib()
    args, keep = _model_args(lp)
    r = np.ascontiguousarray(ray, dtype=np.float64)
    xx = np.zeros(lp.num_cols) if x is None else np.ascontiguousarray(x, dtype=np.float64)
    out = np.zeros(5)
    L.ref_certificate(0 if x is None else 1, *args, _d(xx), _d(r), _d(out))
    del keep
    return {"present": bool(out[0]), "passed": bool(out[1]), "rigorous": bool(out[2]), "measure": out[3],
            "violation": out[4]}


class Backend:
    """The reference CpuBackend over make_scaled_problem(model, scaling options)."""

    def __init__(self, lp, ruiz_iterations=10, pock_chambolle=True, bound_objective_rescaling=True,
                 geometric_mean_iterations=12, geometric_mean_min_log10_range=4.5):
        self.L = lib()
        args, self._keep = _model_args(lp)
        self.m, self.n = lp.num_rows, lp.num_cols
        self.h = self.L.ref_backend_new(*args, ruiz_iterations, int(pock_chambolle), int(bound_objective_rescaling),
                                        geometric_mean_iterations, geometric_mean_min_log10_range)
        self.sizes = []

    def __del__(self):
        if getattr(self, "h", None):
            self.L.ref_backend_free(self.h)
            self.h = None

    def scaled(self, which: int) -> np.ndarray:
        cnt = self.L.ref_scaled_get(self.h, which, None)
        out = np.empty(cnt)
        self.L.ref_scaled_get(self.h, which, _d(out))
        return out

    def structure(self, which: int):
        rows = self.m if which == 0 else self.n
        nnz = self.L.ref_scaled_structure(self.h, which, None, None)
        rp, col = np.empty(rows + 1, dtype=np.int32), np.empty(nnz, dtype=np.int32)
        self.L.ref_scaled_structure(self.h, which, _i(rp), _i(col))
        return rp, col

    def scalars(self):
        out = np.zeros(4)
        self.L.ref_scaled_scalars(self.h, _d(out))
        return {"bound_scale": out[0], "obj_scale": out[1], "log10_range": out[2],
                "geometric_mean_applied": bool(out[3])}

    def norm2_estimate(self) -> float:
        return self.L.ref_norm2(self.h)

    def set_precision(self, mixed: bool):
        self.L.ref_backend_set_precision(self.h, int(mixed))

    def create(self, dual: bool) -> int:
        self.sizes.append(self.m if dual else self.n)
        return self.L.ref_backend_create(self.h, int(dual))

    def upload(self, v, a):
        a = np.ascontiguousarray(a, dtype=np.float64)
        self.L.ref_backend_upload(self.h, v, _d(a), a.size)

    def download(self, v):
        out = np.empty(self.sizes[v])
        self.L.ref_backend_download(self.h, v, _d(out), out.size)
        return out

    def __getattr__(self, name):
        f = getattr(self.L, "ref_backend_" + name)
        return lambda *a: f(self.h, *a)

    def kkt(self, xs, ys):
        out = np.zeros(8)
        self.L.ref_backend_kkt(self.h, xs, ys, _d(out))
        return dict(zip(["primal_residual", "dual_residual", "primal_obj", "dual_obj", "b_norm", "c_norm",
                         "primal_max_rel", "dual_max_rel"], out))
