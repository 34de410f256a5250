"""The C-ABI library: it loads, exports every symbol the headers declare, keeps the reference's
struct layout and enum values, and validates arguments before touching the GPU. CPU only:
no call here launches a kernel."""
import ctypes
import os
import re

import numpy as np
import pytest

import ps26119
import lps

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = []
    for h in ("ps26119.h", "ps26119_backend.h"):
        text = open(os.path.join(ROOT, "include", h)).read()
        names += re.findall(r"PS26119_API [^;{]*?\b(ps26119_\w+)\(", text)
    return names


def test_library_loads_and_exports_every_declared_symbol():
    L = ps26119.load()
    names = declared_symbols()
    assert len(names) >= 30
    for n in names:
        assert hasattr(L, n), n
    assert set(names) == set(ps26119.EXPORTS)


def test_struct_layouts_match_reference_abi():
    # include/ps26119/ps26119.h:33-63 of the reference, x86-64
    assert ctypes.sizeof(ps26119._Options) == 64
    assert ps26119._Options.warm_x.offset == 48
    assert ctypes.sizeof(ps26119._Result) == 256
    assert ps26119._Result.engine.offset == 72 and ps26119._Result.message.offset == 88
    assert ps26119._Result.check.offset == 248


def test_version_and_default_options():
    assert ps26119.version().startswith("0.1.0")
    o = ps26119._Options()
    ps26119.load().ps26119_default_options(ctypes.byref(o))
    assert (o.algorithm, o.precision, o.use_gpu, o.threads) == (0, 0, 0, 1)
    assert o.tolerance == 1e-8 and o.time_limit == 3600.0 and o.iteration_limit == 100_000_000


def _call(L, lp, opt=None, result=True):
    res = ps26119._Result()
    P = ps26119._ptr
    f = lambda a: np.ascontiguousarray(a, dtype=np.float64)
    i = lambda a: np.ascontiguousarray(a, dtype=np.int32)
    a = [f(lp.c), f(lp.col_lower), f(lp.col_upper), f(lp.row_lower), f(lp.row_upper), i(lp.col_start),
         i(lp.row_index), f(lp.value)]
    st = L.ps26119_solve_lp_ex(lp.num_rows, lp.num_cols, lp.sense, lp.offset, P(a[0]), P(a[1]), P(a[2]), P(a[3]),
                               P(a[4]), P(a[5], ctypes.c_int), P(a[6], ctypes.c_int), P(a[7]),
                               ctypes.byref(opt) if opt is not None else None,
                               ctypes.byref(res) if result else None, None, None, None, None, None)
    return st, res


def test_invalid_arguments_never_reach_the_engine():
    """reference c_api.cpp:107-120 and to_options (c_api.cpp:29-56)."""
    L = ps26119.load()
    lp = lps.wyndor()
    st, _ = _call(L, lp, result=False)
    assert st == ps26119.INVALID_ARGUMENT
    bad = lp.with_data(num_rows=-1)
    st, res = _call(L, bad)
    assert st == ps26119.INVALID_ARGUMENT and b"negative dimension" in res.message
    for field, value, text in (("tolerance", -1.0, b"tolerance"), ("iteration_limit", -5, b"iteration_limit"),
                               ("algorithm", 99, b"unknown algorithm"), ("precision", 7, b"unknown precision"),
                               ("threads", -1, b"threads"), ("time_limit", float("nan"), b"time_limit")):
        o = ps26119._options("auto", "fp64", True, 1e-8, 3600.0, 0, 0, 1)
        setattr(o, field, value)
        st, res = _call(L, lp, o)
        assert st == ps26119.INVALID_ARGUMENT, field
        assert text in res.message, (field, res.message)
    dup = lp.with_data(row_index=np.array([0, 0, 1, 2], dtype=np.int32))
    st, res = _call(L, dup)
    assert st == ps26119.INVALID_ARGUMENT and b"invalid model" in res.message


def test_backend_rejects_null_arguments_before_the_device():
    """The plugin ABI checks its arrays and handles like the solve entry points do: a NULL
    array or backend is INVALID_ARGUMENT with a message, never a crash or a device call."""
    L = ps26119.load()
    lp = lps.wyndor()
    P = ps26119._ptr
    f = lambda a: np.ascontiguousarray(a, dtype=np.float64)
    i = lambda a: np.ascontiguousarray(a, dtype=np.int32)
    arrays = [f(lp.c), f(lp.col_lower), f(lp.col_upper), f(lp.row_lower), f(lp.row_upper), i(lp.col_start),
              i(lp.row_index), f(lp.value)]
    for k, text in ((0, b"column data"), (3, b"row bounds"), (6, b"matrix arrays"), (7, b"matrix arrays")):
        args = [P(a, ctypes.c_int) if a.dtype == np.int32 else P(a) for a in arrays]
        args[k] = None
        h = ctypes.c_void_p(1)
        st = L.ps26119_backend_new(ctypes.byref(h), lp.num_rows, lp.num_cols, lp.sense, lp.offset, *args, None, 0)
        assert st == ps26119.INVALID_ARGUMENT, k
        assert not h.value, k
        assert text in L.ps26119_backend_last_error(), (k, L.ps26119_backend_last_error())
    out = ctypes.c_double()
    assert L.ps26119_backend_dot(None, 0, 0, ctypes.byref(out)) == ps26119.INVALID_ARGUMENT
    assert b"null backend" in L.ps26119_backend_last_error()
    assert L.ps26119_backend_sync(None) == ps26119.INVALID_ARGUMENT
    assert L.ps26119_backend_scaled_get(None, 0, None) == -1


def test_cpu_engine_requests_are_refused_without_fallback():
    L = ps26119.load()
    o = ps26119._options("r2hpdhg", "fp64", False, 1e-8, 3600.0, 0, 0, 1)
    st, res = _call(L, lps.wyndor(), o)
    assert st == ps26119.NOT_SOLVED and b"use_gpu" in res.message
    o = ps26119._options("simplex", "fp64", True, 1e-8, 3600.0, 0, 0, 1)
    st, res = _call(L, lps.wyndor(), o)
    assert st == ps26119.NOT_SOLVED and b"not provided" in res.message


def test_no_device_reports_not_solved():
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    r = ps26119.solve_lp([3, 5], [[1, 0], [0, 2], [3, 2]], [-np.inf] * 3, [4, 12, 18], sense=-1)
    assert r.status == ps26119.NOT_SOLVED and "CUDA backend unavailable" in r.message


def test_solve_mps_argument_errors():
    r = ps26119.solve_mps(None)
    assert r.status == ps26119.INVALID_ARGUMENT and "path is NULL" in r.message


def test_engine_options_layout_and_validation():
    """ps26119_engine_options (this library's addition): its defaults, and a negative precision
    switch stall window refused before the engine starts."""
    L = ps26119.load()
    assert ctypes.sizeof(ps26119._EngineOptions) == 48
    eo = ps26119._EngineOptions()
    L.ps26119_default_engine_options(ctypes.byref(eo))
    assert (eo.presolve, eo.check_every, eo.exact_reductions, eo.mixed_stall_checks) == (1, 64, 0, 0)
    r = ps26119.solve_lp([3, 5], [[1, 0], [0, 2], [3, 2]], [-np.inf] * 3, [4, 12, 18], sense=-1, precision="mixed",
                         engine={"mixed_stall_checks": -1})
    assert r.status == ps26119.INVALID_ARGUMENT and "mixed_stall_checks" in r.message
