"""The full r²HPDHG solve on the GPU against the reference CPU engine, through the C ABI.

Parity bars (stated per test):
  * exact mode (reference summation order): the trajectory is BIT-IDENTICAL to the reference
    CPU engine — same status, same iteration count, identical x, y, z and objective.
  * fast mode (tree order for the decision-only sums): same status, iteration count within one
    check (|Δ| <= K = 64), objective within 1e-9 relative, in-process check PASS.
  * C API (presolve on, as the reference's ps26119_solve_lp): the same bars against the
    reference's C-API-level solve.
"""
import json
import os

import numpy as np
import pytest

import lps
import ps26119
from ps26119 import generators as g

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_runs.json")
K = 64
REL_OBJ = 1e-9


def golden(case, precision, presolve):
    for r in json.load(open(GOLDEN))["runs"]:
        if r["case"] == case and r["precision"] == precision and r["presolve"] == presolve:
            return r
    raise KeyError(case)


def gpu_solve(lp, precision="fp64", exact=False, presolve=False, **kw):
    return ps26119.solve_lp(lp.c, (lp.col_start, lp.row_index, lp.value), lp.row_lower, lp.row_upper, lp.col_lower,
                            lp.col_upper, sense=lp.sense, offset=lp.offset, algorithm="r2hpdhg", precision=precision,
                            engine={"presolve": presolve, "exact": exact}, **kw)


def reference_solve(lp, precision="fp64", presolve=False):
    import reference
    if reference.available():
        return reference.solve(lp, presolve=presolve, precision=precision)
    if presolve:
        pytest.skip("reference library not built; the oracle has no presolve")
    import oracle
    return oracle.solve(lp, precision=precision)


CASES = {"wyndor": lps.wyndor, "mixed_rows": lps.mixed_rows, "max_ranged": lps.max_ranged,
         "long_row": lps.long_row, "random_m100_s1": lambda: g.random_lp(100, seed=1),
         "random_m300_s1": lambda: g.random_lp(300, seed=1), "random_m1000_s2": lambda: g.random_lp(1000, seed=2),
         "staircase_T2_s1": lambda: g.staircase_lp(2), "staircase_T4_s1": lambda: g.staircase_lp(4),
         "staircase_T8_s1": lambda: g.staircase_lp(8)}


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("name", sorted(CASES))
def test_exact_mode_trajectory_is_bit_identical(name, precision):
    lp = CASES[name]()
    r = reference_solve(lp, precision)
    s = gpu_solve(lp, precision, exact=True)
    assert s.status_name == r.status, s.message
    assert s.iterations == r.iterations
    assert np.array_equal(s.x, r.x) and np.array_equal(s.y, r.y) and np.array_equal(s.z, r.z)
    assert s.objective == r.objective
    if hasattr(r, "certified_bound"):  # the reference's rounding-proof bound from the same y
        assert s.certified_bound == r.certified_bound or (np.isnan(s.certified_bound) and np.isnan(r.certified_bound))
        assert (s.check == "PASS") == (r.check == 1)


def fast_mode_bar(name, s, r):
    """Fast mode takes in tree order only the sums that feed decisions (KKT statistics,
    objectives, ray tests, the restart residual); every sum that enters the iterates' arithmetic
    (scaling, ‖Ã‖₂, ω0, the PID distances) is in the reference's order. So the trajectory is the
    reference's unless a decision lands within rounding of its threshold, and the bar is the
    iteration count within one check (K = 64) and the objective within 1e-9 relative."""
    assert abs(s.iterations - r.iterations) <= K, (s.iterations, r.iterations)
    assert abs(s.objective - r.objective) <= REL_OBJ * (1 + abs(r.objective))


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("name", sorted(CASES))
def test_fast_mode_matches_reference(name, precision):
    lp = CASES[name]()
    r = reference_solve(lp, precision)
    s = gpu_solve(lp, precision, exact=False)
    assert s.status_name == r.status, s.message
    fast_mode_bar(name, s, r)
    assert s.check == "PASS", s.message


@pytest.mark.parametrize("name", ["random_m300_s1", "staircase_T4_s1", "staircase_T8_s1"])
def test_c_api_exact_mode_with_presolve_is_bit_identical(name):
    """Presolve + exact mode through the C API reproduces the reference's C-API solve exactly."""
    import hashlib
    lp = CASES[name]()
    rec = golden(name, "fp64", True)
    s = gpu_solve(lp, "fp64", exact=True, presolve=True)
    assert s.status_name == rec["status"] and s.iterations == rec["iterations"]
    assert s.objective == float.fromhex(rec["objective"])
    assert hashlib.sha256(s.x.tobytes()).hexdigest() == rec["x_sha256"]
    assert hashlib.sha256(s.y.tobytes()).hexdigest() == rec["y_sha256"]
    assert s.certified_bound == float.fromhex(rec["certified_bound"])


@pytest.mark.parametrize("name", ["wyndor", "mixed_rows", "random_m300_s1", "staircase_T4_s1", "staircase_T8_s1"])
def test_c_api_with_presolve_matches_reference_c_api(name):
    """ps26119_solve_lp_ex (presolve on) vs the reference's solve() with presolve on."""
    lp = CASES[name]()
    rec = golden(name, "fp64", True)
    s = ps26119.solve_lp(lp.c, (lp.col_start, lp.row_index, lp.value), lp.row_lower, lp.row_upper, lp.col_lower,
                         lp.col_upper, sense=lp.sense, offset=lp.offset, algorithm="r2hpdhg")
    assert s.status_name == rec["status"], s.message

    class R:
        iterations = rec["iterations"]
        objective = float.fromhex(rec["objective"])
    fast_mode_bar(name, s, R)
    assert s.check == "PASS"


def test_wyndor_known_answer_through_c_api():
    """reference tests/unit/test_c_api.cpp:33-49 (r²HPDHG row): objective 36, x = (2, 6),
    y1 = 1.5, y2 = 1, in-process check PASS."""
    r = ps26119.solve_lp([3, 5], [[1, 0], [0, 2], [3, 2]], [-np.inf] * 3, [4, 12, 18], sense=-1, algorithm="r2hpdhg")
    assert r.status == ps26119.OPTIMAL, r.message
    assert abs(r.objective - 36) <= 1e-6
    assert np.allclose(r.x, [2, 6], atol=1e-5)
    assert abs(r.y[1] - 1.5) <= 1e-5 and abs(r.y[2] - 1.0) <= 1e-5
    assert r.check == "PASS" and r.engine
    r = ps26119.solve_lp([3, 5], [[1, 0], [0, 2], [3, 2]], [-np.inf] * 3, [4, 12, 18], sense=-1, offset=1.0)
    assert r.status == ps26119.OPTIMAL and abs(r.objective - 37) <= 1e-6  # offset included (test_c_api.cpp:53-58)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_infeasible_and_unbounded_verdicts(precision):
    """reference tests/unit/test_gpu.cpp:193-220: Infeasible and Unbounded on the GPU."""
    s = gpu_solve(lps.infeasible(), precision, exact=False)
    assert s.status == ps26119.INFEASIBLE, s.message
    assert s.dual_ray is not None
    assert s.check == "PASS" and "Farkas certificate" in s.message  # checked on the original model
    s = gpu_solve(lps.unbounded(), precision, exact=False)
    assert s.status == ps26119.UNBOUNDED, s.message
    assert s.primal_ray is not None
    assert s.check == "PASS"  # point and ray checked on the original model
    # through the C API with presolve, as the reference's C API answers (golden records: check 1)
    for lp, name in ((lps.infeasible(), "infeasible"), (lps.unbounded(), "unbounded")):
        rec = golden(name, precision, True)
        s = gpu_solve(lp, precision, exact=False, presolve=True)
        assert s.status_name == rec["status"] and (s.check == "PASS") == (rec["check"] == 1), s.message


def test_repeated_solves_are_bit_identical():
    """Determinism (reference test_gpu.cpp:221-228): same iterations, identical x."""
    lp = g.random_lp(2000, seed=4)
    a = gpu_solve(lp)
    b = gpu_solve(lp)
    assert a.status == b.status == ps26119.OPTIMAL
    assert a.iterations == b.iterations and np.array_equal(a.x, b.x) and np.array_equal(a.y, b.y)


def test_device_entry_point_equals_host_entry_point():
    torch = pytest.importorskip("torch")
    lp = g.random_lp(500, seed=6)
    dev = torch.device("cuda:0")
    t = lambda a, dt: torch.as_tensor(np.ascontiguousarray(a), dtype=dt, device=dev)
    arrs = [t(lp.c, torch.float64), t(lp.col_lower, torch.float64), t(lp.col_upper, torch.float64),
            t(lp.row_lower, torch.float64), t(lp.row_upper, torch.float64), t(lp.col_start, torch.int32),
            t(lp.row_index, torch.int32), t(lp.value, torch.float64)]
    x = torch.empty(lp.num_cols, dtype=torch.float64, device=dev)
    y = torch.empty(lp.num_rows, dtype=torch.float64, device=dev)
    z = torch.empty(lp.num_cols, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream()
    r = ps26119.solve_lp_device(lp.num_rows, lp.num_cols, lp.sense, lp.offset, [a.data_ptr() for a in arrs],
                                engine={"presolve": False}, out=(x.data_ptr(), y.data_ptr(), z.data_ptr()),
                                stream=stream.cuda_stream)
    torch.cuda.synchronize()
    h = gpu_solve(lp)
    assert r.status == h.status == ps26119.OPTIMAL, r.message
    assert r.iterations == h.iterations
    assert np.array_equal(x.cpu().numpy(), h.x) and np.array_equal(y.cpu().numpy(), h.y)
    assert np.array_equal(z.cpu().numpy(), h.z)
    assert r.check == "PASS"


def test_random_10k_matches_recorded_reference_run():
    """The 10k x 15k random LP (249,088 reference iterations) in fast mode, fp64."""
    rec = golden("random_m10000_s1", "fp64", False)
    lp = g.random_lp(10000, seed=1)
    s = gpu_solve(lp, "fp64", exact=False)
    assert s.status_name == "Optimal", s.message
    assert abs(s.iterations - rec["iterations"]) <= K, (s.iterations, rec["iterations"])
    ref_obj = float.fromhex(rec["objective"])
    assert abs(s.objective - ref_obj) <= REL_OBJ * (1 + abs(ref_obj))


def test_mixed_precision_stall_window():
    """mixed_stall_checks (this library's addition to the reference's PrecisionPolicy): a window of
    one check switches to fp64 no later than the reference's 10, a window of 10,000 keeps fp32
    until the 1e-6 switch; every answer is Optimal, checked, and within 1e-6 of the fp64 answer."""
    lp = g.random_lp(3000, seed=8)
    base = gpu_solve(lp, "fp64")
    assert base.status == ps26119.OPTIMAL, base.message
    switches = {}
    for window in (1, 0, 10000):
        s = ps26119.solve_lp(lp.c, (lp.col_start, lp.row_index, lp.value), lp.row_lower, lp.row_upper,
                             lp.col_lower, lp.col_upper, sense=lp.sense, offset=lp.offset, algorithm="r2hpdhg",
                             precision="mixed", engine={"presolve": False, "mixed_stall_checks": window})
        switches[window] = ps26119.last_stats()["switch_iteration"]
        assert s.status == ps26119.OPTIMAL and s.check == "PASS", (window, s.message)
        assert abs(s.objective - base.objective) <= 1e-6 * (1 + abs(base.objective)), window
    assert 0 < switches[1] <= switches[0] <= switches[10000], switches
