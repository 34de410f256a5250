"""PDLP-style restarted averaged PDHG on the GPU (algorithm "pdlp") against the reference's
pdhg::solve_pdlp (src/pdhg/pdlp.cpp:9-126, run from oracle/_ref).

Exact mode reproduces the reference's trajectory bit for bit (status, iterations, x, y, z,
objective); fast mode is held to the answer, as the r²HPDHG engine."""
import numpy as np
import pytest

import ps26119
from ps26119 import generators as g
import lps

pytestmark = pytest.mark.gpu

CASES = {"wyndor": lps.wyndor, "mixed_rows": lps.mixed_rows, "max_ranged": lps.max_ranged,
         "random_m100_s1": lambda: g.random_lp(100, seed=1), "random_m300_s1": lambda: g.random_lp(300, seed=1),
         "staircase_T2_s1": lambda: g.staircase_lp(2), "infeasible": lps.infeasible, "unbounded": lps.unbounded}


def gpu_pdlp(lp, precision="fp64", exact=False, presolve=False, **kw):
    return ps26119.solve_lp(lp.c, (lp.col_start, lp.row_index, lp.value), lp.row_lower, lp.row_upper, lp.col_lower,
                            lp.col_upper, sense=lp.sense, offset=lp.offset, algorithm="pdlp", precision=precision,
                            engine={"presolve": presolve, "exact": exact}, **kw)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("name", sorted(CASES))
def test_exact_pdlp_is_bit_identical_to_reference(ref, name, precision):
    lp = CASES[name]()
    r = ref.solve(lp, precision=precision, algorithm="pdlp", iteration_limit=200_000)
    s = gpu_pdlp(lp, precision, exact=True, iteration_limit=200_000)
    assert s.status_name == r.status, s.message
    assert s.iterations == r.iterations
    assert s.engine == "pdlp-b200"
    if s.x is not None and r.status in ("Optimal", "IterationLimit"):
        assert np.array_equal(s.x, r.x) and np.array_equal(s.y, r.y) and np.array_equal(s.z, r.z)
        assert s.objective == r.objective
    if r.status == "Infeasible":
        assert np.array_equal(s.dual_ray, r.dual_ray)
    assert (s.check == "PASS") == (r.check == 1), s.message


@pytest.mark.parametrize("name", ["wyndor", "random_m300_s1", "staircase_T2_s1"])
def test_fast_pdlp_matches_reference_answer(ref, name):
    lp = CASES[name]()
    r = ref.solve(lp, algorithm="pdlp")
    s = gpu_pdlp(lp, exact=False)
    assert s.status_name == r.status == "Optimal", s.message
    rel = 5e-8 if name.startswith("staircase") else 1e-9
    assert abs(s.objective - r.objective) <= rel * (1 + abs(r.objective))
    assert max(s.primal_residual, s.dual_residual, s.gap) <= 1e-8
    assert s.check == "PASS"


def test_pdlp_through_c_api_with_presolve(ref):
    lp = g.random_lp(300, seed=1)
    r = ref.solve(lp, presolve=True, algorithm="pdlp")
    s = gpu_pdlp(lp, exact=True, presolve=True)
    assert s.status_name == r.status == "Optimal"
    assert s.iterations == r.iterations and s.objective == r.objective
    assert s.certified_bound == r.certified_bound
