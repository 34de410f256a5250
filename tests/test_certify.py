"""Rigorous verification on the host (csrc/certify.cpp) against the reference's own
certified_dual_bound, implied bounds and certificate checks (src/core/safe_bound.cpp,
implied_bounds.cpp, certificates.cpp, run from oracle/_ref). The bound is taken in the
reference's summation order with the same double-double arithmetic, so it must agree bit for bit,
whatever the number of host threads used for the per-column work. CPU only."""
import numpy as np
import pytest

import ps26119
from ps26119 import generators as g
import lps

HAND = [lps.wyndor, lps.mixed_rows, lps.max_ranged, lps.infeasible, lps.unbounded]


def one_sided(lp):
    """The same LP with every column bounded below only (implied bounds become necessary)."""
    return lp.with_data(col_upper=np.full(lp.num_cols, np.inf))


def cases():
    out = [(f.__name__, f()) for f in HAND]
    out += [("long_row", lps.long_row(300, 600)),
            ("random_m100", g.random_lp(100, seed=1)), ("random_m300", g.random_lp(300, seed=2)),
            ("staircase_T2", g.staircase_lp(2, seed=1)),
            ("random_m200_one_sided", one_sided(g.random_lp(200, seed=3))),
            ("staircase_T2_one_sided", one_sided(g.staircase_lp(2, seed=5)))]
    return out


CASES = cases()


def same(a, b):
    return a == b or (np.isnan(a) and np.isnan(b))


@pytest.mark.parametrize("name,lp", CASES, ids=[c[0] for c in CASES])
@pytest.mark.parametrize("use_implied", [True, False])
def test_bound_is_bit_identical_to_reference(ref, name, lp, use_implied):
    rng = np.random.default_rng(4)
    ys = [np.zeros(lp.num_rows), rng.standard_normal(lp.num_rows), 1e-3 * rng.standard_normal(lp.num_rows)]
    s = ref.solve(lp, presolve=False, iteration_limit=50_000)
    if np.all(np.isfinite(s.y)):
        ys.append(s.y)
    for y in ys:
        want = ref.bound(lp, y, use_implied)
        got = ps26119.certified_bound(lp, y, use_implied)
        assert got["finite"] == want["finite"], name
        assert same(got["bound"], want["bound"]), (name, got["bound"], want["bound"])
        assert got["unbounded_row_terms"] == want["unbounded_row_terms"]
        assert got["unbounded_col_terms"] == want["unbounded_col_terms"]


def test_bound_of_a_solved_lp_is_rigorous_and_tight(ref):
    # Wyndor: max 3x1 + 5x2, optimum 36; the bound from the optimal duals is ≥ 36 and close to it
    lp = lps.wyndor()
    s = ref.solve(lp, presolve=False)
    b = ps26119.certified_bound(lp, s.y)
    assert b["finite"] and b["bound"] >= 36.0 - 1e-12 and b["bound"] - 36.0 <= 1e-6


def test_bound_many_columns_uses_threads_bit_identically(ref):
    lp = g.random_lp(50_000, seed=9)  # 75,000 columns: the per-column work is split over threads
    y = np.random.default_rng(2).standard_normal(lp.num_rows)
    for use_implied in (True, False):
        want = ref.bound(lp, y, use_implied)
        got = ps26119.certified_bound(lp, y, use_implied)
        assert got["bound"] == want["bound"] and got["finite"] == want["finite"]


def test_certificates_match_reference(ref):
    inf = lps.infeasible()
    s = ref.solve(inf, presolve=False)
    assert s.status == "Infeasible"
    want = ref.certificate(inf, s.dual_ray)
    got = ps26119.check_certificate(inf, s.dual_ray)
    assert got == want and got["passed"]
    # a wrong Farkas vector fails both
    bad = -s.dual_ray
    assert ps26119.check_certificate(inf, bad) == ref.certificate(inf, bad)
    assert not ps26119.check_certificate(inf, bad)["passed"]
    unb = lps.unbounded()
    s = ref.solve(unb, presolve=False)
    assert s.status == "Unbounded"
    want = ref.certificate(unb, s.primal_ray, x=s.x)
    got = ps26119.check_certificate(unb, s.primal_ray, x=s.x)
    assert got == want and got["passed"]
    flipped = -s.primal_ray
    assert ps26119.check_certificate(unb, flipped, x=s.x) == ref.certificate(unb, flipped, x=s.x)


def test_certificate_of_feasible_lp_never_passes(ref):
    lp = g.random_lp(100, seed=4)
    r = np.random.default_rng(1).standard_normal(lp.num_rows)
    got = ps26119.check_certificate(lp, r)
    assert got == ref.certificate(lp, r) and not got["passed"]


def test_invalid_arguments():
    lp = lps.wyndor()
    ri = lp.row_index.copy()
    ri[0] = lp.num_rows  # a row index out of range
    with pytest.raises(ValueError):
        ps26119.certified_bound(lp.with_data(row_index=ri), np.zeros(lp.num_rows))


def test_certificate_tests_with_infinite_bounds_match_reference(ref):
    """Both certificate tests on models whose rows and columns are one-sided, free or boxed, with
    random multipliers, points and rays: every field (passed, rigorous, measure, violation) equals
    the reference's, so the infinite-bound branches (a picked bound that is infinite counts as a
    violation; the recession cone only constrains the finite sides) take the same terms in the
    same order."""
    rng = np.random.default_rng(12)
    for trial in range(12):
        lp = g.random_lp(300, seed=20 + trial)
        m, n = lp.num_rows, lp.num_cols
        kind_r = rng.integers(0, 4, m)  # 0 equality, 1 >=, 2 <=, 3 free
        b = lp.row_lower.copy()
        rl = np.where((kind_r == 2) | (kind_r == 3), -np.inf, b - (kind_r == 1) * rng.uniform(0, 1, m))
        ru = np.where((kind_r == 1) | (kind_r == 3), np.inf, b + (kind_r == 2) * rng.uniform(0, 1, m))
        kind_c = rng.integers(0, 4, n)  # 0 boxed, 1 lower only, 2 upper only, 3 free
        cl = np.where((kind_c == 2) | (kind_c == 3), -np.inf, 0.0)
        cu = np.where((kind_c == 1) | (kind_c == 3), np.inf, 10.0)
        model = lp.with_data(row_lower=rl, row_upper=ru, col_lower=cl, col_upper=cu)
        r = rng.standard_normal(m) * (rng.uniform(0, 1, m) < 0.7)
        assert ps26119.check_certificate(model, r) == ref.certificate(model, r), trial
        x = np.clip(rng.uniform(-1, 11, n), np.where(np.isfinite(cl), cl, -1e3), np.where(np.isfinite(cu), cu, 1e3))
        ray = rng.standard_normal(n) * (rng.uniform(0, 1, n) < 0.5)
        assert ps26119.check_certificate(model, ray, x=x) == ref.certificate(model, ray, x=x), trial
