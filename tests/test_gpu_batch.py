"""GPU batch engine (ps26119_solve_batch) against the reference's solve_batch
(src/pdhg/batch.cpp:129-441, run from oracle/_ref).

Exact mode takes every per-scenario sum in the reference's order, so each scenario's status,
iteration count, objective and (x, y) are bit-identical to the reference's batch. Fast mode
differs only in the order of the sums; it is held to the answer (objective 1e-9 relative on the
random LPs, 5e-8 on the staircase LPs, as the single-LP engine) and to the reference test's own
contract (tests/unit/test_batch.cpp:28-62: every scenario equals its single solve within 1e-6)."""
import numpy as np
import pytest

import ps26119
from ps26119 import generators as g
import lps

pytestmark = pytest.mark.gpu


def ours(lp, scen, exact, tol=1e-8, iteration_limit=0):
    return ps26119.solve_batch(lp.c, (lp.col_start, lp.row_index, lp.value), lp.row_lower, lp.row_upper,
                               lp.col_lower, lp.col_upper, scenarios=scen, sense=lp.sense, offset=lp.offset,
                               tolerance=tol, iteration_limit=iteration_limit,
                               engine={"exact": exact, "presolve": False})


CASES = [
    ("random_m100_K5", lambda: g.random_lp(100, seed=3), 5),
    ("random_m300_K40", lambda: g.random_lp(300, seed=4), 40),   # 2 slots per lane (W > 32)
    ("staircase_T2_K4", lambda: g.staircase_lp(2, seed=2), 4),
    ("random_m200_K1", lambda: g.random_lp(200, seed=5), 1),
]


@pytest.mark.parametrize("name,make,K", CASES, ids=[c[0] for c in CASES])
def test_exact_batch_is_bit_identical_to_reference(ref, name, make, K):
    lp = make()
    scen = g.scenarios(lp, K, sigma=0.1, seed=7)
    limit = 200_000
    want = ref.batch(lp, scen, threads=4, iteration_limit=limit)
    got = ours(lp, scen, exact=True, iteration_limit=limit)
    assert len(got) == K
    for k in range(K):
        w, r = want[k], got[k]
        assert r.status_name == w["status"], (k, r.message)
        assert r.iterations == w["iterations"], k
        assert r.engine == "r2hpdhg-batch"
        if r.x is not None:
            assert r.objective.hex() == float(w["objective"]).hex(), k
            np.testing.assert_array_equal(r.x, w["x"])
            np.testing.assert_array_equal(r.y, w["y"])


@pytest.mark.parametrize("name,make,K", CASES[:3], ids=[c[0] for c in CASES[:3]])
def test_fast_batch_matches_reference_answers(ref, name, make, K):
    lp = make()
    scen = g.scenarios(lp, K, sigma=0.1, seed=7)
    want = ref.batch(lp, scen, threads=4, iteration_limit=200_000)
    got = ours(lp, scen, exact=False, iteration_limit=200_000)
    for k in range(K):
        if want[k]["status"] != "Optimal":
            continue
        assert got[k].status_name == "Optimal", got[k].message
        o, wo = got[k].objective, want[k]["objective"]
        # the single-LP fast-mode bar: 1e-9 on the random LPs; the staircase LPs' restart
        # decisions are sensitive to last-bit differences, so there the bar is 5e-8
        rel = 5e-8 if name.startswith("staircase") else 1e-9
        assert abs(o - wo) <= rel * (1 + abs(wo)), (k, o, wo)
        assert max(got[k].primal_residual, got[k].dual_residual, got[k].gap) <= 1e-8


def test_scenarios_match_single_solves():
    # reference tests/unit/test_batch.cpp:28-62 on generated LPs: each batch answer equals the
    # single solve of the same scenario model (objective 1e-6 relative), engine r2hpdhg-batch
    lp = g.random_lp(150, seed=12)
    scen = g.scenarios(lp, 6, sigma=0.1, seed=3)
    got = ours(lp, scen, exact=False)
    A = np.zeros((lp.num_rows, lp.num_cols))
    for j in range(lp.num_cols):
        for p in range(lp.col_start[j], lp.col_start[j + 1]):
            A[lp.row_index[p], j] = lp.value[p]
    for k, s in enumerate(scen):
        single = ps26119.solve_lp(s["obj"], (lp.col_start, lp.row_index, lp.value), s["row_lower"], s["row_upper"],
                                  lp.col_lower, lp.col_upper, algorithm="r2hpdhg")
        assert single.status_name == "Optimal" and got[k].status_name == "Optimal", (single.message, got[k].message)
        assert abs(got[k].objective - single.objective) <= 1e-6 * (1 + abs(single.objective))
        # the reported (x, y, z) satisfy z = c − Aᵀy and the objective
        np.testing.assert_allclose(got[k].z, s["obj"] - A.T @ got[k].y, rtol=0, atol=1e-9)
        assert abs(got[k].objective - (lp.offset + s["obj"] @ got[k].x)) <= 1e-9 * (1 + abs(got[k].objective))


def test_bad_scenario_fails_alone_and_max_sense(ref):
    # reference tests/unit/test_batch.cpp:64-80: max_ranged (optimum 21.5), a scenario with a
    # wrong-sized vector (NotSolved alone), a scenario with a changed objective
    lp = lps.max_ranged()
    c2 = lp.c * 1.5
    scen = [{}, {"obj": np.ones(lp.num_cols + 1)}, {"obj": c2}]
    got = ours(lp, scen, exact=True)
    assert got[0].status_name == "Optimal" and abs(got[0].objective - 21.5) <= 1e-6
    assert got[1].status_name == "NotSolved" and "wrong vector sizes" in got[1].message
    assert got[2].status_name == "Optimal"
    single = ref.solve(lp.with_data(c=c2), presolve=False)
    assert abs(got[2].objective - single.objective) <= 1e-6 * (1 + abs(single.objective))
    # crossed bounds in one scenario: Infeasible without running, the others unaffected
    cu = lp.col_upper.copy()
    cl = lp.col_lower.copy()
    cl[0], cu[0] = 2.0, 1.0
    got = ours(lp, [{"col_lower": cl, "col_upper": cu}, {}], exact=True)
    assert got[0].status_name == "Infeasible" and "bounds cross" in got[0].message
    assert got[1].status_name == "Optimal"
    # non-finite data: that scenario alone is NotSolved
    bad_c = lp.c.copy()
    bad_c[1] = np.nan
    got = ours(lp, [{"obj": bad_c}, {}], exact=True)
    assert got[0].status_name == "NotSolved" and got[1].status_name == "Optimal"


def test_empty_batch_and_iteration_limit():
    lp = g.random_lp(100, seed=3)
    assert ours(lp, [], exact=False) == []
    got = ours(lp, g.scenarios(lp, 3, seed=1), exact=False, iteration_limit=128)
    assert all(r.status_name == "IterationLimit" and r.iterations == 128 for r in got)
    assert all(r.x is not None and np.all(np.isfinite(r.x)) for r in got)


def test_batch_is_deterministic():
    lp = g.staircase_lp(2, seed=4)
    scen = g.scenarios(lp, 8, seed=2)
    a = ours(lp, scen, exact=False, iteration_limit=20_000)
    b = ours(lp, scen, exact=False, iteration_limit=20_000)
    for r, s in zip(a, b):
        assert r.iterations == s.iterations and r.objective == s.objective
        np.testing.assert_array_equal(r.x, s.x)


@pytest.mark.parametrize("name,make,K", [("random_m300_K12", lambda: g.random_lp(300, seed=6), 12),
                                         ("staircase_T3_K8", lambda: g.staircase_lp(3, seed=2), 8)],
                         ids=["random_m300_K12", "staircase_T3_K8"])
def test_mixed_batch_reaches_the_target_like_fp64(name, make, K):
    """The mixed form of the batch (fp32 SpMM and iterates until every running slot asks for fp64
    under the reference's PrecisionPolicy, then fp64 to the target): every feasible scenario is
    Optimal at 1e-8 KKT (checked in fp64 on the original model), and its objective is the fp64
    batch's within 1e-6 relative — the error of mixed against fp64, per scenario."""
    lp = make()
    scen = g.feasible_scenarios(lp, K, sigma=0.1, seed=3)
    A = (lp.col_start, lp.row_index, lp.value)
    kw = dict(scenarios=scen, sense=lp.sense, offset=lp.offset, engine={"presolve": False})
    d = ps26119.solve_batch(lp.c, A, lp.row_lower, lp.row_upper, lp.col_lower, lp.col_upper, **kw)
    m = ps26119.solve_batch(lp.c, A, lp.row_lower, lp.row_upper, lp.col_lower, lp.col_upper, precision="mixed", **kw)
    for k in range(K):
        assert d[k].status == ps26119.OPTIMAL and m[k].status == ps26119.OPTIMAL, (k, d[k].message, m[k].message)
        assert max(m[k].primal_residual, m[k].dual_residual, m[k].gap) <= 1e-8
        err = abs(m[k].objective - d[k].objective) / (1.0 + abs(d[k].objective))
        assert err <= 1e-6, (k, err)
