"""The C oracle (oracle/pdhg_oracle.c) is pinned to the REFERENCE: bit-identical trajectories
against the reference built from its own sources (oracle/_ref), the reference's recorded runs
(tests/golden/reference_runs.json), and the known answers of the reference's own unit tests.
CPU only."""
import json
import os

import numpy as np
import pytest

import lps
from ps26119 import generators as g
from conftest import REFERENCE_DATA

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_runs.json")

SMALL = {
    "wyndor": lps.wyndor, "mixed_rows": lps.mixed_rows, "max_ranged": lps.max_ranged,
    "infeasible": lps.infeasible, "unbounded": lps.unbounded, "long_row": lps.long_row,
    "random_m100_s1": lambda: g.random_lp(100, seed=1), "random_m300_s1": lambda: g.random_lp(300, seed=1),
    "random_m1000_s2": lambda: g.random_lp(1000, seed=2), "staircase_T2_s1": lambda: g.staircase_lp(2),
    "staircase_T4_s1": lambda: g.staircase_lp(4), "staircase_T8_s1": lambda: g.staircase_lp(8),
}


def same(a, b):
    return np.array_equal(a, b, equal_nan=True)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("name", sorted(SMALL))
def test_oracle_trajectory_is_bit_identical_to_reference(ref, orc, name, precision):
    lp = SMALL[name]()
    r = ref.solve(lp, presolve=False, precision=precision)
    o = orc.solve(lp, precision=precision)
    assert o.status == r.status, (o.message, r.message)
    if r.status == "Unbounded" and "zero-objective solve" in r.message:
        # the reference dispatcher (solve.cpp:552-581) adds a feasibility solve after the engine
        extra = int(r.message.split("zero-objective solve (")[1].split(" ")[0])
        assert o.iterations == r.iterations - extra
    else:
        assert o.iterations == r.iterations
    if r.status == "Optimal":
        assert same(o.x, r.x) and same(o.y, r.y) and same(o.z, r.z)
        assert o.objective == r.objective
        assert o.primal_weight == r.primal_weight


def test_oracle_matches_recorded_reference_runs(orc):
    """Every engine-level record of the reference (presolve off) is reproduced exactly."""
    import hashlib
    runs = json.load(open(GOLDEN))["runs"]
    checked = 0
    for rec in runs:
        if rec["presolve"] or rec["case"] not in SMALL:
            continue
        lp = SMALL[rec["case"]]()
        o = orc.solve(lp, precision=rec["precision"])
        assert o.status == rec["status"], rec["case"]
        extra = 0
        if "zero-objective solve (" in rec["message"]:  # dispatcher feasibility solve, solve.cpp:552-581
            extra = int(rec["message"].split("zero-objective solve (")[1].split(" ")[0])
        assert o.iterations == rec["iterations"] - extra, rec["case"]
        if rec["status"] == "Optimal":
            assert float.fromhex(rec["objective"]) == o.objective
            assert hashlib.sha256(o.x.tobytes()).hexdigest() == rec["x_sha256"], rec["case"]
            assert hashlib.sha256(o.y.tobytes()).hexdigest() == rec["y_sha256"], rec["case"]
        checked += 1
    assert checked >= 20


def test_oracle_known_answers(orc):
    """Wyndor objective 36 at x = (2, 6) with y = (0, 1.5, 1) (reference test_c_api.cpp:36-41,
    test_pdhg.cpp:125-134) and max_ranged 21.5 (test_batch.cpp:66-73)."""
    s = orc.solve(lps.wyndor())
    assert s.status == "Optimal"
    assert abs(s.objective - 36) <= 1e-6
    assert np.allclose(s.x, [2, 6], atol=1e-5)
    assert np.allclose(s.y[1:], [1.5, 1.0], atol=1e-5)
    s = orc.solve(lps.max_ranged())
    assert s.status == "Optimal" and abs(s.objective - 21.5) <= 1e-6
    assert orc.solve(lps.infeasible()).status == "Infeasible"
    assert orc.solve(lps.unbounded()).status == "Unbounded"


def test_oracle_scaling_and_norm_are_bit_identical(ref, orc):
    for lp in (lps.mixed_rows(), g.random_lp(300), g.staircase_lp(4), lps.long_row()):
        rb = ref.Backend(lp)
        sc = orc.Scaled(lp)
        for which in range(9):
            assert same(rb.scaled(which), sc.get(which)), which
        assert rb.scalars() == sc.scalars()
        assert rb.norm2_estimate() == sc.norm2()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_oracle_backend_ops_match_reference(ref, orc, precision):
    """The op sequence of the reference's Gpu.BackendOpsMatchCpu (test_gpu.cpp:33-95)."""
    for lp in (lps.mixed_rows(), g.random_lp(200), g.staircase_lp(2)):
        sc = orc.Scaled(lp)
        backs = [ref.Backend(lp), orc.Backend(sc)]
        got = []
        for b in backs:
            b.set_precision(precision == "mixed")
            x, x0, xh, xb, gg = (b.create(False) for _ in range(5))
            y, y0, yh, yb, ax = (b.create(True) for _ in range(5))
            b.upload(x, np.sin(1.0 + np.arange(lp.num_cols)))
            b.upload(y, np.cos(2.0 + np.arange(lp.num_rows)))
            b.copy(x0, x)
            b.copy(y0, y)
            for it in range(20):
                w = (it + 1.0) / (it + 2.0)
                b.spmv_t(y, gg)
                b.r2h_primal(x, x0, gg, 0.3, w, 1.0, xh, xb)
                b.spmv(xb, ax)
                b.r2h_dual(y, y0, ax, 0.4, w, 1.0, yh, yb)
            b.primal_step(x, gg, 0.2, xb)
            b.dual_step(y, ax, 0.5, yb)
            b.axpby(0.3, xh, -1.7, xb)
            vecs = [b.download(v) for v in (x, xh, xb, y, yh, yb)]
            scal = [b.dot(x, xh), b.norm2(y), b.diff_norm2(x, x0)]
            got.append((vecs, scal, b.kkt(xh, yh)))
        for va, vb in zip(got[0][0], got[1][0]):
            assert same(va, vb)
        assert got[0][1] == got[1][1]
        assert got[0][2] == got[1][2]


@pytest.mark.skipif(not os.path.isdir(REFERENCE_DATA), reason="reference data not mounted")
def test_oracle_on_reference_netlib_fixtures(ref, orc):
    """The reference's small Netlib fixtures, read by path: the oracle reproduces the reference
    engine bit for bit and meets the published optima (data/netlib_small/optima.csv) to 1e-6."""
    base = os.path.join(REFERENCE_DATA, "netlib_small")
    optima = {}
    for line in open(os.path.join(base, "optima.csv")).read().splitlines()[1:]:
        f = line.split(",")
        optima[f[0]] = float(f[3])
    for name in lps.NETLIB:
        lp = lps.read_lpm(os.path.join(base, name + ".lpm"))
        r = ref.solve(lp, presolve=False)
        o = orc.solve(lp)
        assert o.status == r.status == "Optimal", name
        assert o.iterations == r.iterations, name
        assert same(o.x, r.x), name
        assert abs(o.objective - optima[name]) <= 1e-6 * (1 + abs(optima[name])), name
