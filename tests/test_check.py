"""The in-process optimality check and the certified bound on the host (csrc/solver.cpp
check_solution, csrc/certify.cpp certified_dual_bound) against the reference's
(src/core/solution_checker.cpp:61-133, src/core/safe_bound.cpp:178), on the CPU: both read the
same model file and take the same point; every reported value must be bit-identical. The large
models run the threaded passes (row activity by row block, reduced costs by column range)."""
import subprocess

import numpy as np

from ps26119 import generators as g
from test_io import write_mps
from test_presolve import GENERATED


def _points(lp, rng):
    """Points of three kinds: random, on the bounds (complementary), and slightly off them."""
    n, m = lp.num_cols, lp.num_rows
    lo, up = lp.col_lower, lp.col_upper
    base = np.where(np.isfinite(lo), lo, np.where(np.isfinite(up), up, 0.0))
    yield rng.normal(size=n) * 3, rng.normal(size=m)
    yield base.copy(), rng.normal(size=m) * 1e-3
    yield base + rng.normal(size=n) * 1e-7, rng.normal(size=m)


def test_check_and_bound_match_reference(ref, tmp_path, host_probe):
    _compare(ref, tmp_path, host_probe)


def test_check_without_row_buckets(ref, tmp_path, host_probe_no_buckets):
    # above the bucketing limit the row activity is one sequential pass; same bits
    _compare(ref, tmp_path, host_probe_no_buckets)


def _compare(ref, tmp_path, host_probe):
    rng = np.random.default_rng(21)
    models = {name: GENERATED[name]() for name in ("planted_0", "planted_3", "columns_only_1", "staircase_T3",
                                                     "infeasible_empty_row")}
    models["random_m50000"] = g.random_lp(50_000, seed=9)
    models["planted_sparse"] = GENERATED["planted_sparse"]()
    args, want, names = [], [], []
    for k, (name, lp) in enumerate(models.items()):
        path = str(tmp_path / f"{name}.mps")
        write_mps(lp, path)
        for q, (x, y) in enumerate(_points(lp, rng)):
            fx, fy = tmp_path / f"{k}_{q}_x.bin", tmp_path / f"{k}_{q}_y.bin"
            x.tofile(fx), y.tofile(fy)
            args += [path, str(fx), str(fy)]
            w = ref.check_file(path, x, y)
            assert w is not None, name
            want.append(w)
            names.append((name, q))
    out = tmp_path / "out.bin"
    r = subprocess.run([host_probe, "check", str(out), *args], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    got = np.fromfile(out, dtype=np.float64).reshape(-1, 7)
    assert len(got) == len(want)
    labels = ("passed", "primal", "dual", "gap", "primal_objective", "dual_objective", "certified_bound")
    for (name, q), w, o in zip(names, want, got):
        for f, label in enumerate(labels):
            assert np.array([o[f]]).view(np.uint64)[0] == np.array([w[f]]).view(np.uint64)[0] or \
                (np.isnan(o[f]) and np.isnan(w[f])), (name, q, label, o[f], w[f])


def test_original_kkt_matches_reference(ref, tmp_path, host_probe):
    """original_kkt (csrc/solver.cpp), the presolve wrapper's test of a postsolved point, against
    the reference's (src/core/solve.cpp:77-84 over pdhg::kkt_general): the 8 statistics bit for
    bit and converged() at three tolerances, on the same model files and points; the large
    models run the threaded form."""
    rng = np.random.default_rng(33)
    models = {name: GENERATED[name]() for name in ("planted_1", "columns_only_0", "staircase_T3")}
    models["random_m50000"] = g.random_lp(50_000, seed=10)
    models["planted_sparse"] = GENERATED["planted_sparse"]()
    args, want, names = [], [], []
    for k, (name, lp) in enumerate(models.items()):
        path = str(tmp_path / f"{name}.mps")
        write_mps(lp, path)
        points = list(_points(lp, rng))
        if name in ("staircase_T3", "columns_only_0"):  # the reference's own 1e-8 solution: converged
            s = ref.solve(lp, tol=1e-8, iteration_limit=200_000)  # at 1e-4 and 1e-8, not at 1e-9
            assert s.status == "Optimal", (name, s.status)
            points.append((s.x, s.y))
        for q, (x, y) in enumerate(points):
            fx, fy = tmp_path / f"{k}_{q}_x.bin", tmp_path / f"{k}_{q}_y.bin"
            x.tofile(fx), y.tofile(fy)
            args += [path, str(fx), str(fy)]
            stats = [ref.kkt_file(path, x, y, eps) for eps in (1e-4, 1e-8, 1e-9)]
            assert stats[0] is not None, name
            want.append(np.concatenate([stats[0][:8], [s[8] for s in stats]]))
            names.append((name, q))
    out = tmp_path / "kkt.bin"
    r = subprocess.run([host_probe, "kkt", str(out), *args], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    got = np.fromfile(out, dtype=np.float64).reshape(-1, 11)
    assert len(got) == len(want)
    for (name, q), w, o in zip(names, want, got):
        assert np.array_equal(o.view(np.uint64), w.view(np.uint64)), (name, q, o, w)
    assert {tuple(w[8:]) for w in want} >= {(0.0, 0.0, 0.0), (1.0, 1.0, 0.0)}  # both outcomes seen
