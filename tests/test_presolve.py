"""Presolve R1-R4 (csrc/solver.cpp presolve) against the reference's own presolve
(src/core/presolve.cpp:22-156, run from oracle/_ref), on the CPU. Both sides read the same model
file and digest every decision presolve makes: outcome, counts, row and column maps, fixed
values, the singleton records in order, and the reduced model's fingerprint. `ps26119 info`
prints the library's digest, reference.presolve_file the reference's. Equal digests mean the
reduced model the engine solves and the postsolve data are the reference's, bit for bit."""
import glob
import os
import subprocess

import numpy as np
import pytest

from ps26119 import generators as g
from conftest import REFERENCE_DATA
from test_io import cli, write_mps


def our_presolve(path):
    r = cli("info", path)
    assert r.returncode == 0, r.stdout + r.stderr
    lines = [ln for ln in r.stdout.splitlines() if "presolve digest" in ln]
    return lines[0].split()[-1] if lines else None, r.stdout


def planted(seed):
    """A small LP with every reduction planted: empty rows (feasible), empty columns (finite
    and infinite best bounds, zero cost), fixed columns, and singleton rows that tighten lower
    and upper bounds, some of them chained through columns that the reductions empty."""
    rng = np.random.default_rng(seed)
    m, n = 40, 30
    A = np.where(rng.random((m, n)) < 0.15, rng.normal(size=(m, n)), 0.0)
    A[[3, 17, 29], :] = 0.0                       # empty rows
    A[:, [2, 11, 25]] = 0.0                       # empty columns
    for i, j in ((5, 7), (8, 12), (21, 4), (33, 19), (36, 7)):   # singleton rows
        A[i, :] = 0.0
        A[i, j] = rng.choice([-1.0, 1.0]) * rng.uniform(0.5, 2.0)
    x0 = rng.uniform(0.5, 4.0, n)
    ax = A @ x0
    rl, ru = ax - rng.uniform(0, 1, m), ax + rng.uniform(0, 1, m)
    rl[[7, 15]] = -np.inf
    ru[[9, 22]] = np.inf
    rl[[3, 17]], ru[[3, 17]] = -1.0, 2.0          # 0 inside: removable
    rl[29], ru[29] = 0.0, 0.0
    cl, cu = np.zeros(n), np.full(n, 6.0)
    cu[[1, 9]] = np.inf
    cl[[6, 14, 27]] = cu[[6, 14, 27]] = x0[[6, 14, 27]]   # fixed columns
    c = rng.normal(size=n)
    c[2], c[11], c[25] = 1.0, -1.0, 0.0           # empty columns: lower, upper, zero cost
    cu[11] = np.inf                                # best bound infinite: kept
    return g.from_dense(c, A, rl, ru, cl, cu, offset=1.5)


def infeasible_empty_row():
    lp = planted(7)
    rl, ru = lp.row_lower.copy(), lp.row_upper.copy()
    rl[3], ru[3] = 1.0, 2.0  # an empty row that excludes 0
    return lp.with_data(row_lower=rl, row_upper=ru)


def columns_only(seed, m=50, n=40):
    """Fixed and empty columns only: every row keeps at least three entries in the kept
    columns, so no row is removed and the reduced matrix is the kept columns copied as they
    are (the case of large random LPs, whose empty columns are the only reduction)."""
    rng = np.random.default_rng(seed)
    A = np.where(rng.random((m, n)) < 0.3, rng.normal(size=(m, n)), 0.0)
    fixed, empty = [3, 8, n - 7], [5, n - 10, n - 1]
    A[:, empty] = 0.0
    kept = [j for j in range(n) if j not in fixed and j not in empty]
    for i in range(m):
        for j in kept[i % 7::7][:3]:
            if A[i, j] == 0.0:
                A[i, j] = rng.choice([-1.0, 1.0]) * rng.uniform(0.5, 2.0)
    x0 = rng.uniform(0.5, 4.0, n)
    ax = A @ x0
    rl, ru = ax - rng.uniform(0, 1, m), ax + rng.uniform(0, 1, m)
    cl, cu = np.zeros(n), np.full(n, 6.0)
    cl[fixed] = cu[fixed] = x0[fixed]
    c = rng.normal(size=n)
    c[empty] = [1.0, -1.0, 0.0]
    return g.from_dense(c, A, rl, ru, cl, cu, offset=-0.5)


def planted_sparse(seed, m=70_000):
    """A random sparse LP large enough for the threaded presolve passes (about 420,000 entries),
    with empty rows, singleton rows (equalities among them, which fix their column and start
    chains) and fixed columns planted in it."""
    base = g.random_lp(m, seed=seed)
    rng = np.random.default_rng(seed + 100)
    n = base.num_cols
    cols = np.repeat(np.arange(n), np.diff(base.col_start))
    rows, vals = base.row_index.astype(np.int64), base.value.copy()
    empty = rng.choice(m, 60, replace=False)
    single = rng.choice(np.setdiff1d(np.arange(m), empty), 300, replace=False)
    keep = ~np.isin(rows, empty)
    first = {}  # a singleton row keeps its entry of smallest column
    for k in np.nonzero(np.isin(rows, single))[0]:
        first.setdefault(int(rows[k]), k)
    keep &= ~np.isin(rows, single) | np.isin(np.arange(len(rows)), list(first.values()))
    rows, cols, vals = rows[keep], cols[keep], vals[keep]
    x0 = base.meta["x0"]
    b = np.bincount(rows, weights=vals * x0[cols], minlength=m)
    rl, ru = b.copy(), b.copy()
    rl[empty], ru[empty] = -1.0, 2.0
    loose = single[:150]  # half the singletons are inequalities that tighten one bound
    rl[loose] = b[loose] - np.abs(b[loose]) * 0.5 - 0.1
    ru[loose] = np.inf
    cl, cu = base.col_lower.copy(), base.col_upper.copy()
    fixed = rng.choice(n, 100, replace=False)
    cl[fixed] = cu[fixed] = x0[fixed]
    cs, ri, v = g.csc_from_triplets(m, n, rows, cols, vals)
    return base.with_data(row_lower=rl, row_upper=ru, col_lower=cl, col_upper=cu, col_start=cs, row_index=ri,
                          value=v, name="planted-sparse")


GENERATED = {
    **{f"planted_{s}": (lambda s=s: planted(s)) for s in range(6)},
    **{f"columns_only_{s}": (lambda s=s: columns_only(s)) for s in range(2)},
    "columns_only_large": lambda: columns_only(5, m=400, n=300),
    "planted_sparse": lambda: planted_sparse(3),
    "random_m70000": lambda: g.random_lp(70_000, seed=6),  # empty columns only, threaded copy
    "infeasible_empty_row": infeasible_empty_row,
    "random_m300": lambda: g.random_lp(300, seed=4),
    "staircase_T3": lambda: g.staircase_lp(3, seed=2),
}


@pytest.mark.parametrize("name", sorted(GENERATED))
def test_presolve_decisions_match_reference(ref, tmp_path, name):
    lp = GENERATED[name]()
    path = tmp_path / f"{name}.mps"
    write_mps(lp, path)
    want, counts = ref.presolve_file(str(path))
    got, out = our_presolve(str(path))
    assert want is not None, counts
    assert got == want, (counts, out)


def test_planted_models_exercise_every_rule(ref, tmp_path):
    seen = set()
    for s in range(6):
        path = tmp_path / f"p{s}.mps"
        write_mps(planted(s), path)
        _, (outcome, rows, cols, tightened) = ref.presolve_file(str(path))
        seen.add(outcome)
        assert rows >= 3 + 5 and cols >= 2 + 3 and tightened >= 1  # one empty column is kept (infinite bound)
    path = tmp_path / "inf.mps"
    write_mps(infeasible_empty_row(), path)
    seen.add(ref.presolve_file(str(path))[1][0])
    assert seen == {0, 1}


def _reference_files():
    if not os.path.isdir(REFERENCE_DATA):
        return []
    out = []
    for d in ("netlib_small", "examples", "hand"):
        out += sorted(glob.glob(os.path.join(REFERENCE_DATA, d, "*.mps")) +
                      glob.glob(os.path.join(REFERENCE_DATA, d, "*.lpm")))
    return out


@pytest.mark.parametrize("path", _reference_files(), ids=lambda p: os.path.relpath(p, REFERENCE_DATA))
def test_presolve_on_reference_data_files(ref, path):
    want, info = ref.presolve_file(path)
    got, out = our_presolve(path)
    if want is None:
        assert got is None
    else:
        assert got == want, (info, out)


def test_presolve_without_host_buffer_reuse(ref, tmp_path):
    # PS26119_HOST_REUSE_MB=0: presolve frees its scratch after every call; the decisions are
    # the same as with the buffers kept
    path = tmp_path / "p.mps"
    write_mps(planted(3), path)
    want, _ = ref.presolve_file(str(path))
    from test_io import CLI
    env = dict(os.environ, PS26119_HOST_REUSE_MB="0")
    r = subprocess.run([CLI, "info", str(path)], capture_output=True, text=True, env=env, timeout=120)
    got = [ln for ln in r.stdout.splitlines() if "presolve digest" in ln][0].split()[-1]
    assert r.returncode == 0 and got == want


def test_columns_only_models_remove_no_rows(ref, tmp_path):
    for name in ("columns_only_0", "columns_only_1", "columns_only_large"):
        path = tmp_path / f"{name}.mps"
        write_mps(GENERATED[name](), path)
        _, (outcome, rows, cols, _) = ref.presolve_file(str(path))
        assert outcome == 0 and rows == 0 and cols >= 3, (name, outcome, rows, cols)


def test_presolve_reuses_its_result_across_models(ref, tmp_path):
    # One process presolves a sequence of models into one reused result, the way repeated solves
    # on a thread do: larger and smaller models, reductions with and without removed rows, an
    # unchanged and an infeasible model in between. Every digest equals the reference's.
    order = ["columns_only_large", "planted_0", "columns_only_0", "infeasible_empty_row", "columns_only_1",
             "random_m300", "planted_4", "staircase_T3", "columns_only_large", "planted_0"]
    paths, want = [], []
    for k, name in enumerate(order):
        path = tmp_path / f"{k}_{name}.mps"
        write_mps(GENERATED[name](), path)
        paths.append(str(path))
        want.append(ref.presolve_file(str(path))[0])
    r = cli("info", *paths)
    assert r.returncode == 0, r.stdout + r.stderr
    got = [ln.split()[-1] for ln in r.stdout.splitlines() if "presolve digest" in ln]
    assert got == want, list(zip(order, got, want))


def _read_probe(path, count):
    raw = open(path, "rb").read()
    out, at = [], 0
    for _ in range(count):
        sizes = np.frombuffer(raw, dtype=np.int64, count=3, offset=at)
        at += 24
        if sizes[0] < 0:
            out.append(None)
            continue
        vecs = []
        for s in sizes:
            vecs.append(np.frombuffer(raw, dtype=np.float64, count=int(s), offset=at))
            at += 8 * int(s)
        obj = float(np.frombuffer(raw, dtype=np.float64, count=1, offset=at)[0])
        at += 8
        out.append((*vecs, obj))
    assert at == len(raw)
    return out


def _same_bits(a, b):
    return a.shape == b.shape and np.array_equal(np.asarray(a).view(np.uint64), np.asarray(b).view(np.uint64))


def test_postsolve_matches_reference(ref, tmp_path, host_probe):
    """postsolve (csrc/solver.cpp) against the reference's (src/core/presolve.cpp:158-193) on the
    same presolved models and seeded reduced points: x, y, z and the objective bit for bit. The
    points include ones without x or without y (postsolve then clears what depends on them).
    The jobs run in one process with one reused presolve result, as repeated solves do, and the
    two large LPs run the threaded passes."""
    rng = np.random.default_rng(11)
    models = {name: GENERATED[name]() for name in ("planted_0", "planted_2", "planted_5", "columns_only_0",
                                                     "columns_only_large", "staircase_T3")}
    models["random_m50000"] = g.random_lp(50_000, seed=8)
    models["planted_sparse"] = GENERATED["planted_sparse"]()
    args, want, names = [], [], []
    for k, (name, lp) in enumerate(models.items()):
        path = str(tmp_path / f"{name}.mps")
        write_mps(lp, path)
        _, (outcome, rows, cols, _) = ref.presolve_file(path)
        assert outcome == 0, name
        m, n = lp.num_rows - rows, lp.num_cols - cols
        for variant in ("xy", "x", "y"):
            rx = rng.normal(size=n) if "x" in variant else np.zeros(0)
            ry = rng.normal(size=m) * 3 if "y" in variant else np.zeros(0)
            fx, fy = tmp_path / f"{k}_{variant}_x.bin", tmp_path / f"{k}_{variant}_y.bin"
            rx.tofile(fx), ry.tofile(fy)
            args += [path, str(fx), str(fy)]
            want.append(ref.postsolve_file(path, lp.num_rows, lp.num_cols, rx, ry))
            names.append((name, variant))
    out = tmp_path / "out.bin"
    r = subprocess.run([host_probe, "postsolve", str(out), *args], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    got = _read_probe(out, len(want))
    for (name, variant), w, o in zip(names, want, got):
        assert w is not None and o is not None, (name, variant)
        for q, label in enumerate(("x", "y", "z")):
            assert _same_bits(o[q], w[q]), (name, variant, label)
        assert _same_bits(np.array([o[3]]), np.array([w[3]])) or (np.isnan(o[3]) and np.isnan(w[3])), (name, variant)


def test_presolve_without_row_buckets(ref, tmp_path, host_probe_no_buckets):
    # above the bucketing limit the row counts and XORs take relaxed integer atomics instead;
    # a probe built with a 4,096-entry limit runs that form on the large models
    names = ["planted_sparse", "random_m70000", "planted_2"]
    paths = []
    for name in names:
        path = str(tmp_path / f"{name}.mps")
        write_mps(GENERATED[name](), path)
        paths.append(path)
    out = tmp_path / "digests.txt"
    r = subprocess.run([host_probe_no_buckets, "digest", str(out), *paths], capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr
    got = open(out).read().split()
    assert got == [ref.presolve_file(p)[0] for p in paths]


def test_presolve_same_on_one_host_thread(ref, tmp_path):
    # PS26119_HOST_THREADS=1 runs every host pass on the calling thread: the decisions are the
    # same as with the threaded passes
    from test_io import CLI
    paths = []
    for name in ("planted_sparse", "random_m70000"):
        path = tmp_path / f"{name}.mps"
        write_mps(GENERATED[name](), path)
        paths.append(str(path))
    for threads in ("1", "3"):
        env = dict(os.environ, PS26119_HOST_THREADS=threads)
        r = subprocess.run([CLI, "info", *paths], capture_output=True, text=True, env=env, timeout=300)
        assert r.returncode == 0, r.stderr
        got = [ln.split()[-1] for ln in r.stdout.splitlines() if "presolve digest" in ln]
        assert got == [ref.presolve_file(p)[0] for p in paths], threads
