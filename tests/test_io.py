"""Model files and the command-line tool (csrc/io.cpp, csrc/cli.cpp) against the reference's
readers (src/io/lpm_reader.cpp, mps_reader.cpp, run from oracle/_ref): the model read from a file
must have the reference reader's fingerprint (the FNV-1a hash of every number of the model,
src/core/model.cpp:53-85). CPU tests use the CLI's `info` and `convert` commands; the GPU tests
solve from files through ps26119_solve_mps and `ps26119 solve`."""
import glob
import os
import subprocess

import numpy as np
import pytest

import ps26119
from ps26119 import generators as g
import lps
from conftest import REFERENCE_DATA

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "ps26119-solver_b200", "lib", "ps26119")


def cli(*args):
    return subprocess.run([CLI, *map(str, args)], capture_output=True, text=True, timeout=600)


def our_fingerprint(path):
    r = cli("info", path)
    if r.returncode != 0:
        return None, r.stderr
    line = [ln for ln in r.stdout.splitlines() if "fingerprint" in ln][0]
    return line.split()[-1], r.stdout


def write_mps(lp, path, fixed=False, extras=None, name="GEN"):
    """A free- (or fixed-) format MPS file of an Lp; `extras` adds raw section lines."""
    extras = extras or {}
    def f(*fields):
        if not fixed:
            return " " + " ".join(fields)
        cols = [(1, 2), (4, 12), (14, 22), (24, 36), (39, 47), (49, 61)]
        out = ""
        for (a, b), v in zip(cols, fields):
            out = out.ljust(a) + v
        return out
    num = lambda v: repr(float(v))
    lines = [f"NAME          {name}"]
    if lp.sense < 0:
        lines += ["OBJSENSE", "    MAX"]
    lines.append("ROWS")
    lines.append(f("N", "COST"))
    kinds = []
    for i in range(lp.num_rows):
        lo, up = lp.row_lower[i], lp.row_upper[i]
        k = "E" if lo == up else ("L" if not np.isfinite(lo) else ("G" if not np.isfinite(up) else "R"))
        kinds.append(k)
        lines.append(f("E" if k == "E" else ("L" if k in "LR" else "G"), f"R{i}"))
    lines += extras.get("ROWS", [])
    lines.append("COLUMNS")
    lines += extras.get("COLUMNS_PRE", [])
    for j in range(lp.num_cols):
        if lp.c[j] != 0 or lp.col_start[j] == lp.col_start[j + 1]:  # every column appears once at least
            lines.append(f("", f"X{j}", "COST", num(lp.c[j])))
        for p in range(lp.col_start[j], lp.col_start[j + 1]):
            lines.append(f("", f"X{j}", f"R{lp.row_index[p]}", num(lp.value[p])))
    lines += extras.get("COLUMNS", [])
    lines.append("RHS")
    if lp.offset:
        lines.append(f("", "RHS", "COST", num(-lp.offset)))
    for i, k in enumerate(kinds):
        b = lp.row_lower[i] if k == "G" else lp.row_upper[i]
        if k == "E":
            b = lp.row_lower[i]
        if b != 0:
            lines.append(f("", "RHS", f"R{i}", num(b)))
    lines += extras.get("RHS", [])
    if "R" in kinds:
        lines.append("RANGES")
        for i, k in enumerate(kinds):
            if k == "R":
                lines.append(f("", "RNG", f"R{i}", num(lp.row_upper[i] - lp.row_lower[i])))
    lines.append("BOUNDS")
    for j in range(lp.num_cols):
        lo, up = lp.col_lower[j], lp.col_upper[j]
        if lo == up:
            lines.append(f("FX", "BND", f"X{j}", num(lo)))
            continue
        if not np.isfinite(lo) and not np.isfinite(up):
            lines.append(f("FR", "BND", f"X{j}"))
            continue
        if not np.isfinite(lo):
            lines.append(f("MI", "BND", f"X{j}"))
        elif lo != 0:
            lines.append(f("LO", "BND", f"X{j}", num(lo)))
        if np.isfinite(up):
            lines.append(f("UP", "BND", f"X{j}", num(up)))
    lines += extras.get("BOUNDS", [])
    lines.append("ENDATA")
    with open(path, "w") as fh:
        fh.write("\n".join(lines) + "\n")


def reference_files():
    if not os.path.isdir(REFERENCE_DATA):
        return []
    out = []
    for d in ("netlib_small", "examples", "hand"):
        out += sorted(glob.glob(os.path.join(REFERENCE_DATA, d, "*.mps")) +
                      glob.glob(os.path.join(REFERENCE_DATA, d, "*.lpm")))
    return out


@pytest.mark.parametrize("path", reference_files(), ids=lambda p: os.path.relpath(p, REFERENCE_DATA))
def test_reference_data_files_read_as_the_reference_reads_them(ref, path):
    want, info = ref.read_fingerprint(path)
    got, out = our_fingerprint(path)
    if want is None:
        assert got is None, f"the reference refused ({info}) but we read it"
    else:
        assert got == want, out


GENERATED = {
    "wyndor": lps.wyndor, "max_ranged": lps.max_ranged, "mixed_rows": lps.mixed_rows,
    "random_m60": lambda: g.random_lp(60, seed=3), "staircase_T2": lambda: g.staircase_lp(2, seed=1),
}


@pytest.mark.parametrize("fixed", [False, True])
@pytest.mark.parametrize("name", sorted(GENERATED))
def test_generated_mps_matches_reference_reader(ref, tmp_path, name, fixed):
    lp = GENERATED[name]()
    if lp.offset == 0:
        lp = lp.with_data(offset=2.5)
    path = tmp_path / f"{name}.mps"
    write_mps(lp, path, fixed=fixed)
    want, dims = ref.read_fingerprint(str(path))
    got, out = our_fingerprint(str(path))
    assert want is not None and got == want, out
    assert dims == (lp.num_rows, lp.num_cols, lp.nnz)


def test_mps_rules_match_reference(ref, tmp_path):
    # the format's corner rules: negative UP with default lower, MI/PL/BV, a second RHS set
    # (ignored), an extra N row (dropped), duplicate entries (summed), integer markers,
    # RANGES on E rows of both signs, comments
    lp = g.random_lp(20, seed=5)
    extras = {
        "ROWS": [" N  FREEROW"],
        "COLUMNS_PRE": ["    MARKER                 'MARKER'                 'INTORG'",
                        "    Y0        COST         1.5   R0           2.0",
                        "    Y0        FREEROW      7.0",
                        "    MARKER                 'MARKER'                 'INTEND'"],
        "COLUMNS": ["    X0        R1           0.25", "* a comment line"],
        "RHS": ["    RHS2      R0           99.0"],
        "BOUNDS": [" UP BND       X1           -3.0", " PL BND       X2", " BV BND       Y0",
                   " MI BND       X3"],
    }
    path = tmp_path / "rules.mps"
    write_mps(lp, path, extras=extras)
    text = open(path).read().replace("RHS\n", "RHS\n", 1)
    text = text.replace("BOUNDS\n", "RANGES\n    RNG       R2           4.0\n    RNG       R3           -2.0\nBOUNDS\n", 1) \
        if "RANGES" not in text else text
    open(path, "w").write(text)
    want, dims = ref.read_fingerprint(str(path))
    got, out = our_fingerprint(str(path))
    assert want is not None and got == want, out


@pytest.mark.parametrize("text", ["", "NAME X\nFOO\nENDATA\n", "NAME X\nROWS\n N COST\nCOLUMNS\n X0 NOROW 1.0\nENDATA\n"])
def test_unreadable_mps_is_refused_like_the_reference(ref, tmp_path, text):
    path = tmp_path / "bad.mps"
    path.write_text(text)
    want, _ = ref.read_fingerprint(str(path))
    got, _ = our_fingerprint(str(path))
    assert want is None and got is None
    assert cli("info", path).returncode == 3


def test_lpm_round_trip(tmp_path):
    lp = g.staircase_lp(2, seed=3)
    mps = tmp_path / "s.mps"
    write_mps(lp, mps)
    out = tmp_path / "s.lpm"
    assert cli("convert", mps, out).returncode == 0
    a, _ = our_fingerprint(str(mps))
    b, _ = our_fingerprint(str(out))
    assert a == b
    m = lps.read_lpm(str(out))
    assert m.num_rows == lp.num_rows and m.num_cols == lp.num_cols and m.nnz == lp.nnz


def test_cli_usage_errors():
    assert cli().returncode == 2
    assert cli("frobnicate").returncode == 2
    assert cli("solve").returncode == 2
    assert cli("solve", "x.mps", "--tol", "-1").returncode == 2
    assert cli("--version").stdout.startswith("ps26119")


def test_cli_refuses_an_unwritable_solution_file_before_solving(tmp_path):
    """Exit code 4 (write error) before the model is solved: a missing directory, a directory
    given as the file; a new file in a writable directory is accepted (the solve then runs)."""
    mps = tmp_path / "tiny.mps"
    mps.write_text("NAME TINY\nROWS\n N COST\n L LIM1\nCOLUMNS\n X1 COST 1.0 LIM1 1.0\nRHS\n RHS LIM1 4.0\n"
                   "BOUNDS\n UP BND X1 4.0\nENDATA\n")
    for out in (tmp_path / "missing" / "x.sol", tmp_path):
        r = cli("solve", mps, "--out", out)
        assert r.returncode == 4 and "cannot write the solution file" in r.stderr, (out, r.stderr)
        assert "status" not in r.stdout  # nothing was solved
    r = cli("solve", mps, "--out", tmp_path / "new.sol")
    assert r.returncode != 4 and "cannot write" not in r.stderr


# ------------------------------------------------------------------------------- GPU
def parse_sol(path):
    head, cols = {}, []
    with open(path) as fh:
        lines = fh.read().splitlines()
    assert lines[0] == "PS26119-SOLUTION 1"
    k = 1
    while k < len(lines) and not lines[k].startswith("COLUMNS") and lines[k] != "END":
        key, _, val = lines[k].partition(" ")
        head[key] = val
        k += 1
    if k < len(lines) and lines[k].startswith("COLUMNS"):
        n = int(lines[k].split()[1])
        cols = [float(lines[k + 1 + j].split()[1]) for j in range(n)]
    return head, np.array(cols)


@pytest.mark.gpu
def test_solve_mps_through_c_api_and_cli(ref, tmp_path):
    lp = g.random_lp(200, seed=8).with_data(offset=3.0)
    path = tmp_path / "m.mps"
    write_mps(lp, path)
    sol = tmp_path / "m.sol"
    r = ps26119.solve_mps(str(path), out=str(sol))
    direct = ps26119.solve_lp(lp.c, (lp.col_start, lp.row_index, lp.value), lp.row_lower, lp.row_upper,
                              lp.col_lower, lp.col_upper, offset=lp.offset, algorithm="r2hpdhg")
    assert r.status_name == "Optimal" and r.check == "PASS", r.message
    assert r.objective == direct.objective and r.iterations == direct.iterations
    head, x = parse_sol(str(sol))
    assert head["status"] == "Optimal" and head["model"] == ref.read_fingerprint(str(path))[0]
    assert abs(float(head["objective"]) - r.objective) <= 1e-12 * (1 + abs(r.objective))
    assert abs(lp.offset + lp.c @ x - r.objective) <= 1e-9 * (1 + abs(r.objective))
    out = tmp_path / "cli.sol"
    p = cli("solve", path, "--gpu", "--out", out)
    assert p.returncode == 0, p.stdout + p.stderr
    assert "status     Optimal" in p.stdout and "check      PASS" in p.stdout
    h2, _ = parse_sol(str(out))
    assert float(h2["objective"]) == r.objective


@pytest.mark.gpu
def test_cli_batch_writes_one_solution_per_scenario(tmp_path):
    lp = g.random_lp(100, seed=3)
    files = [tmp_path / "base.mps"]
    write_mps(lp, files[0])
    for k, s in enumerate(g.scenarios(lp, 3, seed=2)):
        f = tmp_path / f"s{k}.mps"
        write_mps(lp.with_data(c=s["obj"], row_lower=s["row_lower"], row_upper=s["row_upper"]), f)
        files.append(f)
    outdir = tmp_path / "out"
    outdir.mkdir()
    p = cli("batch", *files, "--out-dir", outdir)
    assert p.returncode == 0, p.stdout + p.stderr
    for k in range(3):
        head, _ = parse_sol(str(outdir / f"s{k}.sol"))
        assert head["status"] == "Optimal" and head["engine"] == "r2hpdhg-batch"
