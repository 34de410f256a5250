"""Generates tests/golden/reference_runs.json: the REFERENCE solver's own results (built from its
sources into oracle/_ref by oracle/Makefile) on the seeded synthetic LPs and the hand LPs of the
reference's unit tests. The GPU tests compare against these where the reference library is not
loadable, and the CPU tests pin the C oracle to them.

    python tests/golden/make_golden.py [--with-c1]

Each record: case, precision, presolve, status, iterations, objective / dual objective /
primal weight / certified bound (exact, as float.hex), the in-process check, sha256 of x, y, z,
and for small models x and y.
"""
import argparse
import hashlib
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [os.path.join(ROOT, "ps26119-solver_b200"), os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")]

import reference  # noqa: E402
import lps  # noqa: E402
from ps26119 import generators as g  # noqa: E402


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.float64).tobytes()).hexdigest()


def hexf(v):
    return float(v).hex()


def cases(with_c1):
    out = [("wyndor", lps.wyndor), ("mixed_rows", lps.mixed_rows), ("max_ranged", lps.max_ranged),
           ("long_row", lps.long_row), ("infeasible", lps.infeasible), ("unbounded", lps.unbounded),
           ("random_m100_s1", lambda: g.random_lp(100, seed=1)), ("random_m300_s1", lambda: g.random_lp(300, seed=1)),
           ("random_m1000_s2", lambda: g.random_lp(1000, seed=2)), ("staircase_T2_s1", lambda: g.staircase_lp(2)),
           ("staircase_T4_s1", lambda: g.staircase_lp(4)), ("staircase_T8_s1", lambda: g.staircase_lp(8))]
    if with_c1:
        out.append(("random_m10000_s1", lambda: g.random_lp(10000, seed=1)))
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--with-c1", action="store_true", help="also the 10k x 15k random LP (minutes)")
    ap.add_argument("--threads", type=int, default=8)
    a = ap.parse_args()
    records = []
    for name, make in cases(a.with_c1):
        lp = make()
        for precision in ("fp64", "mixed"):
            for presolve in (False, True):
                t = time.time()
                s = reference.solve(lp, presolve=presolve, precision=precision, threads=a.threads)
                rec = {"case": name, "precision": precision, "presolve": presolve, "status": s.status,
                       "iterations": s.iterations, "objective": hexf(s.objective),
                       "dual_objective": hexf(s.dual_objective), "primal_weight": hexf(s.primal_weight),
                       "check": s.check, "certified_bound": hexf(s.certified_bound), "message": s.message, "m": lp.num_rows, "n": lp.num_cols,
                       "nnz": lp.nnz, "x_sha256": digest(s.x), "y_sha256": digest(s.y), "z_sha256": digest(s.z),
                       "seconds": round(time.time() - t, 3)}
                if lp.num_rows + lp.num_cols <= 800:
                    rec["x"] = [hexf(v) for v in s.x]
                    rec["y"] = [hexf(v) for v in s.y]
                records.append(rec)
                print(name, precision, "presolve" if presolve else "engine", s.status, s.iterations, s.objective,
                      f"{time.time() - t:.1f}s", flush=True)
    with open(os.path.join(HERE, "reference_runs.json"), "w") as f:
        json.dump({"generator": "tests/golden/make_golden.py", "reference_threads": a.threads, "runs": records}, f,
                  indent=1)


if __name__ == "__main__":
    main()
