"""The host threading helpers (csrc/parallel.hpp) that the C API's model copy, presolve,
postsolve and the checks use: tests/native/parallel_copy_check.cpp, compiled here, checks
parallel_copy byte for byte against memcpy, that the worker pool behind parallel_ranges
covers every index once with concurrent callers, nested sections and a forked child, and that
parallel_tasks (the certified bound's pipelined sum) runs every task once and never deadlocks a
task that waits on work items others took. CPU only."""
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_parallel_copy_matches_memcpy(tmp_path):
    exe = str(tmp_path / "parallel_copy_check")
    src = os.path.join(ROOT, "tests", "native", "parallel_copy_check.cpp")
    csrc = os.path.join(ROOT, "ps26119-solver_b200", "csrc")
    r = subprocess.run(["g++", "-O2", "-std=c++17", "-I", csrc, src, "-o", exe, "-lpthread"], capture_output=True,
                       text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stdout + r.stderr
