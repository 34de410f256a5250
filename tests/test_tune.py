"""The autotuner's host logic (csrc/tune.hpp): tests/native/tune_check.cpp, compiled here, checks
the variant picked from measured times, the shape classes, the environment switches and the
process cache. CPU only; the GPU side (every variant gives the same bits) is in
tests/test_gpu_tune.py."""
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_tuner_selection_logic(tmp_path):
    exe = str(tmp_path / "tune_check")
    src = os.path.join(ROOT, "tests", "native", "tune_check.cpp")
    csrc = os.path.join(ROOT, "ps26119-solver_b200", "csrc")
    r = subprocess.run(["g++", "-O2", "-std=c++17", "-I", csrc, src, "-o", exe], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([exe], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stdout + r.stderr
