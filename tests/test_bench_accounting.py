"""bench.py's byte accounting, on the CPU: the single-LP roofline numerator B_iter, and the batch
roofline, which must count Ã once per lockstep iteration plus the vectors of the slots still
running (finished scenarios leave the lockstep batch), so that it never reads above the HBM
peak because of slots that are no longer there."""
import os
import sys
from types import SimpleNamespace

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import bench  # noqa: E402


def test_single_lp_bytes_per_iteration():
    m, n, nnz = 1_000_000, 1_500_000, 6_000_000
    assert bench.bytes_per_iteration(m, n, nnz, 8, 8) == 318_000_000  # the fp64 figure of the design notes
    assert bench.bytes_per_iteration(m, n, nnz, 4, 4) == 2 * nnz * 8 + 4 * (m + n) + 4 * (9 * n + 7 * m)


def test_batch_roofline_counts_running_slots_only():
    m, n, nnz = 100, 150, 600
    lp = SimpleNamespace(num_rows=m, num_cols=n, nnz=nnz)
    its = [1000, 400, 250, 1000]  # scenarios finishing at different lockstep iterations
    res = [SimpleNamespace(iterations=k) for k in its]
    stats = {"spmv_kernel_ms": 2.0, "spmv_kernel_launches": 2 * max(its)}
    args = SimpleNamespace(precision="fp64", steps=1)
    out = bench.roofline_batch(lp, args, 0.5, [(res, stats)])
    total = max(its) * (2 * nnz * 12 + 4 * (m + n)) + sum(its) * 8 * (9 * n + 7 * m)
    assert abs(out["algorithmic_bytes"] * max(its) - total) <= 1e-6 * total
    assert abs(out["achieved"] - total / 2.0e-3 / 1e9) <= 1e-9 * out["achieved"]
    assert abs(out["kernel_us_per_iteration"] - 2.0e3 / max(its)) < 1e-12
    # with every slot running to the cap the mean equals the all-slots figure
    full = [SimpleNamespace(iterations=1000) for _ in its]
    out2 = bench.roofline_batch(lp, args, 0.5, [(full, stats)])
    assert out2["algorithmic_bytes"] == 2 * nnz * 12 + 4 * (m + n) + len(its) * 8 * (9 * n + 7 * m)
    assert out["algorithmic_bytes"] < out2["algorithmic_bytes"]
    # mixed precision: 4-byte values and vectors (a lower bound)
    mixed = bench.roofline_batch(lp, SimpleNamespace(precision="mixed", steps=1), 0.5, [(res, stats)])
    assert mixed["algorithmic_bytes"] < out["algorithmic_bytes"]
