"""GPU backend ops against the reference CPU backend, op by op (the check the reference's
tests/unit/test_gpu.cpp:33-95 performs on its CUDA backend), through the C ABI
(include/ps26119_backend.h).

Bar: element-wise ops and CSR products are BIT-IDENTICAL in fp64 and fp32 (same operation
order, no FMA contraction); reductions are bit-identical in exact mode and within 1e-12
relative in fast mode (fixed-order trees)."""
import numpy as np
import pytest

import lps
import ps26119
from ps26119 import generators as g

pytestmark = pytest.mark.gpu


def checker():
    """The reference library where it was built, else the C oracle (identical by test)."""
    import reference
    if reference.available():
        return "reference", reference
    import oracle
    return "oracle", oracle


def cpu_backend(lp):
    kind, mod = checker()
    return mod.Backend(lp) if kind == "reference" else mod.Backend(mod.Scaled(lp))


MODELS = {"mixed_rows": lps.mixed_rows, "random_m200": lambda: g.random_lp(200, seed=3),
          "staircase_T3": lambda: g.staircase_lp(3), "long_row": lps.long_row}


def scaled_of(cpu, which):
    return cpu.scaled(which) if hasattr(cpu, "scaled") else cpu.scaled.get(which)


@pytest.mark.parametrize("exact", [True, False])
@pytest.mark.parametrize("name", sorted(MODELS))
def test_scaled_problem_is_bit_identical(name, exact):
    lp = MODELS[name]()
    gpu = ps26119.Backend(lp, exact=exact)
    kind, mod = checker()
    cpu = mod.Backend(lp) if kind == "reference" else mod.Scaled(lp)
    get = (lambda w: cpu.scaled(w)) if kind == "reference" else (lambda w: cpu.get(w))
    for which in range(9):
        a, b = gpu.scaled(which), get(which)
        if exact or which in (0, 1, 7, 8):
            assert np.array_equal(a, b), which
        else:  # c̃ and the bounds carry the bound/objective scalars, tree sums in fast mode
            fin = np.isfinite(b)
            assert np.array_equal(fin, np.isfinite(a)) and np.array_equal(a[~fin], b[~fin])
            assert np.all(np.abs(a[fin] - b[fin]) <= 1e-14 * np.maximum(1.0, np.abs(b[fin]))), which
    if kind == "reference":
        for which in (0, 1):
            rp, col = gpu.structure(which)
            rrp, rcol = cpu.structure(which)
            assert np.array_equal(rp, rrp) and np.array_equal(col, rcol)
    s_gpu, s_cpu = gpu.scalars(), cpu.scalars()
    if exact:
        assert s_gpu == s_cpu
    else:  # ‖b̃‖, ‖c̃‖ are tree sums in fast mode
        for k in s_cpu:
            assert abs(s_gpu[k] - s_cpu[k]) <= 1e-13 * max(1.0, abs(s_cpu[k])), k
    est_cpu = cpu.norm2_estimate() if kind == "reference" else cpu.norm2()
    est_gpu = gpu.norm2_estimate()
    if exact:
        assert est_gpu == est_cpu
    else:
        assert abs(est_gpu - est_cpu) <= 1e-10 * est_cpu


def run_ops(b, lp):
    """The op sequence of the reference's Gpu.BackendOpsMatchCpu (test_gpu.cpp:52-79)."""
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
    return vecs, [b.dot(x, xh), b.norm2(y), b.diff_norm2(x, x0)], b.kkt(xh, yh)


@pytest.mark.parametrize("exact", [True, False])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("name", sorted(MODELS))
def test_backend_ops_match_reference(name, precision, exact):
    lp = MODELS[name]()
    cpu = cpu_backend(lp)
    gpu = ps26119.Backend(lp, exact=exact)
    for b in (cpu, gpu):
        b.set_precision(precision == "mixed")
    vc, sc, kc = run_ops(cpu, lp)
    vg, sg, kg = run_ops(gpu, lp)
    for k, (a, b) in enumerate(zip(vc, vg)):
        if exact:
            assert np.array_equal(a, b), f"vector {k}"
        else:  # the scaled vectors carry ‖b̃‖, ‖c̃‖ from tree sums: last-bit differences grow over 20 steps
            tol = 1e-5 if precision == "mixed" else 1e-11
            assert np.all(np.abs(a - b) <= tol * (1 + np.abs(a))), f"vector {k}"
    if exact:
        assert sc == sg
        assert kc == kg
    else:
        tol = 1e-5 if precision == "mixed" else 1e-10
        for a, b in zip(sc, sg):
            assert abs(a - b) <= tol * max(1.0, abs(a))
        for key in kc:
            assert abs(kc[key] - kg[key]) <= tol * max(1.0, abs(kc[key])), key


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_fused_kernels_equal_unfused_sequence(precision):
    """Ãᵀy + r2h_primal fused in one kernel equals spmv_t then r2h_primal, bit for bit."""
    lp = g.random_lp(500, seed=5)
    results = []
    for fused in (False, True):
        b = ps26119.Backend(lp, exact=True)
        b.set_precision(precision == "mixed")
        x, x0, xh, xb, gg = (b.create(False) for _ in range(5))
        y, y0, yh, yb, ax = (b.create(True) for _ in range(5))
        b.upload(x, np.sin(0.5 + np.arange(lp.num_cols)))
        b.upload(y, np.cos(1.5 + np.arange(lp.num_rows)))
        b.copy(x0, x)
        b.copy(y0, y)
        for it in range(30):
            w = (it + 1.0) / (it + 2.0)
            if fused:
                b.fused_primal(y, x, x0, 0.25, w, 1.0, xh, xb)
                b.fused_dual(xb, y, y0, 0.35, w, 1.0, yh, yb)
            else:
                b.spmv_t(y, gg)
                b.r2h_primal(x, x0, gg, 0.25, w, 1.0, xh, xb)
                b.spmv(xb, ax)
                b.r2h_dual(y, y0, ax, 0.35, w, 1.0, yh, yb)
        results.append([b.download(v) for v in (x, xh, xb, y, yh, yb)])
    for a, b in zip(*results):
        assert np.array_equal(a, b)


def test_long_rows_match_reference():
    """A 3000-entry row and a 1500-entry column (reference test_gpu.cpp:128-188)."""
    lp = lps.long_row()
    cpu, gpu = cpu_backend(lp), ps26119.Backend(lp, exact=True)
    for precision in ("fp64", "mixed"):
        outs = []
        for b in (cpu, gpu):
            b.set_precision(precision == "mixed")
            x, gg = b.create(False), b.create(False)
            y, ax = b.create(True), b.create(True)
            b.upload(x, np.sin(0.1 * np.arange(lp.num_cols)))
            b.upload(y, np.cos(0.3 * np.arange(lp.num_rows)))
            b.spmv(x, ax)
            b.spmv_t(y, gg)
            outs.append((b.download(ax), b.download(gg)))
        assert np.array_equal(outs[0][0], outs[1][0]) and np.array_equal(outs[0][1], outs[1][1])
