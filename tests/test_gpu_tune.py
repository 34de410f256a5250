"""The autotuner on the GPU: every launch variant of the fused iteration kernels (forced with
PS26119_SLAB_VARIANT) gives a bit-identical exact-mode trajectory — the variants change only how
many gathers are in flight and how many blocks share an SM, never the order of a sum — and an
untuned run records the variants it picked."""
import os

import numpy as np
import pytest

import ps26119
from ps26119 import generators as g

pytestmark = pytest.mark.gpu

NUM_VARIANTS = 7  # kSlabVariants in csrc/spmv.cuh


def solve(lp, exact=True, precision="fp64"):
    return ps26119.solve_lp(lp.c, (lp.col_start, lp.row_index, lp.value), lp.row_lower, lp.row_upper, lp.col_lower,
                            lp.col_upper, sense=lp.sense, offset=lp.offset, algorithm="r2hpdhg", precision=precision,
                            engine={"presolve": False, "exact": exact})


@pytest.mark.parametrize("name", ["random", "staircase"])
def test_every_variant_gives_the_same_bits(name, monkeypatch):
    lp = g.random_lp(3000, seed=3) if name == "random" else g.staircase_lp(6, seed=2)
    runs = []
    for k in range(NUM_VARIANTS):
        monkeypatch.setenv("PS26119_SLAB_VARIANT", str(k))
        r = solve(lp)
        st = ps26119.last_stats()
        assert st["slab_variant_primal"] == k and st["slab_variant_dual"] == k and st["tuned"] == 0
        runs.append(r)
    base = runs[0]
    assert base.status == ps26119.OPTIMAL, base.message
    for r in runs[1:]:
        assert r.status == base.status and r.iterations == base.iterations
        assert np.array_equal(r.x, base.x) and np.array_equal(r.y, base.y) and r.objective == base.objective


def test_tuner_measures_once_per_shape_class(monkeypatch):
    monkeypatch.delenv("PS26119_SLAB_VARIANT", raising=False)
    monkeypatch.delenv("PS26119_AUTOTUNE", raising=False)
    lp = g.random_lp(20000, seed=9)  # a shape class no other test uses
    a = solve(lp, exact=False)
    sa = ps26119.last_stats()
    b = solve(lp, exact=False)
    sb = ps26119.last_stats()
    assert sa["tuned"] == 1 and sb["tuned"] == 0  # the second solve reuses the choice
    assert 0 <= sa["slab_variant_primal"] < NUM_VARIANTS and 0 <= sa["slab_variant_dual"] < NUM_VARIANTS
    assert (sb["slab_variant_primal"], sb["slab_variant_dual"]) == (sa["slab_variant_primal"], sa["slab_variant_dual"])
    assert a.iterations == b.iterations and np.array_equal(a.x, b.x)
