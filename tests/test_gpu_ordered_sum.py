"""The engine's reference-order sums (ps26119_ordered_sum, the kernels behind every exact-mode
reduction) against the sequential evaluation they must reproduce bit for bit.

The reference sums its KKT statistics, objectives and checker terms in plain host loops
(s = init; s += t[i], e.g. pdhg::kkt_general, src/pdhg/cpu_backend.cpp:226-284) and its dots in
la::parallel_sum's 64 ordered chunks (src/la/parallel.h:169-188). numpy's add.accumulate walks an
array in order with one rounding per addition, so it is the oracle here. The inputs are chosen to
break a parallel evaluation: ties at the partial sum's last bit, binade crossings, cancellation
to zero, signed zeros, subnormals, infinities and NaN, and every small length around the
kernels' window (256) and tile (2048) sizes.
"""
import numpy as np
import pytest

import ps26119

pytestmark = pytest.mark.gpu


def seq(t, init):
    return float(np.add.accumulate(np.concatenate([[init], t]))[-1])


def chunk64(t, init):
    n = len(t)
    chunks = min(64, max(1, n))
    parts = [seq(t[n * c // chunks:n * (c + 1) // chunks], 0.0) for c in range(chunks)]
    return seq(np.array(parts), init)


def same(a, b):
    return (np.isnan(a) and np.isnan(b)) or (a == b and np.signbit(a) == np.signbit(b))


def gpu_sum(t, init, order, exact=True):
    import torch
    d = torch.as_tensor(np.ascontiguousarray(t, dtype=np.float64), device="cuda")
    torch.cuda.synchronize()
    return ps26119.ordered_sum(d.data_ptr(), len(t), init, order, exact)


def cases():
    rng = np.random.default_rng(2024)
    yield "normal_1e6", rng.standard_normal(1_000_003), 0.0
    yield "normal_init", rng.standard_normal(300_001), 1e3
    yield "squares_2.5e6", rng.standard_normal(2_500_000) ** 2, 0.0
    yield "uniform_pos", rng.uniform(0, 1, 1_500_000), 0.0
    mag = 10.0 ** rng.uniform(-300, 300, 200_000)
    yield "wide_exponents", mag * rng.choice([-1.0, 1.0], mag.size), 0.0
    yield "halves_at_2^52", rng.choice([0.5, -0.5, 1.5, -1.5, 2.5, 0.25, -0.75], 200_000), 1.5 * 2.0 ** 52
    yield "ones_at_2^53", np.ones(70_000), 2.0 ** 53
    walk = rng.choice([1.0, -1.0], 100_000)
    walk[::7] *= 1e-20
    yield "cancel_near_zero", walk, 0.0
    yield "exact_zero_sum", np.concatenate([np.arange(1, 5001, dtype=float), -np.arange(1, 5001, dtype=float)]), 0.0
    yield "negative_zeros", np.full(10_000, -0.0), -0.0
    yield "negative_zeros_pos_init", np.full(10_000, -0.0), 0.0
    yield "subnormals", rng.integers(-5, 6, 50_000) * 5e-324, 0.0
    yield "geometric", 1.0001 ** np.arange(100_000), 1e-10
    inf = rng.standard_normal(20_000)
    inf[12_345] = np.inf
    yield "one_inf", inf, 0.0
    nan = rng.standard_normal(20_000)
    nan[3] = np.inf
    nan[19_000] = -np.inf
    yield "inf_minus_inf", nan, 0.0
    big = rng.standard_normal(50_000) * 1e305
    yield "overflow", np.abs(big), 0.0
    yield "mixed_signs_large_init", rng.standard_normal(400_000) * 1e-3, -7.5e4


CASES = list(cases())


@pytest.mark.parametrize("order", ["seq", "chunk64"])
@pytest.mark.parametrize("name", [c[0] for c in CASES])
def test_exact_sum_is_the_sequential_evaluation(name, order):
    _, t, init = next(c for c in CASES if c[0] == name)
    want = seq(t, init) if order == "seq" else chunk64(t, init)
    got = gpu_sum(t, init, order)
    assert same(got, want), (name, order, got.hex() if np.isfinite(got) else got,
                             want.hex() if np.isfinite(want) else want)


@pytest.mark.parametrize("n", [0, 1, 2, 31, 32, 33, 255, 256, 257, 2047, 2048, 2049, 4095, 4096, 4097, 8191, 10_000])
def test_exact_sum_small_lengths(n):
    rng = np.random.default_rng(n)
    t = rng.standard_normal(n) * 10.0 ** rng.integers(-3, 4, n)
    for init in (0.0, 0.1, -3.0):
        assert same(gpu_sum(t, init, "seq"), seq(t, init))
        assert same(gpu_sum(t, init, "chunk64"), chunk64(t, init))


def test_fast_tree_is_close_and_deterministic():
    rng = np.random.default_rng(3)
    t = rng.standard_normal(2_000_000)
    a, b = gpu_sum(t, 0.0, "seq", exact=False), gpu_sum(t, 0.0, "seq", exact=False)
    assert a == b
    assert abs(a - seq(t, 0.0)) <= 1e-12 * np.abs(t).sum()
