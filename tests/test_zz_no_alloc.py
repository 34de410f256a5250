"""ps26119_dot_noalloc — the dot product that allocates no device memory (its scratch is a fixed
device array inside the library) — against the backend's dot (ps26119_backend_dot), which
allocates its own scratch. Collected last, and independent of the other tests' state."""
import ctypes

import numpy as np
import pytest

import ps26119
from ps26119 import generators as g

TOL = 1e-11  # relative, the tolerance the fast-mode backend op tests use
MAX_N = 1 << 21


def _noalloc(L, a_dev, b_dev, n, exact, out_dev):
    return L.ps26119_dot_noalloc(n, a_dev.data_ptr(), b_dev.data_ptr(), int(exact), out_dev.data_ptr(), None)


@pytest.mark.gpu
@pytest.mark.parametrize("exact", [True, False])
def test_noalloc_dot_matches_backend_dot_twice(exact):
    import torch
    lp = g.random_lp(3000, seed=11)  # n = 4500 columns
    n = lp.num_cols
    rng = np.random.default_rng(5)
    a, b = rng.standard_normal(n), rng.standard_normal(n)
    be = ps26119.Backend(lp, exact=exact)
    va, vb = be.create(False), be.create(False)
    be.upload(va, a)
    be.upload(vb, b)
    want = be.dot(va, vb)
    L = ps26119.load()
    da = torch.as_tensor(a, device="cuda")
    db = torch.as_tensor(b, device="cuda")
    out = torch.full((1,), np.nan, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    for _ in range(2):  # two calls in a row share the scratch
        out.fill_(np.nan)
        torch.cuda.synchronize()
        rc = _noalloc(L, da, db, n, exact, out)
        assert rc == 0, L.ps26119_backend_last_error().decode()
        torch.cuda.synchronize()
        got = float(out.item())
        assert abs(got - want) <= TOL * (1.0 + abs(want)), (got, want)
        if exact:
            assert got == want  # the reference order: bit for bit
    # once set up, calls take no device memory: the device's free memory does not move
    free_before = torch.cuda.mem_get_info()[0]
    for _ in range(3):
        assert _noalloc(L, da, db, n, exact, out) == 0
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free_before


@pytest.mark.gpu
def test_noalloc_dot_large_and_rejects_beyond_maximum():
    import torch
    L = ps26119.load()
    rng = np.random.default_rng(9)
    n = MAX_N
    a, b = rng.standard_normal(n), rng.standard_normal(n)
    da, db = torch.as_tensor(a, device="cuda"), torch.as_tensor(b, device="cuda")
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    assert _noalloc(L, da, db, n, True, out) == 0
    torch.cuda.synchronize()
    want = float(np.dot(a, b))
    assert abs(float(out.item()) - want) <= 1e-9 * (1.0 + float(np.abs(a * b).sum()))
    # one element beyond the scratch: rejected on the host, nothing launched
    rc = _noalloc(L, da, db, n + 1, True, out)
    assert rc == ps26119.INVALID_ARGUMENT
    assert "exceeds the no-alloc scratch maximum" in L.ps26119_backend_last_error().decode()
    assert L.ps26119_dot_noalloc(-1, None, None, 1, out.data_ptr(), None) == ps26119.INVALID_ARGUMENT
