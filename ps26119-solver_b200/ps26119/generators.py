"""Seeded synthetic LP generators for the workloads this engine is measured on.

Every generator returns an :class:`Lp` in the reference's model contract
(include/ps26119/model.h:18-46 of the reference): minimise/maximise ``c^T x + offset``
subject to ``row_lower <= A x <= row_upper`` and ``col_lower <= x <= col_upper``, with A in
CSC (``col_start`` n+1, ``row_index`` nnz, ``value`` nnz; int32 indices, float64 values;
infinity = ``numpy.inf``). Row indices are sorted inside each column.

Generators (sizes are parameters; the named configurations fix them):

* :func:`random_lp` — equality-constrained random LP, 6 nonzeros per row at distinct,
  uniformly drawn columns with N(0,1) values; x0 ~ U(0,1)^n, b = A x0; 0 <= x <= 10;
  y0 ~ N(0,1)^m and c = A^T y0 + z with z_j ~ U(0,1) on a random half of the columns.
  Feasible (x0) and bounded (box). ``random_lp(10_000)`` is the 10k x 15k case,
  ``random_lp(1_000_000)`` the 1M x 1.5M case.
* :func:`staircase_lp` — multi-period planning LP: T periods, each a 49 x 60 block with
  about 175 nonzeros including the linking entries (log-uniform magnitudes in [1e-2, 1e2], random signs), 30% equality
  rows, inventory-linking -1 entries coupling 5 columns of period t-1 to period t, column
  bounds [0, U(10, 1000)], row bounds built around an interior point x* (feasible by
  construction) with inequality slack proportional to a per-period demand
  U(50, 150) x (1 + 0.3 sin(2 pi h / 24)).
* :func:`scenarios` — K scenarios of a base LP whose objective and finite row bounds are
  multiplied element-wise by lognormal(0, sigma) factors. On the staircase LP this makes most
  scenarios infeasible (the equality rows' right-hand sides no longer agree with each other).
* :func:`feasible_scenarios` — K scenarios that stay feasible: the base's interior point x* is
  multiplied by lognormal(0, sigma) factors (clipped to the column bounds), the row bounds are
  rebuilt around it with the base's slacks times lognormal factors, and the objective is
  multiplied by lognormal factors.

All randomness comes from ``numpy.random.Generator(PCG64(seed))``.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

__all__ = ["Lp", "random_lp", "staircase_lp", "scenarios", "feasible_scenarios", "from_dense",
           "csc_from_triplets"]


@dataclass
class Lp:
    """One LP in the reference model contract (CSC matrix)."""

    num_rows: int
    num_cols: int
    c: np.ndarray
    col_lower: np.ndarray
    col_upper: np.ndarray
    row_lower: np.ndarray
    row_upper: np.ndarray
    col_start: np.ndarray
    row_index: np.ndarray
    value: np.ndarray
    sense: int = 1
    offset: float = 0.0
    name: str = ""
    meta: dict = field(default_factory=dict)

    @property
    def nnz(self) -> int:
        return int(self.col_start[-1])

    def row_activity(self, x: np.ndarray) -> np.ndarray:
        cols = np.repeat(np.arange(self.num_cols), np.diff(self.col_start))
        return np.bincount(self.row_index, weights=self.value * x[cols], minlength=self.num_rows)

    def with_data(self, **kw) -> "Lp":
        d = dict(self.__dict__)
        d.update(kw)
        return Lp(**d)


def csc_from_triplets(m: int, n: int, rows: np.ndarray, cols: np.ndarray, vals: np.ndarray):
    """CSC arrays (col_start, row_index, value) with rows sorted inside each column."""
    order = np.lexsort((rows, cols))
    rows = rows[order].astype(np.int32)
    vals = vals[order].astype(np.float64)
    counts = np.bincount(cols, minlength=n)
    col_start = np.zeros(n + 1, dtype=np.int32)
    np.cumsum(counts, out=col_start[1:])
    return col_start, rows, vals


def from_dense(c, A, row_lower, row_upper, col_lower, col_upper, sense=1, offset=0.0, name="") -> Lp:
    A = np.asarray(A, dtype=np.float64)
    m, n = A.shape
    r, k = np.nonzero(A)
    cs, ri, v = csc_from_triplets(m, n, r, k, A[r, k])
    f = lambda a: np.asarray(a, dtype=np.float64).copy()
    return Lp(m, n, f(c), f(col_lower), f(col_upper), f(row_lower), f(row_upper), cs, ri, v, sense, float(offset),
              name)


def _distinct_columns(rng: np.random.Generator, m: int, n: int, k: int) -> np.ndarray:
    """m x k column indices, distinct inside each row, uniform over [0, n)."""
    cols = rng.integers(0, n, size=(m, k), dtype=np.int64)
    while True:
        s = np.sort(cols, axis=1)
        bad = np.nonzero((s[:, 1:] == s[:, :-1]).any(axis=1))[0]
        if bad.size == 0:
            return cols
        cols[bad] = rng.integers(0, n, size=(bad.size, k), dtype=np.int64)


def random_lp(m: int, n: int | None = None, nnz_per_row: int = 6, seed: int = 1) -> Lp:
    """Random equality LP (see module docstring). n defaults to 1.5 m."""
    if n is None:
        n = (3 * m) // 2
    rng = np.random.Generator(np.random.PCG64(seed))
    cols = _distinct_columns(rng, m, n, nnz_per_row)
    rows = np.repeat(np.arange(m, dtype=np.int64), nnz_per_row)
    cols = cols.reshape(-1)
    vals = rng.standard_normal(m * nnz_per_row)
    x0 = rng.uniform(0.0, 1.0, n)
    b = np.bincount(rows, weights=vals * x0[cols], minlength=m)
    y0 = rng.standard_normal(m)
    z = np.where(rng.uniform(0.0, 1.0, n) < 0.5, rng.uniform(0.0, 1.0, n), 0.0)
    c = np.bincount(cols, weights=vals * y0[rows], minlength=n) + z
    cs, ri, v = csc_from_triplets(m, n, rows, cols, vals)
    return Lp(m, n, c, np.zeros(n), np.full(n, 10.0), b.copy(), b.copy(), cs, ri, v, 1, 0.0,
              f"random-{m}x{n}-s{seed}", {"x0": x0})


def staircase_lp(T: int, seed: int = 1, rows_per: int = 49, cols_per: int = 60, nnz_per: int = 160,
                 n_inventory: int = 5, eq_fraction: float = 0.3) -> Lp:
    """Multi-period staircase planning LP with T periods (see module docstring)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    m, n = T * rows_per, T * cols_per
    rr, cc, vv = [], [], []
    for t in range(T):
        # block entries: drawn uniformly without duplicates, then every empty row and column
        # of the block gets one entry; magnitudes log-uniform in [1e-2, 1e2], random signs
        present = np.zeros(rows_per * cols_per, dtype=bool)
        present[rng.permutation(rows_per * cols_per)[:nnz_per]] = True
        present = present.reshape(rows_per, cols_per)
        for i in np.nonzero(~present.any(axis=1))[0]:
            present[i, rng.integers(0, cols_per)] = True
        for j in np.nonzero(~present.any(axis=0))[0]:
            present[rng.integers(0, rows_per), j] = True
        block = np.where(present, 10.0 ** rng.uniform(-2.0, 2.0, present.shape), 0.0)
        block *= np.where(rng.uniform(0.0, 1.0, present.shape) < 0.5, -1.0, 1.0)
        # inventory k of period t (column cols_per - n_inventory + k) enters row k with +1
        for k in range(n_inventory):
            block[k, cols_per - n_inventory + k] = 1.0
        r, k = np.nonzero(block)
        rr.append(r + t * rows_per)
        cc.append(k + t * cols_per)
        vv.append(block[r, k])
        if t > 0:  # ... and row k of period t with -1 (inventory carried over from t-1)
            rr.append(np.arange(n_inventory) + t * rows_per)
            cc.append(np.arange(n_inventory) + (t - 1) * cols_per + cols_per - n_inventory)
            vv.append(-np.ones(n_inventory))
    rows = np.concatenate(rr).astype(np.int64)
    cols = np.concatenate(cc).astype(np.int64)
    vals = np.concatenate(vv)
    ub = rng.uniform(10.0, 1000.0, n)
    xstar = ub * rng.uniform(0.2, 0.8, n)
    ax = np.bincount(rows, weights=vals * xstar[cols], minlength=m)
    hour = np.arange(T) % 24
    demand = rng.uniform(50.0, 150.0, T) * (1.0 + 0.3 * np.sin(2.0 * np.pi * hour / 24.0))
    d_row = np.repeat(demand, rows_per)
    kind = rng.uniform(0.0, 1.0, m)
    u = rng.uniform(0.0, 1.0, m)
    rl = np.full(m, -np.inf)
    ru = np.full(m, np.inf)
    eq = kind < eq_fraction
    ge = (~eq) & (kind < eq_fraction + (1 - eq_fraction) / 2)
    le = ~(eq | ge)
    rl[eq] = ax[eq]
    ru[eq] = ax[eq]
    rl[ge] = ax[ge] - d_row[ge] * u[ge]
    ru[le] = ax[le] + d_row[le] * u[le]
    c = rng.standard_normal(n)
    cs, ri, v = csc_from_triplets(m, n, rows, cols, vals)
    return Lp(m, n, c, np.zeros(n), ub, rl, ru, cs, ri, v, 1, 0.0, f"staircase-T{T}-s{seed}", {"x0": xstar})


def scenarios(base: Lp, K: int, sigma: float = 0.1, seed: int = 1) -> list[dict]:
    """K scenarios: objective and finite row bounds times lognormal(0, sigma) factors.

    Returns a list of dicts with keys ``obj``, ``row_lower``, ``row_upper`` (float64 arrays),
    the difference format of the reference's ``Scenario`` (include/ps26119/batch.h:23-27).
    """
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for _ in range(K):
        fc = np.exp(sigma * rng.standard_normal(base.num_cols))
        fb = np.exp(sigma * rng.standard_normal(base.num_rows))
        rl = np.where(np.isfinite(base.row_lower), base.row_lower * fb, base.row_lower)
        ru = np.where(np.isfinite(base.row_upper), base.row_upper * fb, base.row_upper)
        out.append({"obj": base.c * fc, "row_lower": rl, "row_upper": ru})
    return out


def feasible_scenarios(base: Lp, K: int, sigma: float = 0.1, seed: int = 1) -> list[dict]:
    """K feasible scenarios of a base LP that carries an interior point ``meta["x0"]`` (the
    generators above record it): x' = clip(x0 · lognormal(0, sigma), col bounds), row bounds
    around A x' (equality rows: A x'; one-sided rows: A x' ∓ base slack · lognormal(0, sigma)),
    objective c · lognormal(0, sigma). Same dict format as :func:`scenarios`."""
    x0 = np.asarray(base.meta["x0"], dtype=np.float64)
    rng = np.random.Generator(np.random.PCG64(seed))
    ax0 = base.row_activity(x0)
    lo_slack = np.where(np.isfinite(base.row_lower), ax0 - base.row_lower, np.inf)
    up_slack = np.where(np.isfinite(base.row_upper), base.row_upper - ax0, np.inf)
    eq = base.row_lower == base.row_upper
    out = []
    for _ in range(K):
        xs = np.clip(x0 * np.exp(sigma * rng.standard_normal(base.num_cols)), base.col_lower, base.col_upper)
        ax = base.row_activity(xs)
        fb = np.exp(sigma * rng.standard_normal(base.num_rows))
        rl = np.where(eq, ax, ax - lo_slack * fb)
        ru = np.where(eq, ax, ax + up_slack * fb)
        fc = np.exp(sigma * rng.standard_normal(base.num_cols))
        out.append({"obj": base.c * fc, "row_lower": rl, "row_upper": ru})
    return out
