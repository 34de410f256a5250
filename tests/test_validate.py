"""Model validation (csrc/solver.cpp Model::validate) against a sequential restatement of the
reference's rules (src/core/model.cpp:93-151): columns in order, and inside a column its entries
in order (row index range, duplicate, finiteness), then column bounds, then row bounds; the first
failing rule gives the message. The library checks column ranges on several threads and must
still report that first error. Malformed models are run through ps26119_solve_lp_ex, which
validates before anything reaches a device."""
import numpy as np
import pytest

import ps26119
from ps26119 import generators as g
from test_abi import _call


def sequential_first_error(lp):
    n, m = lp.num_cols, lp.num_rows
    cs, ri, v, c = lp.col_start, lp.row_index, lp.value, lp.c
    nnz = len(v)
    for j in range(n):
        if cs[j + 1] < cs[j]:
            return f"col_start not monotone at column {j}"
        if not np.isfinite(c[j]):
            return f"objective coefficient of column {j} is not finite"
        assert cs[j + 1] <= nnz, "case outside the restatement (pointer past nnz)"
        seen = set()
        for k in range(cs[j], cs[j + 1]):
            i = int(ri[k])
            if i < 0 or i >= m:
                return f"row index out of range in column {j}"
            if i in seen:
                return f"duplicate entry ({i},{j})"
            seen.add(i)
            if not np.isfinite(v[k]):
                return f"matrix entry ({i},{j}) is not finite"
    for lo, up, what in ((lp.col_lower, lp.col_upper, "column"), (lp.row_lower, lp.row_upper, "row")):
        for k in range(len(lo)):
            if np.isnan(lo[k]) or np.isnan(up[k]):
                return f"{what} bound {k} is NaN"
            if lo[k] == np.inf:
                return f"{what} lower bound {k} is +inf"
            if up[k] == -np.inf:
                return f"{what} upper bound {k} is -inf"
    return ""


@pytest.fixture(scope="module")
def big():
    return g.random_lp(50_000, seed=2)  # 75,000 columns: validated on several threads


def _message(lp):
    st, res = _call(ps26119.load(), lp)
    msg = res.message.decode()
    if st == ps26119.INVALID_ARGUMENT and msg.startswith("invalid model: "):
        return msg[len("invalid model: "):]
    return ""


def _edit(lp, **kw):
    arrays = {k: getattr(lp, k).copy() for k in kw}
    for k, f in kw.items():
        f(arrays[k])
    return lp.with_data(**arrays)


def _cases(lp):
    cs = lp.col_start

    def put(idx, val):
        def f(a):
            a[idx] = val
        return f

    def swap_in_column(j):
        def f(a):
            a[cs[j]], a[cs[j] + 1] = a[cs[j] + 1], a[cs[j]]
        return f

    def dup_in_column(j):
        def f(a):
            a[cs[j] + 1] = a[cs[j]]
        return f

    def both(*fs):
        def f(a):
            for h in fs:
                h(a)
        return f

    return {
        "range_then_nan": dict(row_index=put(cs[40000], -1), value=put(cs[70000], np.nan)),
        "nan_only_late": dict(value=put(cs[70000] + 1, np.inf)),
        "row_index_too_big": dict(row_index=put(cs[123] + 1, lp.num_rows)),
        "duplicate_then_range": dict(row_index=both(dup_in_column(123), put(cs[60000], -7))),
        "duplicate_after_unsorted": dict(row_index=both(swap_in_column(30000), dup_in_column(30001))),
        "unsorted_but_valid": dict(row_index=swap_in_column(5)),
        "objective_nan": dict(c=both(put(70001, np.nan), put(3, np.inf))),
        "not_monotone": dict(col_start=put(50000, int(cs[50001]) + 1)),
        "column_bound_nan": dict(col_lower=put(74999, np.nan)),
        "row_lower_plus_inf": dict(row_lower=put(5, np.inf)),
        "row_upper_minus_inf": dict(row_upper=put(49999, -np.inf)),
    }


CASES = ["range_then_nan", "nan_only_late", "row_index_too_big", "duplicate_then_range", "duplicate_after_unsorted",
         "unsorted_but_valid", "objective_nan", "not_monotone", "column_bound_nan", "row_lower_plus_inf",
         "row_upper_minus_inf"]


@pytest.mark.parametrize("case", CASES)
def test_first_error_matches_sequential_rules(big, case):
    lp = _edit(big, **_cases(big)[case])
    want = sequential_first_error(lp)
    assert (want == "") == (case == "unsorted_but_valid")
    assert _message(lp) == want


def test_pointer_past_nnz_reports_the_decreasing_column(big):
    # a column pointer beyond nnz followed by a decrease: reported as the first decreasing column,
    # without reading past the entry arrays
    cs = big.col_start.copy()
    cs[10] = big.nnz + 100
    lp = big.with_data(col_start=cs)
    assert _message(lp) == "col_start not monotone at column 10"


def test_valid_model_has_no_message(big):
    assert _message(big) == "" and sequential_first_error(big) == ""


def test_calls_of_different_sizes_on_one_thread(big):
    # The C API keeps the calling thread's model copy for its next call: models of other sizes,
    # valid and invalid, must each be judged on their own data only.
    small = g.random_lp(30, seed=5)
    bad_small = _edit(small, value=lambda a: a.__setitem__(3, np.nan))
    bad_big = _edit(big, row_index=lambda a: a.__setitem__(5, -2))
    sequence = [big, bad_small, small, bad_big, small, big, bad_small]
    for lp in sequence:
        assert _message(lp) == sequential_first_error(lp)
