"""The request loop (csrc/serve.{hpp,cpp}, ps26119_server_*): admission by slots and HBM budget
in arrival order, request timing, argument errors; on the GPU, every served result equals the
result of the same LP solved alone through ps26119_solve_lp_ex.

The CPU tests use the server's dry-run mode (requests hold their slot and memory estimate for a
fixed time and are not solved), so the admission policy is checked without a device."""
import threading
import time

import numpy as np
import pytest

import ps26119
from ps26119 import generators as g

HOLD = 0.25  # seconds a dry-run request holds its slot


def _lp(m, seed):
    return g.random_lp(m, seed=seed)


def _starts(srv, ids):
    return [srv.result(i)[1] for i in ids]


def test_slots_bound_the_requests_in_flight():
    with ps26119.Server(slots=3, dry_run_seconds=HOLD) as srv:
        ids = [srv.submit(_lp(50, k)) for k in range(6)]
        times = _starts(srv, ids)
    started = sorted(t[1] for t in times)
    # three start at once, the other three when the first ones finish
    assert started[2] - started[0] < 0.5 * HOLD
    assert started[3] - started[0] >= 0.9 * HOLD
    for sub, st, fin in times:
        assert sub <= st < fin and fin - st >= 0.9 * HOLD


def test_budget_admits_in_arrival_order():
    small, big = _lp(50, 1), _lp(4000, 2)
    with ps26119.Server(slots=8, hbm_budget_bytes=1.0, dry_run_seconds=HOLD) as srv:
        # a budget below any request: only the first request in flight is ever admitted
        ids = [srv.submit(lp) for lp in (big, small, small)]
        times = _starts(srv, ids)
    s = [t[1] for t in times]
    assert s[0] <= s[1] - 0.9 * HOLD and s[1] <= s[2] - 0.9 * HOLD  # one at a time, FIFO


def test_head_of_line_request_waits_for_memory():
    est_small = 1.25 * (60 * 300 + 280 * (50 + 75)) + 32 * 2**20
    with ps26119.Server(slots=8, hbm_budget_bytes=2.5 * est_small, dry_run_seconds=HOLD) as srv:
        a = srv.submit(_lp(50, 1))
        b = srv.submit(_lp(50, 2))
        big = srv.submit(_lp(20000, 3))  # does not fit beside a and b
        c = srv.submit(_lp(50, 4))       # fits, but waits behind the big request
        ta, tb, tbig, tc = (srv.result(i)[1] for i in (a, b, big, c))
    assert abs(ta[1] - tb[1]) < 0.5 * HOLD
    assert tbig[1] >= ta[2] - 1e-3       # the big one starts only when memory is free
    assert tc[1] >= tbig[1] - 1e-3       # arrival order is kept


def test_requests_arriving_while_others_run_start_when_a_slot_frees():
    with ps26119.Server(slots=2, dry_run_seconds=HOLD) as srv:
        first = [srv.submit(_lp(50, k)) for k in range(2)]
        time.sleep(0.5 * HOLD)
        late = srv.submit(_lp(50, 9))
        t_first = [srv.result(i)[1] for i in first]
        t_late = srv.result(late)[1]
    assert t_late[0] > max(t[1] for t in t_first)  # submitted after the first two started
    assert t_late[1] >= min(t[2] for t in t_first) - 1e-3


def test_poll_and_errors():
    with ps26119.Server(slots=1, dry_run_seconds=HOLD) as srv:
        rid = srv.submit(_lp(50, 1))
        assert srv.poll(rid) is None  # still running
        res, times = srv.result(rid)
        assert res.status == ps26119.NOT_SOLVED and res.engine == "dry-run"
        with pytest.raises(KeyError):
            srv.poll(rid)  # forgotten once taken
        bad = _lp(50, 2)
        bad = bad.with_data(row_index=np.where(np.arange(bad.nnz) == 0, -1, bad.row_index).astype(np.int32))
        with pytest.raises(ValueError, match="invalid model: row index out of range"):
            srv.submit(bad)
        with pytest.raises(ValueError, match="tolerance"):
            srv.submit(_lp(50, 3), tolerance=-1.0)
    with pytest.raises(ValueError):
        ps26119.Server(slots=-1)


def test_destroy_finishes_submitted_requests():
    srv = ps26119.Server(slots=2, dry_run_seconds=0.1)
    for k in range(5):
        srv.submit(_lp(50, k))
    t0 = time.perf_counter()
    srv.close()
    assert time.perf_counter() - t0 >= 0.25  # three rounds of 0.1 s


def test_concurrent_submitters():
    with ps26119.Server(slots=4, dry_run_seconds=0.02) as srv:
        ids, lock = [], threading.Lock()

        def worker(k):
            for j in range(5):
                rid = srv.submit(_lp(30, 10 * k + j))
                with lock:
                    ids.append(rid)

        th = [threading.Thread(target=worker, args=(k,)) for k in range(4)]
        for t in th:
            t.start()
        for t in th:
            t.join()
        assert sorted(ids) == list(range(20))
        assert all(srv.result(i)[0].engine == "dry-run" for i in ids)


@pytest.mark.gpu
@pytest.mark.parametrize("grouped", [True, False], ids=["grouped", "solo"])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_served_results_equal_single_solves(grouped, precision):
    """Each request's result is the same alone and in the mix, bit for bit: with the grouped
    kernels (the running requests' iteration kernels launched together, requests joining and
    leaving the group at epoch boundaries) and with each request's own kernels; in fp64 and in
    mixed precision (a request promotes to fp64 while its neighbours still run in fp32)."""
    lps = [_lp(m, seed) for m, seed in ((300, 1), (1200, 2), (50, 3), (2500, 4), (800, 5), (150, 6))]
    with ps26119.Server(slots=4, grouped=grouped) as srv:
        ids = [srv.submit(lp, precision=precision) for lp in lps]
        served = [srv.result(i) for i in ids]
    for lp, (res, (sub, st, fin)) in zip(lps, served):
        alone = ps26119.solve_lp(lp.c, (lp.col_start, lp.row_index, lp.value), lp.row_lower, lp.row_upper,
                                 lp.col_lower, lp.col_upper, sense=lp.sense, offset=lp.offset, algorithm="r2hpdhg",
                                 precision=precision)
        assert res.status == alone.status == ps26119.OPTIMAL and res.check == alone.check == "PASS"
        assert res.iterations == alone.iterations and res.objective == alone.objective
        assert np.array_equal(res.x, alone.x) and np.array_equal(res.y, alone.y)
        assert res.certified_bound == alone.certified_bound
        assert sub <= st < fin


@pytest.mark.gpu
def test_grouped_requests_retire_and_refill():
    """Continuous batching: with 3 slots and 9 requests of very different lengths, short requests
    finish and leave the group while long ones keep running, and queued requests take the freed
    slots and join the running group. Every request ends Optimal with the result of its solo
    solve; some request starts before another that was admitted earlier has finished."""
    lps = [_lp(m, seed) for m, seed in ((2000, 11), (40, 12), (60, 13), (1500, 14), (30, 15), (50, 16), (900, 17),
                                        (20, 18), (70, 19))]
    with ps26119.Server(slots=3, grouped=True) as srv:
        ids = [srv.submit(lp) for lp in lps]
        served = [srv.result(i) for i in ids]
    spans = [(t[1], t[2]) for _, t in served]
    # a refill: a later request started while an earlier, longer one was still running
    assert any(spans[j][0] < spans[i][1] and spans[j][0] > spans[i][0] for i in range(len(lps)) for j in range(i + 1, len(lps)))
    for lp, (res, _) in zip(lps, served):
        alone = ps26119.solve_lp(lp.c, (lp.col_start, lp.row_index, lp.value), lp.row_lower, lp.row_upper,
                                 lp.col_lower, lp.col_upper, sense=lp.sense, offset=lp.offset, algorithm="r2hpdhg")
        assert res.status == ps26119.OPTIMAL and res.iterations == alone.iterations
        assert np.array_equal(res.x, alone.x) and np.array_equal(res.y, alone.y)
