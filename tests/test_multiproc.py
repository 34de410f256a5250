"""The multi-process host logic of bench.py on CPU: two ranks over gloo (world size 2) set up the
process group from the torchrun environment, agree on the max over ranks of their timings,
pass the barrier and leave cleanly. A single LP does not shard (replicas only), so this
bookkeeping is the whole multi-GPU path; the GPU side is one independent solve per rank."""
import multiprocessing as mp
import os
import socket

import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port), CUDA_VISIBLE_DEVICES="")
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    import torch.distributed as dist
    r, w, local = bench.dist_setup()
    v = bench.max_over_ranks(1.5 * (rank + 1), w)
    bench.barrier(w)
    backend = dist.get_backend()
    dist.destroy_process_group()
    q.put((r, w, local, v, backend))


def test_two_ranks_agree_on_the_max_over_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=180)
    for p in procs:
        if p.is_alive():
            p.kill()
            pytest.fail("a rank did not finish")
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in procs)
    assert got == [(0, 2, 0, 3.0, "gloo"), (1, 2, 1, 3.0, "gloo")]


def test_single_process_needs_no_process_group():
    import bench
    assert bench.max_over_ranks(2.5, 1) == 2.5
    bench.barrier(1)


def _serve_rank(rank, world, port, q):
    """One rank of a sharded serving stream in dry-run mode (admission and timing without solving,
    so it runs on a CPU): serves its share and gathers every rank's results."""
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port), CUDA_VISIBLE_DEVICES="")
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path[:0] = [root, os.path.join(root, "ps26119-solver_b200")]
    import bench
    import torch.distributed as dist
    from ps26119 import generators as g, shard
    import ps26119
    r, w, _ = bench.dist_setup()
    reqs = [g.random_lp(m, seed=100 + k) for k, m in enumerate([60, 900, 200, 40, 500, 120, 700, 80, 300])]
    mine = shard.assign(len(reqs), w, [lp.nnz for lp in reqs])[r]
    with ps26119.Server(slots=2, dry_run_seconds=0.01) as srv:
        ids = [srv.submit(reqs[k]) for k in mine]
        local = {k: (srv.result(i)[0].status_name, reqs[k].num_rows) for k, i in zip(mine, ids)}
    got = shard.gather(local, w)
    dist.destroy_process_group()
    q.put((r, mine, sorted(got.items())))


def test_sharded_stream_covers_every_request_once():
    """Request-level multi-GPU (row e): two ranks over gloo split a stream of uneven LPs by
    longest-first assignment, serve their shares independently, and the gathered results cover
    every request exactly once, each with its own LP."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_serve_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=180)
    for p in procs:
        if p.is_alive():
            p.kill()
            pytest.fail("a rank did not finish")
        assert p.exitcode == 0
    out = sorted(q.get(timeout=10) for _ in procs)
    shares = [set(o[1]) for o in out]
    assert shares[0] and shares[1] and not (shares[0] & shares[1]) and shares[0] | shares[1] == set(range(9))
    rows = [60, 900, 200, 40, 500, 120, 700, 80, 300]
    for _, _, got in out:  # every rank sees the whole stream's results
        assert [k for k, _ in got] == list(range(9))
        assert [v[1] for _, v in got] == rows


def test_assignment_balances_and_is_deterministic():
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "ps26119-solver_b200"))
    from ps26119 import shard
    assert shard.assign(7, 3) == [[0, 3, 6], [1, 4], [2, 5]]
    cost = [1, 10, 3, 3, 7, 2]
    parts = shard.assign(6, 2, cost)
    assert parts == shard.assign(6, 2, cost) and sorted(sum(parts, [])) == list(range(6))
    loads = [sum(cost[k] for k in p) for p in parts]
    assert max(loads) - min(loads) <= max(cost)
    assert shard.assign(3, 5, [1, 1, 1]) == [[0], [1], [2], [], []]
    with pytest.raises(ValueError):
        shard.assign(2, 0)
