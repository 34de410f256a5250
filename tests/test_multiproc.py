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
