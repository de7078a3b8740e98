"""The benchmark's multi-rank logic (bench.py: dist_setup, barrier, max_over_ranks, whole_job) on
CPU with two gloo ranks, as torchrun would start them: the job's time is the slowest rank's, and the
whole-job rate counts every rank's replica.  With several GPUs each rank runs its own replica of
the workload (the path is one GPU's; replicas exchange nothing but the timing)."""
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "RANK": str(rank),
                       "LOCAL_RANK": str(rank), "WORLD_SIZE": str(world)})
    sys.path.insert(0, ROOT)
    import torch.distributed as dist

    import bench

    w, r, local = bench.dist_setup(None)
    bench.barrier(w)
    ms_local = 10.0 + 5.0 * r  # rank 1 is the slower one
    ms, value = bench.whole_job(1000, ms_local, w)
    out.put((r, w, ms, value, bench.max_over_ranks(-float(r), w)))
    bench.barrier(w)
    dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_rank_and_count_every_replica():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for pr in procs:
        pr.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for pr in procs:
        pr.join(timeout=60)
        assert pr.exitcode == 0
    for r, w, ms, value, mx in res:
        assert w == 2
        assert ms == 15.0                          # the slower rank's time on every rank
        assert value == pytest.approx(2 * 1000 / 15e-3)  # both replicas' units over that time
        assert mx == 0.0                           # max of (0, -1)
