"""Replica plumbing of bench.py on two gloo ranks (CPU): the job time is the
slowest rank's, the throughput counts every rank's steps, barriers pair up,
and the reference arm prints on rank 0 only."""

import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank), GPE_BENCH_BACKEND="gloo")
    import bench
    import torch.distributed as dist
    w, r, _ = bench.dist_init(world)
    assert (w, r) == (world, rank)
    bench.barrier(w)
    ms = 10.0 * (rank + 1)            # rank 1 is the slow one
    ms_max, value = bench.job_throughput(ms, 100, w)
    bench.barrier(w)

    class A:
        steps, warmup = 5, 3
    ref = bench.reference(A, w, r) if r != 0 else "rank0"
    out.put((rank, ms_max, value, ref))
    dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_gloo_ranks_aggregate_like_the_bench():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=100) for _ in range(world))
    for p in procs:
        p.join(30)
        assert p.exitcode == 0
    for rank, ms_max, value, ref in res:
        assert ms_max == 20.0                       # max over ranks
        assert value == pytest.approx(2 * 100 / 0.020)
    assert res[1][3] is None                        # reference arm: rank 0 only
