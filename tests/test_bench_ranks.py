"""The bench's multi-rank path on CPU: two gloo ranks (one per process, as
torchrun runs replicas or shards) agree on the slowest rank's timings and on
the sum of their counts, and the whole-job rate counts every replica's work
over that time."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

import bench


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mine = [10.0 + 5 * rank, 3.0 - rank]  # rank 1 is slower on the first timing, faster on the second
        q.put((rank, (bench.max_over_ranks(dist, mine, "cpu"), bench.sum_over_ranks(dist, [1.0 + rank, 7.0], "cpu"))))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_ranks_take_the_slowest_timing():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=90) for _ in procs)
    for p in procs:
        p.join(30)
        assert p.exitcode == 0
    assert got[0] == got[1] == ([15.0, 3.0], [3.0, 14.0])


def test_job_rate_counts_every_replica():
    assert bench.job_rate(32768 * 24, 4, 2.0) == 4 * 32768 * 24 / 2.0
