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


def test_full_sweep_roofline_reads_its_phases_and_the_committed_traffic_ratio():
    s0 = dict(sweep_ms=1.0, sweep_bytes=10, sweep_count=2, sweep_phase_ms=[0.1, 0.2, 0.3, 0.4])
    s1 = dict(sweep_ms=3.0, sweep_bytes=10 + 4_000_000_000, sweep_count=3, sweep_phase_ms=[0.2, 1.2, 1.0, 0.6])
    peak = 6543.7
    r = bench.full_sweep_roofline(s0, s1, {"proper": 1}, peak, "measured", "sweep_full_chunglu_div16.md")
    assert r["ms"] == 2.0 and r["algorithmic_bytes"] == 4_000_000_000 and r["sweeps"] == 1
    assert abs(r["achieved"] - 2000.0) < 1e-9 and abs(r["frac"] - 2000.0 / peak) < 1e-12
    ratio = bench.read_row("sweep_full_chunglu_div16.md", "full_sweep_dram_per_algorithmic")
    assert ratio is not None and 0.5 < ratio < 2.0
    assert r["traffic"] == int(ratio * 4_000_000_000)
    ph = r["phases_ms"]
    assert [round(ph[k], 9) for k in ("item_build", "long_row_items", "finalize", "select_commit")] == \
        [0.1, 1.0, 0.7, 0.2]
    assert bench.full_sweep_roofline(s0, s1, {"proper": 1}, peak, "measured")["traffic"] is None
    assert bench.full_sweep_roofline(s0, s1, None, peak, "measured") is None


def test_apply_traffic_rows_are_in_the_committed_profiles():
    for wl, (apply_prof, _, _) in bench.PROFILES.items():
        if apply_prof:
            v = bench.read_traffic(apply_prof, "apply_dram_bytes_per_launch")
            assert v is not None and v > 10 ** 6, wl
