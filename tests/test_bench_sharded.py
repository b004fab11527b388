"""The multi-rank forms of the bench on two gloo ranks (CPU): replicas of the
plain path, and graphs (batched) and tenants (served) placed on the ranks by
resident bytes, each rank running its share; rank 0 alone prints one line
with every rank's work over the slowest rank's time. The engines are replaced by stand-ins that count what they are
given; what runs for real is the bench's placement, generation, client loop
and the host-side reductions."""
import io
import json
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


class _Handle:
    def __init__(self, g, **k):
        self.n = g.n

    def color_core(self, min_degree):
        return 0

    def synchronize(self):
        pass

    def apply(self, ups, mode=0):
        pass

    def publish(self):
        return dict(proper=1)

    def stats(self):
        return dict(kernel_launches=7)

    def close(self):
        pass


class _Batch:
    def __init__(self, graphs, **k):
        self.k = 0

    def color_core(self, min_degree):
        return 0

    def submit(self, k, part):
        pass

    def close_epochs(self):
        pass

    def tick(self):
        return dict(proper=1, device_ms=0.3)

    def tick_begin(self):
        pass

    def tick_end(self):
        return self.tick()

    def tuning(self):
        return {"tile": 512}

    def stats(self):
        self.k += 1
        return dict(kernel_launches=10 * self.k)

    def validate(self):
        return dict(violations=0, uncolored_with_edges=0)

    def close(self):
        pass


class _Server:
    def __init__(self, **k):
        self.n = []
        self.req = 0
        self.vis = 0

    @staticmethod
    def footprint(n, entries, slack_pct=300):
        import streamgc_b200 as S
        return S.lib().sgc_tenant_footprint(n, entries, slack_pct)

    def add_tenant(self, g, epoch_size=0):
        self.n.append(g.n)
        return len(self.n) - 1

    def step(self):
        self.vis = self.req
        return dict(admitted=len(self.n), proper=1, groups_ticked=1, step_ms=0.4)

    def stats(self):
        return dict(requests_visible=self.vis, update_requests=self.req, updates_applied=10 * self.req,
                    resident_bytes=10 ** 9, ticks=5, tier2_ticks=0, tier2_mirror_ticks=0, tier1_sweeps=7,
                    tick_device_ms=1.0, overflows=0, drain_failed=0, device_errors=0, tenants_regrown=0,
                    visible_p50_ms=1.0, visible_p99_ms=2.0, query_p50_ms=0.1, query_p99_ms=0.2)

    def submit(self, t, ups):
        self.req += 1

    def query(self, t, v):
        return np.zeros(len(v), np.uint16)

    def rows(self, t):
        return np.zeros(2, np.uint64), np.zeros(0, np.uint32)

    def close(self):
        pass


class _PlainHandle:
    def __init__(self, g, **k):
        self.n = g.n
        self.k = 0

    def color_core(self, min_degree):
        return 0

    def apply(self, ups, mode=0):
        pass

    def apply_ptr(self, ptr, n, mode=0):
        pass

    def publish(self):
        return dict(tier1_iterations=1, tier1_last_count=0, tier2_ran=0, tier2_fixed=0, tier2_gave_up=0,
                    drained=0, drain_failed=0, proper=1, incremental=1)

    def repair(self):
        return dict(self.publish(), incremental=0)

    def synchronize(self):
        pass

    def cuda_stream(self):
        return 0

    def stats(self):
        self.k += 1
        return dict(sweep_ms=1.0 * self.k, sweep_bytes=10 ** 9 * self.k, sweep_count=3 * self.k,
                    kernel_launches=100 * self.k, h2d_bytes=0, d2h_bytes=0)

    def validate(self):
        return dict(violations=0, uncolored_with_edges=0, max_color=12, edges=1, out_of_range=0)

    def snapshot(self):
        return np.zeros(self.n, np.uint16)

    def colors(self):
        return np.zeros(self.n, np.uint16)

    def close(self):
        pass


class _Event:
    n = 0

    def __init__(self, enable_timing=True):
        _Event.n += 1
        self.t = _Event.n

    def record(self, s=None):
        pass

    def elapsed_time(self, o):
        return 0.25 * (o.t - self.t)


class _Tensor:
    def to(self, *a, **k):
        return self

    def data_ptr(self):
        return 0

    def pin_memory(self):
        return self

    def add_(self, x):
        return self


class _Stream:
    def __init__(self, *a, **k):
        pass

    def synchronize(self):
        pass


def _small_specs(count, seed=42, **k):
    rng = np.random.default_rng(seed)
    fams = ("delaunay", "rmat", "chung_lu")
    return [dict(index=i, family=fams[i % 3], n=int(rng.integers(1024, 4096)), epoch=1024, seed=seed * 1000 + i)
            for i in range(count)]


def _rank(rank, world, port, form, q, workload="small", large_div=1):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK="0", SGC_DIST_BACKEND="gloo")
    import types

    import torch
    torch.cuda.set_device = lambda *a: None
    torch.cuda.synchronize = lambda *a: None
    import bench
    import streamgc_b200 as S
    from streamgc_b200 import workloads as W
    S.StreamGC, S.Batch, S.Server = (_PlainHandle if form == "plain" else _Handle), _Batch, _Server
    if form == "plain":
        import contextlib
        torch.cuda.ExternalStream = _Stream
        torch.cuda.Event = _Event
        torch.cuda.stream = lambda st: contextlib.nullcontext()
        torch.from_numpy = lambda arr: _Tensor()
        torch.empty = lambda *a, **k: _Tensor()
    W.batch_specs = _small_specs
    real_rmat = S.Graph.rmat
    S.Graph.rmat = staticmethod(lambda scale, ef, a=0.57, b=0.19, c=0.19, seed=42:
                                real_rmat(min(scale, 10), min(ef, 8), a, b, c, seed))
    args = types.SimpleNamespace(gpus=world, steps=2, warmup=3, batch_graphs=6, autotune=False, served_rate=2e5,
                                 served_seconds=0.3, served_staleness_us=2000, served_check=False,
                                 served_regrow=False, sorted_rows=False, workload=workload, cpu_batches=0,
                                 cpu_seconds=1.0, profile_window=False, graph_publish=False, ingest=False,
                                 latency_epochs=4, validate_steps=True, large_div=large_div,
                                 full_repair_every=0, profile_full_sweep=True,
                                 profile_full_sweep_window=False)
    out, err = io.StringIO(), None
    old = sys.stdout
    sys.stdout = out
    try:
        {"plain": bench.run_ours, "batched": bench.run_batched, "served": bench.run_served}[form](args)
    except Exception as e:  # reported to the parent
        err = repr(e)
    finally:
        sys.stdout = old
    q.put((rank, out.getvalue(), err))


@pytest.mark.timeout(600)
@pytest.mark.parametrize("form", ["plain", "batched", "served"])
def test_two_ranks_share_the_work(form):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, form, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = {}
    for _ in procs:
        r, text, err = q.get(timeout=540)
        got[r] = (text, err)
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    assert got[0][1] is None and got[1][1] is None, (got[0][1], got[1][1])
    lines = [json.loads(l) for l in got[0][0].splitlines() if l.startswith("{")]
    assert len(lines) == 1 and not [l for l in got[1][0].splitlines() if l.startswith("{")]
    line = lines[0]
    assert line["n_gpus"] == 2 and line["value"] > 0
    if form == "plain":  # replicas: twice one replica's epochs over the slowest replica's time
        assert line["config"]["parallelism"] == "replicas x2"
        assert line["value"] == pytest.approx(2 * 2 * 32768 / (line["ms_per_step"] * 2 / 1e3))
        assert line["config"]["snapshots_validated"] == 2 and line["config"]["snapshot_violations"] == 0
        assert line["latency_ms"]["samples"] == 4
        return
    assert line["form"] == form
    assert line["config"]["placement"].startswith("2 ranks")
    specs = _small_specs(6 if form == "batched" else 63, seed=42 if form == "batched" else 43)
    if form == "batched":
        assert line["config"]["vertices"] == sum(s["n"] for s in specs)
    else:
        assert line["config"]["vertices"] == sum(s["n"] for s in specs) + (1 << 22)  # the R-MAT 2^22 tenant's spec


@pytest.mark.timeout(600)
def test_replicas_share_one_host_copy_of_the_large_graph():
    """Replicas of the large workload (here scaled down): rank 0 generates it
    and shares the arrays through /dev/shm, the other rank maps them; the
    files are gone once both handles exist."""
    import glob
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, "plain", q, "large", 8192)) for r in range(2)]
    for p in procs:
        p.start()
    got = {}
    for _ in procs:
        r, text, err = q.get(timeout=540)
        got[r] = (text, err)
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    assert got[0][1] is None and got[1][1] is None, (got[0][1], got[1][1])
    line = [json.loads(l) for l in got[0][0].splitlines() if l.startswith("{")][0]
    assert line["config"]["workload"] == "chunglu65m_div8192_churn" and line["n_gpus"] == 2
    assert not glob.glob(f"/dev/shm/sgc_large_8192_{port}_*")
