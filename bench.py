#!/usr/bin/env python
"""Throughput of the streaming graph-coloring path on B200.

Workload (default, `--workload large`): Chung-Lu graph with 65,608,366
vertices, expected degrees from a power law with exponent 2.1 scaled to an
average of 55 and capped at 100,000 (seed 42; ~1.8 G undirected edges, a
slack CSR of ~14.3 G slots with 64-bit row offsets), colored by one full
repair of its loaded rows, then the reference's 50/50 churn stream of
10,000,000 updates (seed 42), epoch E = 32,768 (`--epoch-size` 4,096 and
262,144 give the epoch sweep), histogram threshold 64, alpha = 4.
`--workload skewed`: R-MAT graph with 2^20 vertices and edge factor 48
(a,b,c,d = .57,.19,.19,.05; ~44.4M undirected edges), colored by its
degree-sorted init stream, then a dense stream of 2,000,000 updates over the
k-core at the 90th percentile of core numbers (two inserts of non-adjacent
core pairs per delete). `--workload small`: Delaunay triangulation of 131,072
uniform points (seed 42) with the reference's 50/50 churn of 1,000,000 updates.

One step = one epoch: E updates applied concurrently (one warp per update)
followed by the repaired publish (compaction of edited rows, overflow drain,
fused rebuild + Tier-1 sweeps, Tier-2 when needed, double-buffered snapshot).
`value` times steps on the device with CUDA events on the library's stream,
inputs resident in HBM, L2 flushed (256 MiB write) before every timed step;
every published snapshot is validated between the timed steps. `e2e` times
the same steps through the C ABI from pinned host memory with the
host->device copy of each batch and the read-back of the step's counters
inside the timed region. Update-to-visible latency is the time from a batch's
submission through the C ABI (host memory) to the return of the publish that
makes it visible, over `--latency-epochs` further epochs.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "updates/sec on 1 B200 (plain vs batched/served); p50/p99 update-to-visible ms"
E = 32768
HIST_THR = 64
CORE_MIN_DEGREE = 256  # a graph loaded without its init stream: vertices colored one by one before the repair


def log(*a):
    print("[bench]", *a, file=sys.stderr, flush=True)


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def shared_workload(dist, rank, kind, stream_len, large_div):
    """Replicas on one node: rank 0 generates the workload and writes its
    arrays to /dev/shm; the other ranks map them read-only after a barrier.
    Returns the workload and the files to remove once every rank built its
    handle."""
    import streamgc_b200 as S
    tag = f"/dev/shm/sgc_{kind}_{large_div}_{os.environ.get('MASTER_PORT', '0')}"
    names = ["row_ptr", "col_idx", "degree", "stream"]
    if rank == 0:
        g, init, bench, desc = build_workload(kind, stream_len, large_div)
        for nm, arr in zip(names, [g.row_ptr, g.col_idx, g.degree, bench]):
            arr.tofile(f"{tag}_{nm}")
        with open(f"{tag}_desc.json", "w") as f:
            json.dump(desc, f)
    dist.barrier()
    if rank != 0:
        rp = np.memmap(f"{tag}_row_ptr", dtype=np.uint64, mode="r")
        col = np.memmap(f"{tag}_col_idx", dtype=np.uint32, mode="r")
        deg = np.memmap(f"{tag}_degree", dtype=np.uint32, mode="r")
        g = S.Graph(rp, col, deg)
        bench = np.fromfile(f"{tag}_stream", dtype=S.EDGE_UPDATE)
        desc = json.load(open(f"{tag}_desc.json"))
        init = None
    return g, init, bench, desc, [f"{tag}_{nm}" for nm in names] + [f"{tag}_desc.json"]


def build_workload(kind, stream_len, large_div=1):
    import streamgc_b200 as S
    t = time.time()
    if kind == "skewed":
        g = S.Graph.rmat(20, 48, 0.57, 0.19, 0.19, seed=42)
        bench, k, csize = g.kcore_stream(stream_len, 90.0, 42)
        desc = dict(workload="rmat20_ef48_kcore90_dense", graph="R-MAT scale 20, edge factor 48, (.57,.19,.19,.05), seed 42",
                    vertices=g.n, undirected_edges=g.nnz // 2, stream=f"k-core dense, {stream_len} updates, 2 inserts per delete, seed 42",
                    core_k=k, core_vertices=csize)
    elif kind == "large":
        nv = 65_608_366 // large_div  # large_div > 1: the same family scaled down (profiling captures)
        g = S.Graph.chung_lu(nv, 2.1, 55.0, 100_000.0, 42)
        bench = g.churn_stream(stream_len, 50, 42)
        desc = dict(workload="chunglu65m_churn" if large_div == 1 else f"chunglu65m_div{large_div}_churn",
                    graph=f"Chung-Lu, {nv:,} vertices, exponent 2.1, avg degree 55, cap 100,000, seed 42",
                    vertices=g.n, undirected_edges=g.nnz // 2, stream=f"churn 50% insert, {stream_len} updates, seed 42")
    else:
        g = S.Graph.delaunay(131072, seed=42)
        bench = g.churn_stream(stream_len, 50, 42)
        desc = dict(workload="delaunay17_churn", graph="Delaunay of 131072 uniform points, seed 42", vertices=g.n,
                    undirected_edges=g.nnz // 2, stream=f"churn 50% insert, {stream_len} updates, seed 42")
    # the large graph is colored from its loaded rows by one full repair: its
    # init stream (every edge, sorted by endpoint degrees) is 1.8 G updates
    init = None if kind == "large" else g.init_stream()
    desc.update(epoch_size=E, histogram_threshold=HIST_THR, alpha=4,
                init=(f"core of degree >= {CORE_MIN_DEGREE} colored one by one in descending degree order, then one "
                      "full repair of the loaded rows") if init is None else "init stream (every edge as an ADD)")
    log(f"workload {desc['workload']}: n={g.n} m={g.nnz // 2} init={0 if init is None else len(init)} "
        f"stream={len(bench)} ({time.time() - t:.1f}s)")
    return g, init, bench, desc


class ClockSampler:
    """nvidia-smi samples (200 ms) of SM clock and throttle reasons while running."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                       "-lms", "200", "-i", str(self.device)], stdout=subprocess.PIPE,
                                      stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.p = None
        return self

    def __exit__(self, *a):
        self.lines = []
        if self.p:
            time.sleep(0.25)
            self.p.terminate()
            try:
                out, _ = self.p.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.p.kill()
                out, _ = self.p.communicate()
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in getattr(self, "lines", []):
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for name, val in zip(names, f[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def read_row(profile, row):
    """A figure from a committed ncu summary under profiles/ (its
    `| row | value |` line), if present."""
    p = os.path.join(ROOT, "profiles", profile)
    try:
        for line in open(p):
            if line.startswith(f"| {row} |"):
                return float(line.split("|")[2])
    except (OSError, ValueError):
        pass
    return None


def read_traffic(profile, row):
    """A per-launch DRAM byte count from a committed ncu summary."""
    v = read_row(profile, row)
    return int(v) if v is not None else None


# The ncu summaries each workload's roofline traffic comes from.
# per workload: the apply capture, the per-epoch sweep capture, the full-sweep
# capture (the large workload's are taken on its family at 1/16 scale with the
# same epoch of 32,768 updates)
PROFILES = {
    "skewed": ("apply_skewed_rmat20.md", "sweep_items_skewed_rmat20.md", None),
    "large": ("apply_chunglu_div16.md", None, "sweep_full_chunglu_div16.md"),
    "small": (None, None, None),
}


def max_over_ranks(dist, values, device):
    """Element-wise maximum of per-rank timings over all ranks (every rank gets it)."""
    import torch
    t = torch.tensor(list(values), device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t]


def sum_over_ranks(dist, values, device):
    """Element-wise sum of per-rank counts over all ranks (every rank gets it)."""
    import torch
    t = torch.tensor(list(values), device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return [float(x) for x in t]


def dist_backend():
    """NCCL between GPU ranks; SGC_DIST_BACKEND=gloo runs the host-side
    reductions of the sharded forms on CPU ranks (tests)."""
    return os.environ.get("SGC_DIST_BACKEND", "nccl")


def reduce_device(local):
    return "cpu" if dist_backend() == "gloo" else f"cuda:{local}"


def init_dist(world):
    """The process group of a multi-rank run (short timeout), else None."""
    if world <= 1:
        return None
    import datetime
    import torch.distributed as dist
    dist.init_process_group(dist_backend(), timeout=datetime.timedelta(seconds=600))
    return dist


def job_rate(units_per_rank, world, seconds):
    """Whole-job throughput of `world` replicas timed by the slowest rank."""
    return world * units_per_rank / seconds


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def run_ours(a):
    import torch
    import streamgc_b200 as S

    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    dist = init_dist(world)
    nbatch = a.warmup + 2 * a.steps + a.cpu_batches + a.latency_epochs
    base_len = {"skewed": 2_000_000, "small": 1_000_000, "large": 10_000_000}[a.workload]
    stream_len = max(base_len, nbatch * E)
    if dist and a.workload == "large":  # one copy of the 1.8 G-edge graph in host memory for all ranks
        g, init, bench, desc, shm = shared_workload(dist, rank, a.workload, stream_len, a.large_div)
    else:
        g, init, bench, desc = build_workload(a.workload, stream_len, a.large_div)
        shm = []

    t = time.time()
    # no periodic full repair: every published snapshot is checked by the validator instead.
    # Profiling times the sweeps of eager repairs (the full repair after the run); a
    # captured publish runs its sweeps inside one graph launch.
    h = S.StreamGC(g, epoch_size=E, histogram_threshold=HIST_THR, slack_pct=300, max_batch=1 << 20,
                   device=local, profile=True, exact_select=True, graph_publish=a.graph_publish,
                   sorted_rows=a.sorted_rows, full_repair_every=a.full_repair_every)
    for s in range(0, 0 if init is None else len(init), 1 << 20):
        h.apply(init[s:s + (1 << 20)], S.MODE_CONCURRENT)
    t1 = time.time()
    core = h.color_core(CORE_MIN_DEGREE) if init is None else 0  # no init stream: the dense core first
    t2 = time.time()
    rep = h.publish()
    h.synchronize()
    if shm:  # every rank's handle holds its own copy now
        dist.barrier()
        if rank == 0:
            for f in shm:
                os.remove(f)
    log(f"init colored on GPU in {time.time() - t:.1f}s (handle {t1 - t:.1f}s, core of {core} vertices "
        f"{t2 - t1:.1f}s, full repair {time.time() - t2:.1f}s): {rep}")
    if not rep["proper"]:
        raise SystemExit("init coloring not proper")

    dev_stream = torch.from_numpy(bench.view(np.uint8)).to(f"cuda:{local}")
    dptr = dev_stream.data_ptr()
    ext = torch.cuda.ExternalStream(h.cuda_stream(), device=f"cuda:{local}")
    flush = torch.empty(64 << 20, dtype=torch.int32, device=f"cuda:{local}")  # 256 MiB > 126 MB L2
    pinned = torch.from_numpy(bench.view(np.uint8)).pin_memory()
    hptr = pinned.data_ptr()

    def step(ptr, b, mid=None):
        h.apply_ptr(ptr + b * E * 16, E, S.MODE_CONCURRENT)
        if mid is not None:
            mid.record(ext)  # end of the apply kernels on the handle's stream
        return h.publish()

    b = 0
    for _ in range(a.warmup):
        step(dptr, b)
        b += 1
    h.synchronize()
    st0 = h.stats()
    evs = []
    reps = []
    checks = []  # validator on each published snapshot, between the timed steps
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    if a.profile_window:
        torch.cuda.profiler.start()  # ncu --profile-from-start off captures the timed steps only
    with ClockSampler(local) as clk:
        for _ in range(a.steps):
            with torch.cuda.stream(ext):
                flush.add_(1)
            e0 = torch.cuda.Event(enable_timing=True)
            ea = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(ext)
            reps.append(step(dptr, b, ea))
            e1.record(ext)
            evs.append((e0, ea, e1))
            b += 1
            if a.validate_steps:
                ext.synchronize()
                v = h.validate()
                v["snapshot_is_colors"] = bool(np.array_equal(h.snapshot(), h.colors()))  # what queries read
                checks.append(v)
        ext.synchronize()
        torch.cuda.synchronize()
        if a.profile_window:
            torch.cuda.profiler.stop()
        step_ms = [x.elapsed_time(z) for x, _, z in evs]
        apply_ms = [x.elapsed_time(y) for x, y, _ in evs]
        st1 = h.stats()
        # e2e: same steps through the C ABI from pinned host memory, wall clock
        h.synchronize()
        d0 = h.stats()
        t0 = time.perf_counter()
        if a.ingest:  # the next batch's copy staged before this epoch's publish
            h.stage_ptr(hptr + b * E * 16, E)
        for k in range(a.steps):
            if a.ingest:
                h.apply_staged(S.MODE_CONCURRENT)
                if k + 1 < a.steps:
                    h.stage_ptr(hptr + (b + 1) * E * 16, E)
                h.publish()
            else:
                step(hptr, b)
            h.stats()  # the step's result read back to the host
            b += 1
        h.synchronize()
        e2e_s = time.perf_counter() - t0
        d1 = h.stats()
    # update-to-visible: a batch submitted from pinned host memory through the
    # C ABI until the publish that contains it has returned
    vis_ms = []
    for _ in range(a.latency_epochs):
        t0 = time.perf_counter()
        h.apply_ptr(hptr + b * E * 16, E, S.MODE_CONCURRENT)
        h.publish()
        h.synchronize()
        vis_ms.append(1e3 * (time.perf_counter() - t0))
        b += 1
    # one full repair after the run (every vertex swept; not in any timed figure): the
    # sweep kernels' bandwidth over the whole graph, and a last properness check
    fs0 = h.stats()
    if a.profile_full_sweep and a.profile_full_sweep_window:
        h.synchronize()
        torch.cuda.profiler.start()
    full_rep = h.repair() if a.profile_full_sweep else None
    if a.profile_full_sweep and a.profile_full_sweep_window:
        h.synchronize()
        torch.cuda.profiler.stop()
    fs1 = h.stats()
    total_ms = sum(step_ms)
    if dist:
        total_ms, e2e_s = max_over_ranks(dist, [total_ms, e2e_s], reduce_device(local))
    val = h.validate()
    cpu = None
    if rank == 0 and world == 1 and a.cpu_batches > 0:
        cpu = cpu_baseline(g, h, bench, b, a.cpu_batches, a.cpu_seconds)
    if rank == 0:
        updates = world * a.steps * E
        peak, peak_kind = load_peaks()
        sweep_ms = st1["sweep_ms"] - st0["sweep_ms"]
        sweep_bytes = st1["sweep_bytes"] - st0["sweep_bytes"]
        sweeps = st1["sweep_count"] - st0["sweep_count"]
        achieved = (sweep_bytes / (sweep_ms / 1e3) / 1e9) if sweep_ms > 0 else None
        apply_prof, sweep_prof, _ = PROFILES[a.workload] if E == 32768 else (None, None, None)
        traffic = read_traffic(sweep_prof, "sweep_dram_bytes_per_launch") if sweep_prof else None
        apply_traffic = read_traffic(apply_prof, "apply_dram_bytes_per_launch") if apply_prof else None
        apply_avg = sum(apply_ms) / len(apply_ms)
        bpu = cpu.pop("bytes_per_update", None) if cpu else None

        def pctl(v, q):
            v = sorted(v)
            return v[min(len(v) - 1, int(round(q * (len(v) - 1))))] if v else None
        pk = f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs, burst copy)" if peak_kind == "measured" else "fallback"
        roof_sweep = {"bound": "hbm", "kernel": "tier-1 sweep (sweep_items + finalize + fac + commit)",
                      "achieved": achieved, "peak": peak, "unit": "GB/s",
                      "frac": achieved / peak if achieved is not None else None, "peak_kind": pk,
                      "note": None if achieved is not None else "sweeps run inside the captured publish graph "
                              "and are not timed one by one; roofline_full_sweep times them over every vertex",
                      "traffic": traffic, "algorithmic_bytes_per_sweep": sweep_bytes / max(1, sweeps),
                      "sweep_ms_avg": sweep_ms / max(1, sweeps), "sweeps_timed": sweeps}
        roof_apply = None
        if bpu:  # the dominant kernel: algorithmic bytes per update under its own rules over the apply time
            ach = bpu * E / (apply_avg / 1e3) / 1e9
            roof_apply = {"bound": "hbm", "kernel": "concurrent apply (conc_prep_insert + conc_prep_prev + "
                          "conc_apply_kernel)", "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
                          "peak_kind": pk, "traffic": apply_traffic,
                          "algorithmic_bytes": "per update, the array elements the concurrent apply's rules read "
                          "and write (record; 32-ary base-run search and tail scan up to the high-water mark; "
                          "state, bitmap and degree words; recolor walk and early-exit reduce over the live "
                          "extent), counted by the oracle run under those rules on the CPU sample",
                          "algorithmic_bytes_per_launch": bpu * E, "apply_ms_avg": apply_avg}
        conf = dict(desc)
        conf.update(mode="concurrent (warp per edge) + repaired publish per epoch, exact color selection"
                    + (", publish as one CUDA graph" if a.graph_publish else "")
                    + (", e2e through the ingest slots" if a.ingest else "")
                    + (", rows kept as one sorted run" if a.sorted_rows else ""),
                    l2="flushed before every timed step (256 MiB write)", parallelism=f"replicas x{world}",
                    valid_after_run=val["violations"] == 0 and val["uncolored_with_edges"] == 0,
                    colors_used=int(val["max_color"]), static_greedy_colors=None,
                    tier1_sweeps_per_step=round(sweeps / max(1, a.steps), 2),
                    tier2_runs_in_timed=sum(r["tier2_ran"] for r in reps),
                    all_published_proper=all(r["proper"] for r in reps),
                    full_repair_every=a.full_repair_every,
                    snapshots_validated=len(checks),
                    snapshot_violations=sum(int(c["violations"]) + int(c["uncolored_with_edges"]) +
                                            (0 if c.get("snapshot_is_colors", True) else 1) for c in checks),
                    max_colors_in_timed=max((int(c["max_color"]) for c in checks), default=None),
                    reference_gpu=reference_gpu(a.workload))
        out = {
            "metric": METRIC, "value": job_rate(a.steps * E, world, total_ms / 1e3), "unit": "updates/s", "n_gpus": world,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": total_ms / a.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic", "config": conf,
            "latency_ms": {"update_to_visible_p50": pctl(vis_ms, 0.50), "update_to_visible_p99": pctl(vis_ms, 0.99),
                           "samples": len(vis_ms), "epoch_device_ms_p50": pctl(step_ms, 0.50),
                           "what": "per epoch of E updates: submit from pinned host memory through the C ABI to "
                                   "the return of the publish that makes it visible (wall clock)"},
            "roofline": roof_apply if roof_apply else roof_sweep,
            "roofline_sweep": roof_sweep,
            "roofline_full_sweep": full_sweep_roofline(fs0, fs1, full_rep, peak, pk, PROFILES[a.workload][2]),
            "apply": {"ms_per_epoch": apply_avg, "share_of_step": apply_avg / (total_ms / a.steps),
                      "algorithmic_bytes_per_update": bpu},
            "e2e": {"value": world * a.steps * E / e2e_s, "unit": "updates/s",
                    "h2d_bytes_per_step": (d1["h2d_bytes"] - d0["h2d_bytes"]) // a.steps,
                    "d2h_bytes_per_step": (d1["d2h_bytes"] - d0["d2h_bytes"]) // a.steps},
            "gpu_launches": st1["kernel_launches"] - st0["kernel_launches"],
            "clocks": clk.summary(),
            "cpu_baseline": cpu,
        }
        print(json.dumps(out), flush=True)
    h.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def full_sweep_roofline(s0, s1, rep, peak, peak_kind, profile=None):
    """The sweep kernels over every vertex (the full repair run after the
    timed steps): algorithmic bytes (8 per live entry + 28 per vertex) over
    their CUDA-event time. `traffic`: the DRAM bytes per algorithmic byte of
    a committed capture of the same sweep, times this sweep's algorithmic
    bytes."""
    if rep is None:
        return None
    ms = s1["sweep_ms"] - s0["sweep_ms"]
    by = s1["sweep_bytes"] - s0["sweep_bytes"]
    n = s1["sweep_count"] - s0["sweep_count"]
    if ms <= 0 or n <= 0:
        return None
    ach = by / (ms / 1e3) / 1e9
    ph = [b - a for a, b in zip(s0.get("sweep_phase_ms", [0] * 4), s1.get("sweep_phase_ms", [0] * 4))]
    ratio = read_row(profile, "full_sweep_dram_per_algorithmic") if profile else None
    return {"bound": "hbm", "kernel": "tier-1 sweep over every vertex (sweep_items + finalize + fac + commit)",
            "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak, "peak_kind": peak_kind,
            "algorithmic_bytes": by, "sweeps": n, "ms": ms, "proper": rep["proper"],
            "traffic": int(ratio * by) if ratio else None,
            "traffic_source": (f"profiles/{profile}: DRAM bytes per algorithmic byte x this sweep's bytes"
                               if ratio else None),
            "phases_ms": dict(zip(("item_build", "long_row_items", "finalize", "select_commit"), ph))}


def cpu_baseline(g, h, bench, first_batch, nb, budget_s):
    """The oracle (CPU restatement, OpenMP where order-independent) run under
    the concurrent configuration's rules, timed on the GPU's current state and
    the next batches of the same stream. The slot slab is downloaded straight
    into the oracle's own (one host copy of it, whatever the graph's size)."""
    from oracle import oracle as O
    import resource
    t = time.perf_counter()
    o = O.Oracle(g.row_ptr, g.col_idx, g.degree, hist_threshold=HIST_THR, exact=True, conc=True)
    ptr, nbytes = o.col_data()
    h.download_into("col", ptr, nbytes)
    o.load_state_inplace(g.row_ptr, g.col_idx, h.states(), h.bitmaps())
    o.load_rows_model(h.highwater(), h.base_runs(), h.holes())
    # the GPU's last publish was proper on mirror-complete rows: same repair rules from here
    o.set_repair_state(clean=True, asym=False)
    o.set_full_repair_every(0)  # as the GPU arm: no periodic full repair
    load_s = time.perf_counter() - t
    o.reset_bytes()
    done = 0
    t0 = time.perf_counter()
    for k in range(max(1, nb // 2)):  # all threads on the first half, one core on the second
        lo = (first_batch + k) * E
        if lo + E > len(bench):
            break
        o.process_stream_repaired(bench[lo:lo + E], E, E)
        done += 1
        if time.perf_counter() - t0 > budget_s:
            break
    dt = time.perf_counter() - t0
    bytes_update = o.counters()["bytes_update"]
    cores = int(O.lib().og_num_threads())
    # the same rules on one core: the next epochs, half the time budget
    O.lib().og_set_threads(1)
    done1 = 0
    t1 = time.perf_counter()
    for k in range(done, nb):
        lo = (first_batch + k) * E
        if lo + E > len(bench):
            break
        o.process_stream_repaired(bench[lo:lo + E], E, E)
        done1 += 1
        if time.perf_counter() - t1 > budget_s / 2:
            break
    dt1 = time.perf_counter() - t1
    O.lib().og_set_threads(cores)
    o.close()
    if not done:
        return None
    rss_gb = resource.getrusage(resource.RUSAGE_SELF).ru_maxrss / 2**20
    return {"value": done * E / dt, "unit": "updates/s", "cores": cores, "kind": "port",
            "bytes_per_update": bytes_update / (done * E),
            "single_core": ({"value": done1 * E / dt1, "cores": 1, "sample": f"{done1} further epochs of {E} updates"}
                            if done1 else None),
            "sample": f"{done} epochs of {E} updates following the GPU-timed ones, from the GPU's state, under the "
                      f"concurrent configuration's rules (updates in stream order + repaired epoch, {dt:.1f}s)",
            "host": host_facts(), "state_load_s": round(load_s, 1), "peak_rss_gb": round(rss_gb, 1)}


def host_facts():
    """CPU model, thread count and C++ runtime of this host (the stream
    generators call libstdc++'s distributions)."""
    model = None
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                model = line.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    libstdcxx = None
    for d in ("/usr/lib/x86_64-linux-gnu", "/usr/lib64", "/usr/lib"):
        try:
            names = sorted(f for f in os.listdir(d) if f.startswith("libstdc++.so.6."))
        except OSError:
            continue
        if names:
            libstdcxx = names[-1]
            break
    return {"cpu_model": model, "threads": os.cpu_count(), "libstdcxx": libstdcxx}


def reference_gpu(workload):
    """The reference's own kernels (built for sm_100a from its sources) on the
    same graph and stream: measured by oracle/ref_gpu_runs.py on a B200 and
    kept in tests/golden/ref_gpu_runs.json (profiles/reference_kernels_sm100a.md)."""
    if workload == "large":
        return {"unavailable": "the reference's row offsets are 32-bit (include/streamgc.cuh:56-58): its slack CSR "
                               "cannot address this graph's ~14.3 G slots"}
    name = {"small": "delaunay17_churn", "skewed": "rmat20_ef48_kcore90_dense"}[workload]
    try:
        r = json.load(open(os.path.join(ROOT, "tests", "golden", "ref_gpu_runs.json")))[name]
    except (OSError, KeyError, ValueError):
        return None
    return {"source": "tests/golden/ref_gpu_runs.json (oracle/ref_gpu_runs.py, one B200)",
            "bench_updates_per_s_wall": r["bench_updates_per_s"],
            "kernels_ms_per_epoch": r["apply_plus_epoch_ms_per_epoch"],
            "final_colors": r["final_colors"], "snapshots": "unrepaired at epochs; repaired at phase end"}


def run_reference(a):
    """The path's CPU restatement (the oracle: the reference has no CPU
    implementation of its own) on the same workload, under the same rules as
    the GPU arm (exact selection, independent-set repair, the concurrent
    apply's row layout), all host threads, one epoch of E updates plus its
    repaired publish per step. The large graph starts from a first-fit
    coloring of its rows (its init stream is 1.8 G updates); the others from
    their init streams."""
    world, rank, _ = dist_setup()
    if rank != 0:
        return
    from oracle import oracle as O
    stream_len = max({"skewed": 2_000_000, "small": 1_000_000, "large": 10_000_000}[a.workload],
                     (a.warmup + a.steps) * E)
    g, init, bench, desc = build_workload(a.workload, stream_len, a.large_div)
    t = time.time()
    o = O.Oracle(g.row_ptr, g.col_idx, g.degree, hist_threshold=HIST_THR, exact=True, conc=True)
    o.set_full_repair_every(a.full_repair_every)  # the GPU arm's repair cadence
    if init is None:
        colors = o.color_greedy()
        how = f"first-fit coloring of the loaded rows in id order ({colors} colors)"
    else:
        o.process_stream_repaired(init, len(init), len(init))
        how = "init stream (every edge as an ADD) + repaired publish"
    del g
    log(f"oracle initial coloring {time.time() - t:.1f}s: {how}")
    for k in range(a.warmup):
        o.process_stream_repaired(bench[k * E:(k + 1) * E], E, E)
    times = []
    for k in range(a.warmup, a.warmup + a.steps):
        t0 = time.perf_counter()
        o.process_stream_repaired(bench[k * E:(k + 1) * E], E, E)
        times.append(time.perf_counter() - t0)
    total = sum(times)
    v = a.steps * E / total
    cores = int(O.lib().og_num_threads())
    colors = int(o.colors().max())
    o.close()
    conf = dict(desc)
    conf.update(init=how, mode="CPU oracle under the concurrent configuration's rules (exact selection, "
                "independent-set repair, base runs with tombstones): updates in stream order + repaired epoch",
                parallelism="1 process", colors_after=colors)
    out = {"impl": "reference", "metric": METRIC, "value": v, "unit": "updates/s", "n_gpus": world,
           "steps": a.steps, "warmup": a.warmup, "ms_per_step": 1e3 * total / a.steps, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic", "config": conf,
           "cpu_baseline": {"value": v, "unit": "updates/s", "cores": cores, "kind": "port",
                            "sample": f"{a.steps} epochs of {E} updates after {a.warmup} warm-up epochs",
                            "host": host_facts()},
           "e2e": {"value": v, "unit": "updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
           "workload_generation": "the library's host-side generators (C++; no GPU is used by this arm)"}
    print(json.dumps(out), flush=True)


def run_batched(a):
    """Batched form: `--batch-graphs` seeded graphs (Delaunay / R-MAT / Chung-Lu,
    vertex counts log-uniform in [1,024, 2,097,152], epoch sizes in {1,024,
    8,192, 32,768}), each with its own churn stream (16x its edge count, the
    first ticks' worth generated). A tick submits one epoch of every graph. The
    same graphs and updates run twice: per-graph plain launches (one handle per
    graph: apply + publish per epoch) and the batched engine (one tick = one
    CUDA-graph launch). Both arms start from the same coloring of the loaded
    rows (each graph's core of degree >= CORE_MIN_DEGREE one vertex at a time,
    then a full repair) and are wall-clock timed from host memory."""
    import torch
    import streamgc_b200 as S
    from streamgc_b200 import workloads as W

    from streamgc_b200 import placement as P

    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    dev = reduce_device(local)
    dist = init_dist(world)
    ticks = a.warmup + a.steps
    specs_all = W.batch_specs(a.batch_graphs, seed=42)
    # independent graphs: each rank holds a share balanced by resident bytes
    share = P.place([P.spec_footprint(sp) for sp in specs_all], world)[rank]
    specs = [specs_all[i] for i in share]
    t = time.time()
    data = W.build_all(specs, lambda sp: (ticks + (16 if a.autotune else 0)) * sp["epoch"],
                       procs=max(1, min(8, (os.cpu_count() or 2) // world)))
    log(f"batched: {len(data)} graphs generated in {time.time() - t:.1f}s; "
        f"{sum(d['spec']['n'] for d in data)} vertices, {sum(int(d['row_ptr'][-1]) for d in data) // 2} edges")
    graphs = [S.Graph(d["row_ptr"], d["col"]) for d in data]
    epochs = [d["spec"]["epoch"] for d in data]

    def tick_parts(k, t_):
        ch = data[k]["churn"]
        lo = t_ * epochs[k]
        return ch[lo:lo + epochs[k]] if lo < len(ch) else None

    # ---- arm 1: per-graph plain launches ----
    t = time.time()
    hs = [S.StreamGC(gr, epoch_size=epochs[k], histogram_threshold=HIST_THR, slack_pct=300,
                     max_batch=max(epochs[k], 1 << 16), device=local, exact_select=True, full_repair_every=0)
          for k, gr in enumerate(graphs)]
    for h in hs:  # colored from its loaded rows (core first, then a full repair), as the batched arm is
        h.color_core(CORE_MIN_DEGREE)
        if not h.publish()["proper"]:
            raise SystemExit("plain arm init not proper")
        h.synchronize()
    torch.cuda.synchronize()
    log(f"plain arm: {len(hs)} handles created and colored in {time.time() - t:.1f}s")
    plain_ticks, plain_updates, plain_ok = [], 0, True
    if dist:
        dist.barrier()
    for t_ in range(ticks):
        t0 = time.perf_counter()
        n_up = 0
        for k, h in enumerate(hs):
            part = tick_parts(k, t_)
            if part is None or len(part) == 0:
                continue
            h.apply(part, S.MODE_CONCURRENT)
            r = h.publish()
            plain_ok &= r["proper"] == 1
            n_up += len(part)
        torch.cuda.synchronize()
        if t_ >= a.warmup:
            plain_ticks.append(time.perf_counter() - t0)
            plain_updates += n_up
    log(f"plain arm: {ticks} ticks in {time.time() - t:.1f}s since creation")
    plain_launches = sum(h.stats()["kernel_launches"] for h in hs)
    for h in hs:
        h.close()
    del hs
    torch.cuda.synchronize()

    # ---- arm 2: the batched engine ----
    t = time.time()
    cap = max(sum(epochs), 1 << 20)
    b = S.Batch(graphs, epoch_sizes=epochs, max_tick_updates=cap, device=local, profile=True,
                sorted_rows=a.sorted_rows)
    # the rows hold every edge from creation; the first tick colors all graphs
    # from scratch and publishes them (as the served form admits tenants)
    b.close_epochs()
    b.color_core(CORE_MIN_DEGREE)  # every graph's dense core first; the first tick repairs the rest
    if not b.tick()["proper"]:
        raise SystemExit("batched init not proper")
    log(f"batched arm: created and colored in {time.time() - t:.1f}s")
    tuning = b.tuning()
    tstate = {"t": 0}
    if a.autotune:
        def feed():
            for k in range(len(graphs)):
                part = tick_parts(k, tstate["t"])
                if part is not None and len(part):
                    b.submit(k, part)
            tstate["t"] += 1
        tuning = b.autotune(feed, ticks_per_candidate=1)
        log(f"tuner chose {tuning} in {tstate['t']} ticks")
    st0 = b.stats()
    lat, adm, dev_ms, b_updates, b_ok = [], [], [], 0, True
    base_t = tstate["t"]  # ticks the tuner consumed

    def submit_tick(t_):
        n_up = 0
        for k in range(len(graphs)):
            part = tick_parts(k, base_t + t_)
            if part is None or len(part) == 0:
                continue
            b.submit(k, part)
            n_up += len(part)
        return n_up

    if dist:
        dist.barrier()
    with ClockSampler(local) as clk:
        # the next tick's updates are staged while the current tick runs on the device
        sub_t = time.perf_counter()
        n_next = submit_tick(0)
        for t_ in range(ticks):
            if t_ == a.warmup:
                t_first = sub_t  # the first timed tick's updates were submitted here
            t0, n_up = sub_t, n_next
            ta = time.perf_counter()
            b.tick_begin()
            if t_ + 1 < ticks:
                sub_t = time.perf_counter()
                n_next = submit_tick(t_ + 1)
            r = b.tick_end()
            b_ok &= r["proper"] == 1
            if t_ >= a.warmup:
                tv = time.perf_counter()
                lat.append(tv - t0)  # submission to visibility
                adm.append(tv - ta)  # admission to the GPU (tick start) to visibility
                dev_ms.append(r["device_ms"])
                b_updates += n_up
        t_last = time.perf_counter()
    st1 = b.stats()
    val = b.validate()
    b.close()
    ls = sorted(lat)
    p50, p99 = ls[len(ls) // 2], ls[min(len(ls) - 1, int(round(0.99 * (len(ls) - 1))))]
    la = sorted(adm)
    a50, a99 = la[len(la) // 2], la[min(len(la) - 1, int(round(0.99 * (len(la) - 1))))]
    dev_p50 = sorted(dev_ms)[len(dev_ms) // 2]
    fam = {f: sum(1 for d in data if d["spec"]["family"] == f) for f in W.FAMILIES}
    nv = sum(d["spec"]["n"] for d in data)
    ne = sum(int(d["row_ptr"][-1]) for d in data) // 2
    ok = int(b_ok and plain_ok)
    valid = int(val["violations"] == 0 and val["uncolored_with_edges"] == 0)
    launches = st1["kernel_launches"] - st0["kernel_launches"]
    plain_time, batch_time = sum(plain_ticks), t_last - t_first
    if dist:  # every rank ran its own share: slowest rank's time, every rank's work
        plain_time, batch_time, p50, p99, a50, a99, dev_p50 = max_over_ranks(
            dist, [plain_time, batch_time, p50, p99, a50, a99, dev_p50], dev)
        sums = sum_over_ranks(dist, [plain_updates, b_updates, plain_launches, launches, nv, ne,
                                     *[fam[f] for f in W.FAMILIES]], dev)
        plain_updates, b_updates, plain_launches, launches, nv, ne = (int(x) for x in sums[:6])
        fam = {f: int(x) for f, x in zip(W.FAMILIES, sums[6:])}
        ok, valid = (int(x) for x in sum_over_ranks(dist, [ok, valid], dev))
        ok, valid = ok == world, valid == world
        dist.destroy_process_group()
        if rank != 0:
            return
    plain_v = plain_updates / plain_time
    batch_v = b_updates / batch_time
    out = {
        "metric": METRIC, "form": "batched", "value": batch_v, "unit": "updates/s", "n_gpus": world,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": 1e3 * batch_time / len(lat), "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
        "config": {"workload": f"batched_{len(specs_all)}_graphs", "families": fam,
                   "vertices": nv, "undirected_edges": ne,
                   "placement": f"{world} ranks, graphs balanced by resident bytes" if world > 1 else "one GPU",
                   "epoch_sizes": "per graph in {1024, 8192, 32768}", "tick": "one epoch of every graph",
                   "mode": "concurrent apply, independent-set repair, CUDA-graph tick", "tuning": tuning,
                   "autotuned": bool(a.autotune), "all_ticks_proper": bool(ok),
                   "valid_after_run": bool(valid)},
        "plain_per_graph": {"value": plain_v, "unit": "updates/s", "ms_per_tick": 1e3 * plain_time / len(plain_ticks),
                            "launches": plain_launches},
        "speedup_vs_plain": batch_v / plain_v,
        "latency_ms": {"update_to_visible_p50": 1e3 * p50, "update_to_visible_p99": 1e3 * p99,
                       "admission_to_visible_p50": 1e3 * a50, "admission_to_visible_p99": 1e3 * a99,
                       "tick_wall_ms": 1e3 * batch_time / len(lat), "tick_device_ms_p50": dev_p50,
                       "what": "update_to_visible: from a tick's submission (made while the previous tick runs) "
                               "to the end of the tick that publishes it; admission_to_visible: from the tick's "
                               "start on the GPU to that end"},
        "gpu_launches": launches,
        "clocks": clk.summary(),
    }
    print(json.dumps(out), flush=True)


def mirror_checksum(rp, col):
    """Sum over entries x->y of H(x,y) - H(y,x) (mod 2^64): 0 when every entry has its mirror."""
    n = len(rp) - 1
    x = np.repeat(np.arange(n, dtype=np.uint64), np.diff(rp.astype(np.int64)))
    y = col.astype(np.uint64)
    with np.errstate(over="ignore"):
        ha = ((x << np.uint64(32)) | y) * np.uint64(0x9E3779B97F4A7C15)
        hb = ((y << np.uint64(32)) | x) * np.uint64(0x9E3779B97F4A7C15)
        d = (ha ^ (ha >> np.uint64(29))).sum(dtype=np.uint64) - (hb ^ (hb >> np.uint64(29))).sum(dtype=np.uint64)
    return int(d)


def run_served(a):
    """Served form: 64 tenants (63 drawn as in the batched form, plus an R-MAT
    graph with 2^22 vertices and edge factor 16) behind the request loop. Each
    tenant's update requests arrive as a Poisson process at a rate proportional
    to its expected edge count, sizes log-uniform in [1, 32,768], 50/50
    insert/delete; single-vertex queries are 20% of the requests. A client
    thread replays the arrivals in real time (submits and queries), a second
    thread steps the server; the offered load is `--served-rate` updates/s over
    `--served-seconds`. Under torchrun every rank serves the tenants placed on
    its GPU (balanced by resident bytes) with their own arrivals."""
    import threading
    import torch
    import streamgc_b200 as S
    from streamgc_b200 import placement as P
    from streamgc_b200 import workloads as W

    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    dev = reduce_device(local)
    dist = init_dist(world)
    rate, dur = a.served_rate, a.served_seconds
    specs = W.batch_specs(63, seed=43)
    specs.append(dict(index=63, family="rmat22", n=1 << 22, edge_factor=16, epoch=32768, seed=43 * 100003 + 63))
    T = len(specs)
    est = [P.expected_entries(sp) for sp in specs]
    mine = P.place([P.footprint(sp["n"], e) for sp, e in zip(specs, est)], world)[rank]
    # arrivals of every tenant (the same on every rank), from expected sizes
    rng = np.random.default_rng(43)
    max_b = 32768
    mean_b = (max_b - 1) / math.log(max_b + 1)
    events = []
    need = [0] * T
    for k in range(T):
        req_rate = rate * est[k] / sum(est) / mean_b  # update requests per second of this tenant
        t_ = 0.0
        while True:
            t_ += rng.exponential(1.0 / (req_rate / 0.8))  # updates are 80% of the requests
            if t_ >= dur:
                break
            if rng.random() < 0.2:
                events.append((t_, k, 0, 0))
            else:
                m = int(min(max_b, math.floor(math.exp(rng.uniform(0.0, math.log(max_b + 1))))))
                m = max(1, m)
                events.append((t_, k, 1, m))
                need[k] += m
    events.sort()
    mset = set(mine)
    events = [e for e in events if e[1] in mset]

    t = time.time()
    small = [specs[k] for k in mine if k < T - 1]
    built = W.build_all(small, lambda sp: need[sp["index"]] + 1,
                        procs=max(1, min(8, (os.cpu_count() or 2) // world))) if small else []
    data = {d["spec"]["index"]: d for d in built}
    if T - 1 in mset:
        big = specs[-1]
        g22 = S.Graph.rmat(22, 16, 0.57, 0.19, 0.19, seed=big["seed"])
        data[T - 1] = dict(spec=big, row_ptr=g22.row_ptr, col=g22.col_idx,
                           churn=g22.churn_stream(need[T - 1] + 1, 50, big["seed"]))
    short = [k for k in mine if len(data[k]["churn"]) < need[k]]
    if short:
        raise SystemExit(f"served: churn streams of tenants {short} are shorter than their offered updates")
    log(f"served (rank {rank}): {len(mine)} of {T} tenants generated in {time.time() - t:.1f}s; "
        f"{len(events)} requests over {dur}s")
    srv = S.Server(hbm_budget_bytes=150 << 30, max_tick_updates=1 << 22, max_staleness_us=a.served_staleness_us,
                   device=local, profile=True, regrow=a.served_regrow, sorted_rows=a.sorted_rows)
    tids = {k: srv.add_tenant(S.Graph(data[k]["row_ptr"], data[k]["col"]), epoch_size=data[k]["spec"]["epoch"])
            for k in mine}
    t = time.time()
    r0 = srv.step()  # admission: every tenant colored and published
    log(f"admitted {r0['admitted']} tenants in {time.time() - t:.1f}s (proper={r0['proper']})")
    st0 = srv.stats()
    pos = {k: 0 for k in mine}
    stop = threading.Event()
    errors = []
    steps = []

    def stepper():
        try:
            while not stop.is_set():
                r = srv.step()
                if not r["proper"]:
                    raise RuntimeError("improper step")
                if r["groups_ticked"]:
                    steps.append(r["step_ms"])
                else:
                    time.sleep(0.0002)
        except Exception as e:
            errors.append(e)

    th = threading.Thread(target=stepper)
    qv = np.zeros(1, dtype=np.uint32)
    if dist:
        dist.barrier()
    with ClockSampler(local) as clk:
        th.start()
        t0 = time.perf_counter()
        late = 0.0
        for (te, k, kind, m) in events:
            now = time.perf_counter() - t0
            if te > now:
                time.sleep(te - now)
            else:
                late = max(late, now - te)
            if kind == 0:
                qv[0] = rng.integers(0, data[k]["spec"]["n"])
                srv.query(tids[k], qv)
            else:
                srv.submit(tids[k], data[k]["churn"][pos[k]:pos[k] + m])
                pos[k] += m
        t_sub = time.perf_counter() - t0
        deadline = time.time() + 60
        while time.time() < deadline:  # let every request become visible
            st = srv.stats()
            if st["requests_visible"] - st0["requests_visible"] >= st["update_requests"] - st0["update_requests"]:
                break
            time.sleep(0.01)
        t_end = time.perf_counter() - t0
        stop.set()
        th.join()
    if errors:
        raise SystemExit(f"served run failed: {errors[0]}")
    st = srv.stats()
    asym = None
    if a.served_check:  # every tenant's live rows must still hold each entry's mirror
        asym = [k for k in mine if mirror_checksum(*srv.rows(tids[k]))]
    srv.close()
    applied = st["updates_applied"] - st0["updates_applied"]
    ls = sorted(steps)
    step_p50 = ls[len(ls) // 2] if ls else 0.0
    step_p99 = ls[min(len(ls) - 1, int(round(0.99 * (len(ls) - 1))))] if ls else 0.0
    nv = sum(data[k]["spec"]["n"] for k in mine)
    ne = sum(int(data[k]["row_ptr"][-1]) for k in mine) // 2
    cnt = [applied, len(events), sum(1 for e in events if e[2] == 0), st["resident_bytes"], nv, ne,
           st["ticks"] - st0["ticks"], st["tier2_ticks"] - st0["tier2_ticks"],
           st["tier2_mirror_ticks"] - st0["tier2_mirror_ticks"], st["tier1_sweeps"] - st0["tier1_sweeps"],
           st["tick_device_ms"] - st0["tick_device_ms"], sum(need[k] for k in mine), st["overflows"],
           st["drain_failed"], st["device_errors"], len(steps), sum(steps), st["tenants_regrown"]]
    worst = [t_end, t_sub, late, st["visible_p50_ms"], st["visible_p99_ms"], st["query_p50_ms"], st["query_p99_ms"],
             step_p50, step_p99]
    if dist:  # tenants on every rank: every rank's work, the slowest rank's times and latencies
        cnt = sum_over_ranks(dist, cnt, dev)
        worst = max_over_ranks(dist, worst, dev)
        if asym is not None:
            flags = sum_over_ranks(dist, [1.0 if k in asym else 0.0 for k in range(T)], dev)
            asym = [k for k in range(T) if flags[k]]
        dist.destroy_process_group()
        if rank != 0:
            return
    (applied, nreq, nq, resident, nv, ne, ticks, t2, t2m, sweeps, tick_ms, offered, ovf, dfail, derr,
     nsteps, steps_ms, regrown) = cnt
    t_end, t_sub, late, v50, v99, q50, q99, step_p50, step_p99 = worst
    out = {
        "metric": METRIC, "form": "served", "value": applied / t_end, "unit": "updates/s", "n_gpus": world,
        "steps": int(nsteps), "warmup": 1, "ms_per_step": steps_ms / max(1, nsteps), "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
        "config": {"workload": "served_64_tenants", "offered_updates_per_s": rate, "seconds": dur,
                   "tenants": T, "vertices": int(nv), "undirected_edges": int(ne),
                   "placement": f"{world} ranks, tenants balanced by resident bytes" if world > 1 else "one GPU",
                   "requests": int(nreq), "queries": int(nq),
                   "batch_sizes": "log-uniform [1, 32768]", "arrival_rate": "proportional to expected edges",
                   "max_staleness_us": a.served_staleness_us,
                   "hbm_budget_gb": 150, "resident_gb": round(resident / 2**30, 2),
                   "client_max_lag_s": round(late, 4), "submit_window_s": round(t_sub, 3),
                   "timed_s": round(t_end, 3), "ticks": int(ticks), "tier2_ticks": int(t2),
                   "tier2_mirror_ticks": int(t2m), "sweeps_per_tick": round(sweeps / max(1, ticks), 2),
                   "tick_device_ms_total": round(tick_ms, 1), "offered_updates": int(offered),
                   "overflows": int(ovf), "drain_failed": int(dfail), "device_errors": int(derr),
                   "asymmetric_tenants": asym, "regrow": bool(a.served_regrow), "tenants_regrown": int(regrown)},
        "latency_ms": {"update_to_visible_p50": v50, "update_to_visible_p99": v99,
                       "query_p50": q50, "query_p99": q99, "step_p50": step_p50, "step_p99": step_p99},
        "clocks": clk.summary(),
    }
    print(json.dumps(out), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=24)
    ap.add_argument("--warmup", type=int, default=4)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="large", choices=["skewed", "small", "large"],
                    help="plain path: skewed (R-MAT 2^20 x 48, k-core stream), small (Delaunay 2^17 churn), "
                         "large (Chung-Lu 65.6 M vertices, ~1.8 G edges, 10 M churn)")
    ap.add_argument("--sorted-rows", action="store_true",
                    help="compaction keeps rows of up to 1024 live entries as one sorted run (SGC_OPT_SORTED_ROWS)")
    ap.add_argument("--ingest", action="store_true",
                    help="plain path, e2e: batches staged through the two ingest slots (copy of the next "
                         "batch overlapping this epoch's publish)")
    ap.add_argument("--eager-publish", dest="graph_publish", action="store_false",
                    help="plain path: publish with one host round trip per repair sweep instead of replaying "
                         "the captured publish graph (SGC_OPT_GRAPH_PUBLISH, the default)")
    ap.add_argument("--graph-publish", dest="graph_publish", action="store_true", help=argparse.SUPPRESS)
    ap.add_argument("--epoch-size", type=int, default=32768,
                    help="plain path: updates per epoch (the large workload's sweep uses 4096, 32768, 262144)")
    ap.add_argument("--cpu-batches", type=int, default=8, help="epochs timed on the CPU baseline (0: skip)")
    ap.add_argument("--no-full-sweep", dest="profile_full_sweep", action="store_false",
                    help="plain path: skip the full repair after the run (its sweep bandwidth is reported)")
    ap.add_argument("--full-repair-every", type=int, default=0,
                    help="plain path: every k-th publish repairs every vertex (0: only when the incremental rule "
                         "cannot be used); every published snapshot is validated either way")
    ap.add_argument("--large-div", type=int, default=1,
                    help="large workload scaled down by this factor (same family; for profiling captures)")
    ap.add_argument("--latency-epochs", type=int, default=128,
                    help="plain path: epochs timed one by one from submission to visibility after the e2e steps")
    ap.add_argument("--no-validate-steps", dest="validate_steps", action="store_false",
                    help="plain path: skip the validator on each published snapshot between timed steps")
    ap.add_argument("--cpu-seconds", type=float, default=20.0)
    ap.add_argument("--profile-window", action="store_true",
                    help="bracket the device-timed steps with cudaProfilerStart/Stop (for ncu)")
    ap.add_argument("--profile-full-sweep-window", action="store_true",
                    help="bracket the full repair after the run with cudaProfilerStart/Stop instead (for ncu)")
    ap.add_argument("--form", default="plain", choices=["plain", "batched", "served"],
                    help="plain: one graph (the headline); batched: many graphs per tick; served: request loop")
    ap.add_argument("--batch-graphs", type=int, default=256)
    ap.add_argument("--autotune", action="store_true", help="batched: run the tuner on the warm-up ticks first")
    ap.add_argument("--served-rate", type=float, default=20e6, help="served: offered updates per second")
    ap.add_argument("--served-seconds", type=float, default=8.0)
    ap.add_argument("--served-staleness-us", type=int, default=2000)
    ap.add_argument("--served-check", action="store_true", help="served: check every tenant's rows for mirrors after the run")
    ap.add_argument("--served-regrow", action="store_true",
                    help="served: re-admit tenants whose rows dropped entries, with rebuilt rows")
    a = ap.parse_args()
    global E
    E = a.epoch_size
    if a.workload == "large" and "--cpu-seconds" not in sys.argv:
        a.cpu_seconds = 30.0
    if a.warmup < 3:
        raise SystemExit("--warmup must be >= 3")
    if a.impl == "reference":
        run_reference(a)
    elif a.form == "batched":
        run_batched(a)
    elif a.form == "served":
        run_served(a)
    else:
        run_ours(a)


if __name__ == "__main__":
    main()
