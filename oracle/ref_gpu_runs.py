"""TEST INFRASTRUCTURE: the reference's own kernels, compiled for sm_100a from
the reference sources (oracle/_ref/ref_driver), run at their own launch shape
(one warp per update, 256-thread blocks; algorithms/streamgc/src/streamgc.cu:847-853)
through the reference's full single-GPU protocol on the plain workloads:
init stream, drain_and_compact, phase-end Tier-1 loop and Tier-2, bench stream
with epoch steps every 32,768 updates, drain_and_compact, Tier-1, Tier-2.

Prints one JSON object per workload: the reference's bench-stream time (wall
clock, as its bench_stream_ms), CUDA-event time of its local_update_kernel
launches and of its epoch steps, and the color count and violations of its
final coloring. These are the GPU bar and the color bound the library's
concurrent configuration is compared with.

    python oracle/ref_gpu_runs.py OUT_DIR [small] [skewed]   # on a GPU box
"""
from __future__ import annotations

import json
import os
import struct
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

E = 32768
THR = 64


def workload(kind):
    """The bench's plain workloads (same generators, seeds and sizes)."""
    import streamgc_b200 as S
    if kind == "small":
        g = S.Graph.delaunay(131072, seed=42)
        bench = g.churn_stream(1_000_000, 50, 42)
        name = "delaunay17_churn"
    else:
        g = S.Graph.rmat(20, 48, 0.57, 0.19, 0.19, seed=42)
        bench, _, _ = g.kcore_stream(2_000_000, 90.0, 42)
        name = "rmat20_ef48_kcore90_dense"
    return name, g, g.init_stream(), bench


def case_file(path, g, init, bench):
    n = g.n
    hdr = struct.pack("<IQIIIIQQ", n, g.nnz, THR, E, E, 300, len(init), len(bench))
    with open(path, "wb") as f:
        f.write(hdr)
        f.write(g.row_ptr.astype("<u4").tobytes())
        f.write(g.col_idx.astype("<u4").tobytes())
        f.write(g.degree.astype("<u4").tobytes())
        f.write(init.tobytes())
        f.write(bench.tobytes())


def records(path):
    out = {}
    data = open(path, "rb").read()
    i = 0
    cur = None
    while i < len(data):
        tag = data[i:i + 16].split(b"\0", 1)[0].decode()
        (nb,) = struct.unpack("<Q", data[i + 16:i + 24])
        payload = data[i + 24:i + 24 + nb]
        i += 24 + nb
        if nb == 0:
            cur = tag
        else:
            out[(cur, tag)] = payload
    return out


def run(out_dir, kinds):
    driver = os.path.join(ROOT, "oracle", "_ref", "ref_driver")
    os.makedirs(out_dir, exist_ok=True)
    res = {}
    for kind in kinds:
        t = time.time()
        name, g, init, bench = workload(kind)
        cin = os.path.join(out_dir, f"ref_{kind}.bin")
        cout = os.path.join(out_dir, f"ref_{kind}.dump")
        case_file(cin, g, init, bench)
        gen_s = time.time() - t
        t = time.time()
        p = subprocess.run([driver, "--in", cin, "--out", cout, "--launch", "ref", "--repair", "--no-dump"],
                           capture_output=True, text=True)
        run_s = time.time() - t
        if p.returncode != 0:
            raise SystemExit(f"ref_driver failed on {kind}: {p.stdout[-2000:]} {p.stderr[-2000:]}")
        r = records(cout)
        fin = struct.unpack("<4d", r[("final", "values")])
        ms = struct.unpack("<12d", r[("timing", "ms")])
        os.remove(cin)
        os.remove(cout)
        epochs = int(ms[6])
        res[name] = {
            "vertices": g.n, "undirected_edges": g.nnz // 2, "init_updates": len(init), "bench_updates": len(bench),
            "epoch_size": E, "histogram_threshold": THR, "launch": "local_update_kernel<<<ceil(32n/256), 256>>> "
            "(one warp per update), epoch steps and repair kernels at thread per vertex",
            "init_ms": ms[0], "bench_stream_ms": ms[1], "bench_updates_per_s": len(bench) / (ms[1] / 1e3),
            "bench_apply_kernel_ms": ms[3], "bench_epoch_kernels_ms": ms[4], "bench_epoch_wall_ms": ms[5],
            "bench_epochs": epochs,
            "apply_plus_epoch_ms_per_epoch": (ms[3] + ms[4]) / max(1, epochs),
            "tier1_iterations": [ms[7], ms[8]], "tier2_fixed": [ms[9], ms[10]], "bench_phase_repair_ms": ms[11],
            "final_colors": int(fin[0]), "final_violations": int(fin[1]), "final_uncolored_with_edges": int(fin[2]),
            "final_edges": int(fin[3]), "generate_s": gen_s, "run_s": run_s,
        }
        print(json.dumps({name: res[name]}), flush=True)
    with open(os.path.join(out_dir, "ref_gpu_runs.json"), "w") as f:
        json.dump(res, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    if len(sys.argv) < 2:
        raise SystemExit(__doc__)
    run(sys.argv[1], sys.argv[2:] or ["small", "skewed"])
