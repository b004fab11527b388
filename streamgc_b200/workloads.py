"""Synthetic workloads of the batched and served forms: many seeded graphs of
uneven sizes (Delaunay, R-MAT, Chung-Lu) with their own churn streams.

Each graph's family, vertex count (log-uniform) and epoch size come from a
generator seeded with (seed, index), so a spec list is reproducible. Graphs
are generated in worker processes (spawned, before any CUDA use in them).
"""
import math
import multiprocessing as mp
import os

import numpy as np

FAMILIES = ("delaunay", "rmat", "chung_lu")


def batch_specs(count=256, seed=42, n_lo=1024, n_hi=2_097_152, epochs=(1024, 8192, 32768)):
    """One spec per graph: family uniform over the three, vertex count
    log-uniform in [n_lo, n_hi], epoch size uniform over `epochs`."""
    specs = []
    for i in range(count):
        rng = np.random.default_rng([seed, i])
        fam = FAMILIES[int(rng.integers(3))]
        n = int(round(math.exp(rng.uniform(math.log(n_lo), math.log(n_hi)))))
        specs.append(dict(index=i, family=fam, n=n, epoch=int(rng.choice(epochs)), seed=seed * 100003 + i))
    return specs


def induce(row_ptr, col, n):
    """The subgraph on vertices [0, n)."""
    rp = np.asarray(row_ptr, dtype=np.uint64)[: n + 1]
    c = np.asarray(col, dtype=np.uint32)[: int(rp[-1])]
    keep = c < n
    owner = np.repeat(np.arange(n, dtype=np.int64), np.diff(rp).astype(np.int64))
    cnt = np.bincount(owner[keep], minlength=n).astype(np.uint64)
    out_rp = np.zeros(n + 1, dtype=np.uint64)
    np.cumsum(cnt, out=out_rp[1:])
    return out_rp, np.ascontiguousarray(c[keep])


def make_graph(spec):
    """(row_ptr, col) of a spec's graph. R-MAT: edge factor 48, (a,b,c) =
    (.57,.19,.19), generated at the next power of two and restricted to the
    first n vertices; Chung-Lu: exponent 2.1, average degree 17, degrees capped
    at 100,000."""
    import streamgc_b200 as S
    n, seed = spec["n"], spec["seed"]
    if spec["family"] == "delaunay":
        g = S.Graph.delaunay(n, seed=seed)
        return g.row_ptr, g.col_idx
    if spec["family"] == "rmat":
        scale = max(1, math.ceil(math.log2(n)))
        g = S.Graph.rmat(scale, 48, 0.57, 0.19, 0.19, seed=seed)
        if g.n == n:
            return g.row_ptr, g.col_idx
        return induce(g.row_ptr, g.col_idx, n)
    g = S.Graph.chung_lu(n, 2.1, 17.0, 100000.0, seed)
    return g.row_ptr, g.col_idx


def _build(args):
    spec, stream_len = args
    import streamgc_b200 as S
    rp, col = make_graph(spec)
    g = S.Graph(rp, col)
    m = int(rp[-1]) // 2
    size = min(16 * m, stream_len) if stream_len is not None else 16 * m
    churn = g.churn_stream(max(size, 0), 50, spec["seed"])
    return spec["index"], rp, col, churn


def build_all(specs, stream_len_of, procs=None):
    """Graphs and churn streams for every spec, in worker processes.

    Each churn stream is 16x the graph's edge count; stream_len_of(spec)
    bounds it (None: no bound), and a shorter stream is a prefix of a longer
    one. Returns a list of dicts (spec, row_ptr, col, churn) in spec order; a
    graph's init stream (every edge as an ADD) comes from init_stream(d) when
    needed."""
    procs = procs or max(1, min(8, (os.cpu_count() or 2)))
    order = sorted(specs, key=lambda s: -s["n"])
    jobs = [(s, stream_len_of(s)) for s in order]
    pos = {s["index"]: i for i, s in enumerate(specs)}
    out = [None] * len(specs)
    ctx = mp.get_context("spawn")
    with ctx.Pool(procs) as pool:
        for idx, rp, col, churn in pool.imap_unordered(_build, jobs):
            out[pos[idx]] = dict(spec=specs[pos[idx]], row_ptr=rp, col=col, churn=churn)
    return out


def init_stream(d):
    """Every edge of a built graph as an ADD, in the reference's init order."""
    import streamgc_b200 as S
    return S.Graph(d["row_ptr"], d["col"]).init_stream()
