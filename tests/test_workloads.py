"""Workload generators of the batched and served forms (host only): seeded
spec lists, graph families, churn streams as prefixes, and the init stream."""
import numpy as np

import streamgc_b200 as S
from streamgc_b200 import workloads as W


def test_specs_are_seeded_and_in_range():
    a = W.batch_specs(64, seed=7)
    b = W.batch_specs(64, seed=7)
    assert a == b
    assert a != W.batch_specs(64, seed=8)
    assert [s["index"] for s in a] == list(range(64))
    for s in a:
        assert s["family"] in W.FAMILIES
        assert 1024 <= s["n"] <= 2_097_152
        assert s["epoch"] in (1024, 8192, 32768)
    # a longer list starts with the shorter one
    assert W.batch_specs(80, seed=7)[:64] == a


def test_induce_keeps_the_subgraph():
    g = S.Graph.rmat(8, 8, 0.57, 0.19, 0.19, seed=3)
    rp, col = W.induce(g.row_ptr, g.col_idx, 100)
    assert len(rp) == 101 and int(rp[-1]) == len(col)
    assert col.size == 0 or int(col.max()) < 100
    # every kept entry was an entry of the original rows
    full = {(u, int(v)) for u in range(100) for v in g.col_idx[g.row_ptr[u]:g.row_ptr[u + 1]] if v < 100}
    kept = {(u, int(v)) for u in range(100) for v in col[rp[u]:rp[u + 1]]}
    assert kept == full


def test_build_all_orders_by_spec_and_streams_are_prefixes():
    specs = [dict(index=0, family="delaunay", n=1500, epoch=1024, seed=11),
             dict(index=1, family="rmat", n=900, epoch=1024, seed=12),
             dict(index=2, family="chung_lu", n=1200, epoch=1024, seed=13)]
    short = W.build_all(specs, lambda sp: 500, procs=2)
    full = W.build_all(specs, lambda sp: None, procs=2)
    for s, d, f in zip(specs, short, full):
        assert d["spec"] is s
        assert np.array_equal(d["row_ptr"], f["row_ptr"]) and np.array_equal(d["col"], f["col"])
        m = int(f["row_ptr"][-1]) // 2
        assert len(f["churn"]) == 16 * m
        assert len(d["churn"]) == 500
        assert np.array_equal(d["churn"], f["churn"][:500])
        init = W.init_stream(d)
        assert len(init) == m
