"""The plain workloads at their full sizes through the concurrent
configuration, against the reference's own kernels run on the same graphs and
streams (tests/golden/ref_gpu_runs.json, written by oracle/ref_gpu_runs.py on
a B200: the reference's launch shape, epoch steps and phase-end Tier-1/Tier-2).

Every snapshot published at an epoch boundary is proper, and the final
coloring uses at most the reference's final color count + COLOR_SLACK."""
import json
import os

import numpy as np
import pytest

import bench
import streamgc_b200 as S

pytestmark = pytest.mark.gpu

REF = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "ref_gpu_runs.json")))
COLOR_SLACK = 4
E = 32768


@pytest.mark.parametrize("kind, stream_len", [("small", 1_000_000), ("skewed", 2_000_000)])
def test_full_size_run_proper_and_within_reference_colors(kind, stream_len):
    g, init, ups, desc = bench.build_workload(kind, stream_len)
    ref = REF[desc["workload"]]
    assert (ref["vertices"], ref["undirected_edges"], ref["bench_updates"]) == (g.n, g.nnz // 2, len(ups))
    with S.StreamGC(g, epoch_size=E, histogram_threshold=64, max_batch=1 << 20, exact_select=True) as h:
        for s in range(0, len(init), 1 << 20):
            h.apply(init[s:s + (1 << 20)], S.MODE_CONCURRENT)
        assert h.publish()["proper"] == 1
        worst = 0
        for s in range(0, len(ups), E):
            h.apply(ups[s:s + E], S.MODE_CONCURRENT)
            rep = h.publish()
            v = h.validate()
            assert rep["proper"] == 1 and v["violations"] == 0 and v["uncolored_with_edges"] == 0, (s, v)
            worst = max(worst, int(v["max_color"]))
        h.drain_and_compact()
        rep = h.publish()
        v = h.validate()
        assert rep["proper"] == 1 and v["violations"] == 0
        colors = int(h.colors().max())
    assert ref["final_violations"] == 0
    assert colors <= ref["final_colors"] + COLOR_SLACK, (colors, ref["final_colors"])
    assert worst <= ref["final_colors"] + COLOR_SLACK
