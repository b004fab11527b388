"""Many graphs on one GPU (include/streamgc_batch.h): the batched engine
against the oracle and against itself.

  - stream-order mode: each graph's published colors are the same alone, in
    the mix, and in the oracle (exact selection, incremental repairs);
  - the captured CUDA-graph tick and the eager tick give the same colors;
  - concurrent mode: every tick's coloring is proper, per graph, on the
    graph's own live rows;
  - the tuner runs on live ticks and leaves the results proper;
  - queries answer from the published snapshot."""
import numpy as np
import pytest

import streamgc_b200 as S
from oracle import oracle as O
from tests.golden import make_golden as MG

pytestmark = pytest.mark.gpu

NAMES = ["delaunay2k", "rmat11", "overflow512"]
E = 1024  # updates per tick and per epoch for every graph


def _cases():
    return [MG.build_case(n) for n in NAMES]


def _graph(c):
    return S.Graph(c["rp"], c["col"], c["deg"])


def _ticks(c, count):
    ups = np.concatenate([c["init"], c["bench"]])
    return [ups[s:s + E] for s in range(0, min(len(ups), count * E), E)]


def _proper_on_rows(b, k, snap):
    rp, col = b.rows(k)
    v = O.validate_colors(rp, col, snap)
    return v["violations"] == 0 and v["uncolored_with_edges"] == 0


def test_stream_order_alone_mixed_and_oracle_agree():
    cases = _cases()
    T = 10
    sched = [_ticks(c, T) for c in cases]
    thr = [c["thr"] for c in cases]
    mixed = S.Batch([_graph(c) for c in cases], epoch_sizes=[E] * len(cases), thresholds=thr, stream_order=True)
    alone = [S.Batch([_graph(c)], epoch_sizes=[E], thresholds=[c["thr"]], stream_order=True) for c in cases]
    oracles = []
    for c in cases:
        o = O.Oracle(c["rp"], c["col"], c["deg"], hist_threshold=c["thr"], slack_pct=300, exact=True)
        o.set_full_repair_every(0)
        oracles.append(o)
    try:
        for t in range(T):
            for k, c in enumerate(cases):
                part = sched[k][t] if t < len(sched[k]) else None
                if part is None or len(part) == 0:
                    continue
                mixed.submit(k, part)
                alone[k].submit(0, part)
                oracles[k].apply(part)
            rm = mixed.tick()
            assert rm["proper"] == 1
            for k, c in enumerate(cases):
                ra = alone[k].tick()
                assert ra["proper"] == 1
                if t < len(sched[k]) and len(sched[k][t]) == E:
                    oracles[k].publish_repair()
                    sm, sa = mixed.snapshot(k), alone[k].snapshot(0)
                    so = oracles[k].snapshot()
                    assert np.array_equal(sm, sa), (NAMES[k], t)
                    assert np.array_equal(sm, so), (NAMES[k], t)
                    assert _proper_on_rows(mixed, k, sm)
        assert mixed.stats()["device_error"] == 0
    finally:
        mixed.close()
        for a in alone:
            a.close()
        for o in oracles:
            o.close()


def test_cuda_graph_tick_equals_eager_tick():
    cases = _cases()
    T = 6
    sched = [_ticks(c, T) for c in cases]
    thr = [c["thr"] for c in cases]
    kw = dict(epoch_sizes=[E] * len(cases), thresholds=thr, stream_order=True)
    bg = S.Batch([_graph(c) for c in cases], cuda_graph=True, **kw)
    be = S.Batch([_graph(c) for c in cases], cuda_graph=False, **kw)
    try:
        for t in range(T):
            for k in range(len(cases)):
                if t < len(sched[k]):
                    bg.submit(k, sched[k][t])
                    be.submit(k, sched[k][t])
            rg, re_ = bg.tick(), be.tick()
            assert rg["proper"] == re_["proper"] == 1
            assert rg["tier1_iterations"] == re_["tier1_iterations"]
            for k in range(len(cases)):
                assert np.array_equal(bg.snapshot(k), be.snapshot(k))
    finally:
        bg.close()
        be.close()


def test_concurrent_ticks_publish_proper_colorings():
    cases = _cases()
    T = 10
    sched = [_ticks(c, T) for c in cases]
    b = S.Batch([_graph(c) for c in cases], epoch_sizes=[E] * len(cases), thresholds=[c["thr"] for c in cases])
    try:
        for t in range(T):
            for k in range(len(cases)):
                if t < len(sched[k]):
                    b.submit(k, sched[k][t])
            r = b.tick()
            assert r["proper"] == 1
            for k in range(len(cases)):
                assert _proper_on_rows(b, k, b.snapshot(k)), (NAMES[k], t)
        assert b.validate()["violations"] == 0
        assert b.stats()["device_error"] == 0
    finally:
        b.close()


def test_autotune_runs_on_live_ticks():
    cases = _cases()
    sched = [_ticks(c, 40) for c in cases]
    b = S.Batch([_graph(c) for c in cases], epoch_sizes=[E] * len(cases), profile=True)
    state = {"t": 0}

    def feed():
        t = state["t"]
        for k in range(len(cases)):
            if t < len(sched[k]):
                b.submit(k, sched[k][t])
        state["t"] = t + 1

    try:
        chosen = b.autotune(feed, ticks_per_candidate=1)
        assert chosen["repair_tile"] in (256, 512, 1024, 2048)
        assert chosen["apply_blocks_per_sm"] >= 1
        feed()
        assert b.tick()["proper"] == 1
        for k in range(len(cases)):
            assert _proper_on_rows(b, k, b.snapshot(k))
    finally:
        b.close()


def test_query_reads_the_published_snapshot():
    c = MG.build_case("rmat11")
    b = S.Batch([_graph(c), _graph(c)], epoch_sizes=[E, 2 * E])
    try:
        parts = _ticks(c, 3)
        b.submit(0, parts[0])
        b.submit(1, parts[0])
        b.tick()  # graph 0 publishes (E reached), graph 1 does not yet
        v = np.arange(0, len(c["deg"]), 7, dtype=np.uint32)
        assert np.array_equal(b.query(0, v), b.snapshot(0)[v])
        assert not b.snapshot(1).any()
        b.submit(1, parts[1])
        b.tick()
        assert b.snapshot(1).any()
        assert np.array_equal(b.query(1, v), b.snapshot(1)[v])
        bad = b.query(1, np.array([len(c["deg"]) + 5], dtype=np.uint32))
        assert bad[0] == 0
    finally:
        b.close()


def test_submits_during_a_tick_stage_the_next_one():
    """With the tick split (begin / end), the next tick's updates are submitted
    while the current tick runs; in stream order the snapshots equal those of
    submit-then-tick."""
    cases = _cases()
    T = 8
    sched = [_ticks(c, T) for c in cases]
    thr = [c["thr"] for c in cases]
    a = S.Batch([_graph(c) for c in cases], epoch_sizes=[E] * len(cases), thresholds=thr, stream_order=True)
    b = S.Batch([_graph(c) for c in cases], epoch_sizes=[E] * len(cases), thresholds=thr, stream_order=True)

    def submit(batch, t):
        for k in range(len(cases)):
            part = sched[k][t] if t < len(sched[k]) else None
            if part is not None and len(part):
                batch.submit(k, part)

    try:
        submit(b, 0)
        for t in range(T):
            submit(a, t)
            ra = a.tick()
            b.tick_begin()
            if t + 1 < T:
                submit(b, t + 1)  # staged while tick t runs
            rb = b.tick_end()
            assert ra["proper"] == rb["proper"] == 1 and ra["updates"] == rb["updates"]
            for k in range(len(cases)):
                assert np.array_equal(a.snapshot(k), b.snapshot(k)), (NAMES[k], t)
    finally:
        a.close()
        b.close()
