"""Row layout invariants on the device (sgc_check_state): after every batch,
publish and tick the rows of a handle keep their high-water marks inside the
row capacity, only free slots past the mark, vertex ids in range, a sorted
base run (exact selection) or sorted never-edited rows, hole counters that
never wrap, and colors in range; in stream order and in concurrent batches.
Then the stream-ingest slots against direct applies, and the captured-graph
publish."""
import time

import numpy as np
import pytest

import streamgc_b200 as S
from tests.golden import make_golden as MG

pytestmark = pytest.mark.gpu

NAMES = ["delaunay2k", "rmat11", "overflow512"]


def _clean(rep):
    return rep["bad_rows"] == 0 and rep["flags"] == 0 and rep["first_bad"] == 0xFFFFFFFF


@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("exact", [False, True])
def test_rows_keep_their_invariants(name, exact):
    c = MG.build_case(name)
    g = S.Graph(c["rp"], c["col"], c["deg"])
    ups = np.concatenate([c["init"], c["bench"]])
    with S.StreamGC(g, epoch_size=c["E"], histogram_threshold=c["thr"], slack_pct=c["slack"],
                    exact_select=exact) as h:
        rep = h.check_state()
        assert rep["rows"] == len(c["rp"]) - 1
        assert _clean(rep), rep
        mode = S.MODE_CONCURRENT if exact else S.MODE_DETERMINISTIC
        B = 2048
        for i, s in enumerate(range(0, len(ups), B)):
            h.apply(ups[s:s + B], mode)
            assert _clean(h.check_state()), (i, h.check_state())
            if i % 4 == 3:
                if exact:
                    assert h.publish()["proper"] == 1
                else:
                    h.epoch()
                assert _clean(h.check_state()), (i, "after epoch", h.check_state())


def test_batched_rows_keep_their_invariants():
    cases = [MG.build_case(n) for n in NAMES]
    E = 1024
    b = S.Batch([S.Graph(c["rp"], c["col"], c["deg"]) for c in cases], epoch_sizes=[E] * len(cases),
                thresholds=[c["thr"] for c in cases])
    try:
        assert _clean(b.check_state())
        scheds = [np.concatenate([c["init"], c["bench"]]) for c in cases]
        for t in range(12):
            for k, u in enumerate(scheds):
                part = u[t * E:(t + 1) * E]
                if len(part):
                    b.submit(k, part)
            assert b.tick()["proper"] == 1
            assert _clean(b.check_state()), (t, b.check_state())
    finally:
        b.close()


@pytest.mark.parametrize("name", ["delaunay2k", "overflow512"])
def test_staged_batches_match_direct_applies(name):
    """Stream ingest (sgc_stage / sgc_apply_staged): in stream order, batches
    staged ahead (two slots, the next one copied before the current epoch
    ends) give the same colors and rows as the same batches applied directly."""
    c = MG.build_case(name)
    ups = np.concatenate([c["init"], c["bench"]])
    B = c["batch"]
    parts = [ups[s:s + B] for s in range(0, len(ups), B)]
    kw = dict(epoch_size=c["E"], histogram_threshold=c["thr"], slack_pct=c["slack"], max_batch=max(B, 1024))
    with S.StreamGC(S.Graph(c["rp"], c["col"], c["deg"]), **kw) as a, \
            S.StreamGC(S.Graph(c["rp"], c["col"], c["deg"]), **kw) as b:
        b.stage(parts[0])
        for i, p in enumerate(parts):
            a.apply(p, S.MODE_DETERMINISTIC)
            if i + 1 < len(parts):
                b.stage(parts[i + 1])  # copied while batch i is applied
            b.apply_staged(S.MODE_DETERMINISTIC)
            if i % 3 == 2:
                a.epoch()
                b.epoch()
                assert np.array_equal(a.colors(), b.colors()), i
        assert np.array_equal(a.states(), b.states())
        assert np.array_equal(a.col(), b.col())
        with pytest.raises(S.StreamGCError):
            b.apply_staged(S.MODE_DETERMINISTIC)  # nothing staged


def test_sorted_rows_keep_one_run():
    """SGC_OPT_SORTED_ROWS: after a forced compaction every row of at most 1024
    live entries is one strictly ascending run; publishes stay proper and the
    rows keep their invariants."""
    c = MG.build_case("rmat11")
    g = S.Graph(c["rp"], c["col"], c["deg"])
    ups = np.concatenate([c["init"], c["bench"]])
    with S.StreamGC(g, epoch_size=c["E"], histogram_threshold=c["thr"], slack_pct=c["slack"],
                    exact_select=True, sorted_rows=True) as h:
        for s in range(0, len(ups), 2048):
            h.apply(ups[s:s + 2048], S.MODE_CONCURRENT)
            assert h.publish()["proper"] == 1
            assert _clean(h.check_state())
        h.drain_and_compact()
        assert _clean(h.check_state())
        rp, hw, col = h.row_ptr(), h.highwater(), h.col()
        for x in range(len(hw)):
            if hw[x] <= 1024:
                run = col[rp[x]:rp[x] + hw[x]].astype(np.int64)
                assert np.all(np.diff(run) > 0), x


@pytest.mark.parametrize("name", ["delaunay2k", "rmat11"])
def test_graph_publish_is_proper_and_keeps_invariants(name):
    """The captured-graph publish (SGC_OPT_GRAPH_PUBLISH): every published
    snapshot proper, the rows' invariants kept, the same counters advancing as
    with the eager publish."""
    c = MG.build_case(name)
    g = S.Graph(c["rp"], c["col"], c["deg"])
    ups = np.concatenate([c["init"], c["bench"]])
    with S.StreamGC(g, epoch_size=c["E"], histogram_threshold=c["thr"], slack_pct=c["slack"],
                    exact_select=True, graph_publish=True) as h:
        B = 2048
        for i, s in enumerate(range(0, len(ups), B)):
            h.apply(ups[s:s + B], S.MODE_CONCURRENT)
            rep = h.publish()
            assert rep["proper"] == 1, (i, rep)
            assert rep["tier1_iterations"] >= 1
            assert _clean(h.check_state()), (i, h.check_state())
            snap = h.snapshot()
            assert np.array_equal(snap, h.colors())  # the published half holds the current colors
        v = h.validate()
        assert v["violations"] == 0 and v["uncolored_with_edges"] == 0
        st = h.stats()
        assert st["epochs"] >= len(ups) // B and st["tier1_sweeps"] >= st["epochs"]


def test_ingest_ring_matches_direct_applies():
    """A producer thread feeds the stream into a ring smaller than the stream
    (it wraps around many times; pushes that do not fit are retried); the
    stepping thread lets the GPU drain it one host batch at a time, in stream
    order. States, bitmaps and rows equal direct applies of the same batches."""
    import threading
    c = MG.build_case("rmat11")
    ups = np.concatenate([c["init"], c["bench"]])
    batch = 2048
    g = S.Graph(c["rp"], c["col"], c["deg"])
    with S.StreamGC(g, epoch_size=c["E"], histogram_threshold=c["thr"], max_batch=batch) as a, \
            S.StreamGC(g, epoch_size=c["E"], histogram_threshold=c["thr"], max_batch=batch) as b:
        b.ring_create(12)  # 4,096 slots
        done = threading.Event()

        def produce():
            pos = 0
            while pos < len(ups):
                k = b.ring_push(ups[pos:pos + 3000])
                pos += k
                if k == 0:
                    time.sleep(0.0002)
            done.set()

        th = threading.Thread(target=produce)
        th.start()
        applied = 0
        for s0 in range(0, len(ups), batch):
            part = ups[s0:s0 + batch]
            a.apply(part, S.MODE_DETERMINISTIC)
            got = 0
            while got < len(part):
                k = b.ring_apply(len(part) - got, S.MODE_DETERMINISTIC)
                if k == 0:
                    time.sleep(0.0002)
                got += k
            assert got == len(part)
            applied += got
            if (s0 // batch) % 4 == 3:
                a.epoch()
                b.epoch()
        th.join(30)
        assert done.is_set() and applied == len(ups)
        assert b.ring_apply(batch, S.MODE_DETERMINISTIC) == 0
        for name in ("states", "bitmaps", "col", "hist"):
            assert np.array_equal(getattr(a, name)(), getattr(b, name)()), name
        assert b.stats()["h2d_bytes"] >= 16 * len(ups)
