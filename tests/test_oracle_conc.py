"""The oracle under the concurrent apply's rules (sorted base runs with
tombstones, tail inserts, reads bounded by the high-water mark, lazy
compaction, early-exit color reduction), in stream order: the same live edge
set as the stream-order rules, proper repaired epochs, and byte counts that
only cover the slots those rules read."""
import numpy as np
import pytest

from oracle import oracle as O
from tests.golden import make_golden as MG


def _live_edges(o):
    rp = o.row_ptr()
    col = o.col()
    n = len(rp) - 1
    x = np.repeat(np.arange(n, dtype=np.int64), np.diff(rp.astype(np.int64)))
    keep = col < n  # free slots and tombstones hold no vertex id
    return set(zip(x[keep].tolist(), col[keep].tolist()))


@pytest.mark.parametrize("name", ["delaunay2k", "rmat11"])
def test_concurrent_rules_keep_the_edge_set_and_publish_proper_epochs(name):
    c = MG.build_case(name)
    runs = {}
    for conc in (False, True):
        o = O.Oracle(c["rp"], c["col"], c["deg"], hist_threshold=c["thr"], exact=True, conc=conc)
        o.process_stream_repaired(c["init"], len(c["init"]), len(c["init"]))
        reps = []
        o.reset_bytes()
        for s in range(0, len(c["bench"]), c["E"]):
            o.apply(c["bench"][s:s + c["E"]])
            reps.append(o.publish_repair())
        runs[conc] = (o, reps, o.counters()["bytes_update"])
    (a, ra, ba), (b, rb, bb) = runs[False], runs[True]
    assert _live_edges(a) == _live_edges(b)
    assert all(r["proper"] for r in ra + rb)
    v = O.validate_colors(b.row_ptr(), b.col(), b.colors())
    assert v["violations"] == 0 and v["uncolored_with_edges"] == 0
    assert int(b.colors().max()) <= int(a.colors().max()) + 4
    assert ba > 0 and bb > 0
    a.close()
    b.close()


def test_concurrent_rules_bytes_do_not_depend_on_slack():
    """Every read under the concurrent rules stops at a row's high-water mark,
    so more slack (and no overflow either way) leaves the bytes per update
    unchanged; the stream-order rules scan whole capacities and count more."""
    c = MG.build_case("delaunay2k")
    got = {}
    for conc in (False, True):
        for slack in (300, 700):
            o = O.Oracle(c["rp"], c["col"], c["deg"], hist_threshold=c["thr"], slack_pct=slack, exact=True,
                         conc=conc)
            o.process_stream_repaired(c["init"], len(c["init"]), len(c["init"]))
            o.reset_bytes()
            o.process_stream_repaired(c["bench"], c["E"], c["E"])
            k = o.counters()
            assert k["overflow_lost"] == 0 and k["drain_failed"] == 0
            got[conc, slack] = (k["bytes_update"], o.colors())
            o.close()
    assert got[True, 300][0] == got[True, 700][0]
    assert np.array_equal(got[True, 300][1], got[True, 700][1])
    assert got[False, 700][0] > got[False, 300][0]
