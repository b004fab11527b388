"""Host-side rules of the exact-selection repair, on the oracle (no GPU): the
incremental repair (first sweep over the vertices touched since the last
repair) leaves every published coloring proper, runs only when the last repair
ended proper on mirror-complete rows, and a full repair comes every Nth time
or whenever it is forced."""
import numpy as np
import pytest

from oracle import oracle as O
from tests.golden import make_golden as MG


def _publish_all(g, c):
    reps = []
    for ups in (c["init"], c["bench"]):
        for s in range(0, len(ups), c["batch"]):
            g.apply(ups[s:s + c["batch"]])
            reps.append(g.publish_repair())
            v = O.validate_colors(g.row_ptr(), g.col(), g.snapshot())
            assert v["violations"] == 0 and v["uncolored_with_edges"] == 0
    return reps


@pytest.mark.parametrize("name", ["delaunay2k", "rmat11"])
def test_incremental_repairs_keep_every_snapshot_proper(name):
    c = MG.build_case(name)
    g = O.Oracle(c["rp"], c["col"], c["deg"], hist_threshold=c["thr"], slack_pct=c["slack"], exact=True)
    g.set_full_repair_every(0)  # full only when required
    reps = _publish_all(g, c)
    assert all(r["proper"] for r in reps)
    assert reps[0]["incremental"] == 0  # nothing known yet: the first repair is full
    assert sum(r["incremental"] for r in reps[1:]) == len(reps) - 1


def test_full_repair_cadence():
    c = MG.build_case("delaunay2k")
    g = O.Oracle(c["rp"], c["col"], c["deg"], hist_threshold=c["thr"], slack_pct=c["slack"], exact=True)
    g.set_full_repair_every(3)
    reps = _publish_all(g, c)
    pattern = [r["incremental"] for r in reps]
    # full, then two incremental repairs per full one
    assert pattern[:7] == [0, 1, 1, 0, 1, 1, 0]


def test_planted_colors_force_a_full_repair():
    c = MG.build_case("rmat11")
    g = O.Oracle(c["rp"], c["col"], c["deg"], hist_threshold=c["thr"], slack_pct=c["slack"], exact=True)
    g.set_full_repair_every(0)
    g.apply(c["init"][:c["batch"]])
    assert g.publish_repair()["incremental"] == 0
    g.apply(c["init"][c["batch"]:2 * c["batch"]])
    assert g.publish_repair()["incremental"] == 1
    st = np.random.default_rng(3).integers(0, 5, size=len(c["deg"])).astype(np.uint32)
    g.set_states(st)  # colors from elsewhere
    rep = g.publish_repair()
    assert rep["incremental"] == 0 and rep["proper"] == 1
    assert g.publish_repair(force_full=True)["incremental"] == 0


def test_overflowing_rows_force_full_repairs_until_mirrored():
    """Rows that overflowed may miss mirror entries: repairs stay full (with the
    checksum) until a full repair finds the rows mirror-complete again."""
    c = MG.build_case("overflow512")
    g = O.Oracle(c["rp"], c["col"], c["deg"], hist_threshold=c["thr"], slack_pct=c["slack"], exact=True)
    g.set_full_repair_every(0)
    reps = _publish_all(g, c)
    assert all(r["proper"] for r in reps)
    assert g.counters()["drain_failed"] > 0 or g.counters()["overflow_lost"] > 0 or \
        any(r["incremental"] == 0 for r in reps[1:])
