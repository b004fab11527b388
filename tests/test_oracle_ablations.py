"""The reference's ablation builds (its Makefile abl-* targets) as oracle
options: what each one changes, on the golden cases."""
import numpy as np

from oracle import oracle as O
from tests.golden import make_golden as MG


def _run(c, ablations=()):
    o = O.Oracle(c["rp"], c["col"], c["deg"], hist_threshold=c["thr"], slack_pct=c["slack"], ablations=ablations)
    o.process_stream(c["init"], c["E"], c["batch"])
    o.phase_end()
    o.process_stream(c["bench"], c["E"], c["batch"])
    ovf = o.overflow_count()
    it, last, fixed = o.phase_end()
    return o, ovf


def test_no_overflow_drops_inserts_instead_of_buffering():
    c = MG.build_case("overflow512")
    base, base_ovf = _run(c)
    abl, ovf = _run(c, ("no_overflow",))
    k = abl.counters()
    assert base_ovf > 0  # the default build buffers them for the drain
    assert ovf == 0 and k["overflow_lost"] == 0 and k["drain_failed"] == 0
    v = O.validate_colors(abl.row_ptr(), abl.col(), abl.colors())
    assert v["violations"] == 0 and v["uncolored_with_edges"] == 0


def test_force_bitmap_changes_how_histogram_rows_choose():
    c = MG.build_case("rmat11")
    assert int((c["deg"] > c["thr"]).sum()) > 0
    base, _ = _run(c)
    abl, _ = _run(c, ("force_bitmap",))
    assert not np.array_equal(base.states(), abl.states())
    v = O.validate_colors(abl.row_ptr(), abl.col(), abl.colors())
    assert v["violations"] == 0 and v["uncolored_with_edges"] == 0


def test_live_degree_priority_only_changes_tier1():
    """Updates use the frozen priority in both builds: states before the first
    phase end are identical; Tier-1 differs once live degrees drift."""
    c = MG.build_case("rmat11")
    a = O.Oracle(c["rp"], c["col"], c["deg"], hist_threshold=c["thr"])
    b = O.Oracle(c["rp"], c["col"], c["deg"], hist_threshold=c["thr"], ablations=("live_deg",))
    for o in (a, b):
        o.process_stream(c["init"], c["E"], c["batch"])
    assert np.array_equal(a.states(), b.states())
    for o in (a, b):
        o.phase_end()
        o.process_stream(c["bench"], c["E"], c["batch"])
        o.phase_end()
    v = O.validate_colors(b.row_ptr(), b.col(), b.colors())
    assert v["violations"] == 0 and v["uncolored_with_edges"] == 0
