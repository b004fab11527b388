"""CUDA path vs the oracle (and the reference's own kernels via the golden
epoch hashes): bit-exact for every integer array at every epoch boundary."""
import json
import os

import numpy as np
import pytest

import streamgc_b200 as S
from oracle import oracle as O
from tests import _util
from tests.golden import make_golden as MG

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", list(MG.CASES))
def test_deterministic_mode_matches_oracle_every_epoch(name):
    c = MG.build_case(name)
    ora = list(_util.oracle_epochs(c))
    gpu = list(_util.gpu_epochs(c, S.MODE_DETERMINISTIC))
    assert [t for t, _ in ora] == [t for t, _ in gpu]
    for (tag, a), (_, b) in zip(ora, gpu):
        for k in _util.ARRAY_NAMES:
            if not np.array_equal(a[k], b[k]):
                bad = np.nonzero(a[k] != b[k])[0][:8]
                pytest.fail(f"{name} {tag} {k}: first differing indices {bad.tolist()} "
                            f"oracle={a[k][bad].tolist()} gpu={b[k][bad].tolist()}")


@pytest.mark.skipif(not os.path.exists(MG.GOLDEN_JSON), reason="golden epoch fixtures not generated yet")
@pytest.mark.parametrize("name", list(MG.CASES))
def test_deterministic_mode_matches_reference_kernels(name):
    gold = json.load(open(MG.GOLDEN_JSON))[name]
    c = MG.build_case(name)
    n = 0
    for tag, arrays in _util.gpu_epochs(c, S.MODE_DETERMINISTIC):
        for k in _util.ARRAY_NAMES:
            assert _util.sha(arrays[k]) == gold["epochs"][tag][k], f"{name} {tag} {k}"
        n += 1
    assert n == len(gold["epochs"])


@pytest.mark.skipif(not os.path.exists(MG.GOLDEN_SCALE_JSON), reason="full-size epoch fixtures not generated yet")
@pytest.mark.parametrize("name", list(MG.SCALE_CASES))
def test_deterministic_mode_matches_reference_kernels_full_size(name):
    """Delaunay 2^17 with the 1 M-update churn stream, E = 32,768: every state
    array equals the reference's kernels' at all 43 epoch boundaries."""
    gold = json.load(open(MG.GOLDEN_SCALE_JSON))[name]
    c = MG.build_case(name)
    n = 0
    for tag, arrays in _util.gpu_epochs(c, S.MODE_DETERMINISTIC):
        for k in _util.ARRAY_NAMES:
            assert _util.sha(arrays[k]) == gold["epochs"][tag][k], f"{name} {tag} {k}"
        n += 1
    assert n == len(gold["epochs"]) == 43


def _both(name):
    c = MG.build_case(name)
    g = O.Oracle(c["rp"], c["col"], c["deg"], hist_threshold=c["thr"], slack_pct=c["slack"])
    h = S.StreamGC(S.Graph(c["rp"], c["col"], c["deg"]), epoch_size=c["E"], histogram_threshold=c["thr"],
                   slack_pct=c["slack"], max_batch=c["batch"])
    return c, g, h


@pytest.mark.parametrize("name", list(MG.CASES))
def test_phase_end_repair_matches_oracle(name):
    """Reference epochs during each phase, then drain_and_compact + Tier-1
    (Jacobi) + Tier-2 at phase end: bit-exact states, bitmaps and CSR."""
    c, g, h = _both(name)
    try:
        for ups in (c["init"], c["bench"]):
            g.process_stream(ups, c["E"], c["batch"])
            since = 0
            for s in range(0, len(ups), c["batch"]):
                part = ups[s:s + c["batch"]]
                h.apply(part)
                since += len(part)
                if since >= c["E"]:
                    h.epoch()
                    since = 0
            it, last, fixed = g.phase_end()
            rep = h.repair()
            assert (rep["tier1_iterations"], rep["tier1_last_count"]) == (it, last)
            assert rep["tier2_fixed"] == fixed
            assert np.array_equal(h.states(), g.states())
            assert np.array_equal(h.bitmaps(), g.bitmaps())
            assert np.array_equal(h.col(), g.col())
            v, w = h.validate(), g.validate()
            assert v == w, (v, w)
            assert v["violations"] == 0
    finally:
        h.close()
        g.close()


@pytest.mark.parametrize("name", ["rmat11", "delaunay2k", "rmat11_thr16_a2"])
def test_independent_set_repair_matches_oracle(name):
    """Exact selection + independent-set Tier-1 (the concurrent configuration's
    repair) on planted conflicts: bit-exact with the oracle (Tier-1 sweeps,
    counts, Tier-2 fixes, states, bitmaps) and proper at the end. Random colors
    from a 6-color palette on a dense graph can need more sweeps than Tier-1
    allows; Tier-2 then finishes, identically on both sides."""
    c = MG.build_case(name)
    g = O.Oracle(c["rp"], c["col"], c["deg"], hist_threshold=c["thr"], slack_pct=c["slack"], exact=True)
    h = S.StreamGC(S.Graph(c["rp"], c["col"], c["deg"]), histogram_threshold=c["thr"], slack_pct=c["slack"],
                   exact_select=True)
    try:
        st = np.random.default_rng(11).integers(0, 6, size=len(c["deg"])).astype(np.uint32)
        g.set_states(st)
        h.upload("states", st)
        it, last, fixed = g.phase_end()
        rep = h.repair()
        assert (rep["tier1_iterations"], rep["tier1_last_count"], rep["tier2_fixed"]) == (it, last, fixed)
        # the loop ends when nothing is left to visit; Tier-2 runs only after 64 unconverged sweeps
        assert rep["proper"] == 1 and rep["tier2_ran"] == (1 if fixed else 0)
        assert np.array_equal(h.states(), g.states())
        assert np.array_equal(h.bitmaps(), g.bitmaps())
        assert h.validate()["violations"] == 0
    finally:
        h.close()
        g.close()


@pytest.mark.parametrize("name", ["delaunay2k", "rmat11", "overflow512"])
def test_incremental_publish_matches_oracle(name):
    """Exact selection, updates in stream order, one publish per batch: the
    incremental repairs (first sweep over the touched vertices, pushes to
    losing neighbors, bitmap hints) and the full ones every 4th repair give
    states, bitmaps and repair reports bit-exact with the oracle, and every
    published snapshot is proper."""
    c = MG.build_case(name)
    g = O.Oracle(c["rp"], c["col"], c["deg"], hist_threshold=c["thr"], slack_pct=c["slack"], exact=True)
    g.set_full_repair_every(4)
    h = S.StreamGC(S.Graph(c["rp"], c["col"], c["deg"]), epoch_size=c["E"], histogram_threshold=c["thr"],
                   slack_pct=c["slack"], max_batch=c["batch"], exact_select=True, full_repair_every=4)
    try:
        seen_incr = 0
        for ups in (c["init"], c["bench"]):
            for s in range(0, len(ups), c["batch"]):
                part = ups[s:s + c["batch"]]
                h.apply(part, S.MODE_DETERMINISTIC)
                g.apply(part)
                rep = h.publish()
                ora = g.publish_repair()
                for k in ("tier1_iterations", "tier1_last_count", "incremental", "tier2_ran", "proper",
                          "tier2_fixed"):
                    assert rep[k] == ora[k], (k, rep, ora)
                assert rep["proper"] == 1
                seen_incr += rep["incremental"]
                assert np.array_equal(h.states(), g.states())
                assert np.array_equal(h.bitmaps(), g.bitmaps())
                v = O.validate_colors(h.row_ptr(), h.col(), h.snapshot())
                assert v["violations"] == 0 and v["uncolored_with_edges"] == 0
        # rows that overflow may miss mirror entries: those repairs stay full
        assert seen_incr > 0 or h.stats()["overflow_pending"] + h.stats()["drain_failed"] + \
            h.stats()["overflow_lost"] > 0 or name == "overflow512"
        assert h.stats()["device_error"] == 0
    finally:
        h.close()
        g.close()


def test_tier2_exact_on_forced_conflicts():
    """Conflicts planted in the state: Tier-1 alone vs the oracle, then Tier-2."""
    c = MG.build_case("rmat11")
    g = O.Oracle(c["rp"], c["col"], c["deg"], hist_threshold=c["thr"])
    h = S.StreamGC(S.Graph(c["rp"], c["col"], c["deg"]), histogram_threshold=c["thr"])
    try:
        rng = np.random.default_rng(5)
        st = (rng.integers(0, 4, size=len(c["deg"]))).astype(np.uint32)  # colors 0..3: many conflicts
        g.set_states(st)
        h.upload("states", st)
        it, last, fixed = g.phase_end()
        rep = h.repair()
        assert (rep["tier1_iterations"], rep["tier1_last_count"], rep["tier2_fixed"]) == (it, last, fixed)
        assert np.array_equal(h.states(), g.states())
        assert h.validate()["violations"] == g.validate()["violations"]
    finally:
        h.close()
        g.close()


COLOR_SLACK = 4  # concurrent mode may use at most this many colors above the sequential reference


@pytest.mark.parametrize("exact", [True, False])
@pytest.mark.parametrize("name", ["delaunay2k", "rmat11", "overflow512"])
def test_concurrent_mode_publishes_proper_snapshots(name, exact):
    """Concurrent batches: every published snapshot is proper on the live CSR,
    the edge multiset per row equals the sequential one, and -- with exact
    color selection, the concurrent configuration -- colors stay within the
    sequential reference's count + COLOR_SLACK. (With the reference's drifting
    histograms the count depends on the interleaving, so only properness holds.)"""
    c = MG.build_case(name)
    g = O.Oracle(c["rp"], c["col"], c["deg"], hist_threshold=c["thr"], slack_pct=c["slack"])
    h = S.StreamGC(S.Graph(c["rp"], c["col"], c["deg"]), epoch_size=c["E"], histogram_threshold=c["thr"],
                   slack_pct=c["slack"], max_batch=c["batch"], exact_select=exact)
    try:
        g.process_stream_repaired(c["init"], c["E"], c["batch"])
        for ups in (c["init"], c["bench"]):
            for s in range(0, len(ups), c["batch"]):
                h.apply(ups[s:s + c["batch"]], S.MODE_CONCURRENT)
                rep = h.publish()
                assert rep["proper"] == 1
                snap = h.snapshot()
                assert np.array_equal(snap, h.colors())  # the published half holds the current colors
                v = O.validate_colors(h.row_ptr(), h.col(), snap)
                assert v["violations"] == 0 and v["uncolored_with_edges"] == 0
        g.process_stream_repaired(c["bench"], c["E"], c["batch"])
        g.drain_and_compact()
        h.drain_and_compact()
        oracle_colors = int(g.colors().max())
        # same live edge multiset per row as the sequential oracle, unless a full
        # row made an insert wait in the overflow buffer and then drop (which edge
        # loses the last slot depends on the order the inserts arrive in)
        st, oc = h.stats(), g.counters()
        no_drop = st["drain_failed"] == 0 and st["overflow_lost"] == 0 and oc["drain_failed"] == 0 \
            and oc["overflow_lost"] == 0
        gr, gc = h.row_ptr(), h.col()
        orp, ocol = g.row_ptr(), g.col()
        for x in range(len(c["deg"]) if no_drop else 0):
            a = np.sort(gc[gr[x]:gr[x + 1]])
            b = np.sort(ocol[orp[x]:orp[x + 1]])
            assert np.array_equal(a, b), f"row {x}"
        if exact:
            assert int(h.colors().max()) <= oracle_colors + COLOR_SLACK
        assert h.stats()["device_error"] == 0
    finally:
        h.close()
        g.close()


def test_validator_matches_oracle_on_improper_state():
    c = MG.build_case("overflow512")
    g = O.Oracle(c["rp"], c["col"], c["deg"])
    h = S.StreamGC(S.Graph(c["rp"], c["col"], c["deg"]))
    try:
        st = np.random.default_rng(1).integers(0, 3, size=len(c["deg"])).astype(np.uint32)
        g.set_states(st)
        h.upload("states", st)
        assert h.validate() == g.validate()
    finally:
        h.close()
        g.close()


def test_core_coloring_then_full_repair_matches_oracle():
    """A loaded power-law graph colored without an init stream: the high-degree
    core one vertex at a time (sgc_color_core), then one full repair. States
    equal the oracle's after each step; the result is proper."""
    g = S.Graph.chung_lu(30000, 2.1, 17.0, 3000.0, 11)
    o = O.Oracle(g.row_ptr, g.col_idx, g.degree, hist_threshold=64, exact=True)
    h = S.StreamGC(g, histogram_threshold=64, exact_select=True)
    try:
        k = h.color_core(96)
        assert k == o.color_core(96) > 0
        assert np.array_equal(h.states(), o.states())
        rep = h.publish()
        ref = o.publish_repair()
        assert rep["proper"] == 1 == ref["proper"]
        assert rep["tier1_iterations"] == ref["tier1_iterations"]
        assert np.array_equal(h.states(), o.states())
        v = h.validate()
        assert v["violations"] == 0 and v["uncolored_with_edges"] == 0
        assert h.color_core(96) == 0  # nothing left uncolored
    finally:
        h.close()
        o.close()


@pytest.mark.parametrize("name, ablation", [("overflow512", "no_overflow"), ("rmat11", "force_bitmap"),
                                            ("rmat11", "live_deg"), ("rmat11_thr16_a2", "live_deg")])
def test_ablation_builds_match_oracle(name, ablation):
    """The reference's abl-* builds as handle options: deterministic epochs and
    phase-end repairs bit-exact with the oracle under the same ablation."""
    c = MG.build_case(name)
    g = O.Oracle(c["rp"], c["col"], c["deg"], hist_threshold=c["thr"], slack_pct=c["slack"], ablations=(ablation,))
    h = S.StreamGC(S.Graph(c["rp"], c["col"], c["deg"]), epoch_size=c["E"], histogram_threshold=c["thr"],
                   slack_pct=c["slack"], max_batch=c["batch"], ablations=(ablation,))
    try:
        for ups in (c["init"], c["bench"]):
            since = 0
            for s in range(0, len(ups), c["batch"]):
                part = ups[s:s + c["batch"]]
                h.apply(part, S.MODE_DETERMINISTIC)
                g.apply(part)
                since += len(part)
                if since >= c["E"]:
                    h.epoch()
                    g.epoch()
                    since = 0
            rep = h.repair()
            it, last, fixed = g.phase_end()
            assert (rep["tier1_iterations"], rep["tier1_last_count"], rep["tier2_fixed"]) == (it, last, fixed)
            for k, a, b in (("states", h.states(), g.states()), ("bitmaps", h.bitmaps(), g.bitmaps()),
                            ("col", h.col(), g.col()), ("hist", h.hist(), g.hist())):
                assert np.array_equal(a, b), f"{name} {ablation} {k}"
            assert h.stats()["overflow_pending"] == g.overflow_count()
    finally:
        h.close()
        g.close()
