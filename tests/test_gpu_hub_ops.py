"""Row-scale operations of concurrent batches (HubOp): on a row longer than
8,192 live entries, a color reduction whose first 512 entries show no holder
of the freed color, and the recolor of a conflict loser, are finished by the
block-wide pass after the batch. Checked on two cliques of hubs with
thousands of leaves each: the single-update cases land exactly where the rule
says, and mixed batches publish proper snapshots with the expected rows and
clean layouts."""
import numpy as np
import pytest

import streamgc_b200 as S
from oracle import oracle as O

pytestmark = pytest.mark.gpu

ADD, DEL = 0, 1  # EdgeUpdate types

HUBS = 20          # hubs per clique
LEAVES0 = 8300     # leaves of the first hub of a clique (every hub row is longer than 8,192 entries)


def _graph():
    pairs = []
    n = 0
    groups = []
    for _ in range(2):
        hubs = list(range(n, n + HUBS))
        n += HUBS
        groups.append(hubs)
        for i in hubs:
            for j in hubs:
                if i < j:
                    pairs.append((i, j))
    for gi, hubs in enumerate(groups):
        for k, hb in enumerate(hubs):
            for _ in range(LEAVES0 + 20 * k + gi):  # distinct degrees: distinct priorities
                pairs.append((hb, n))
                n += 1
    return n, np.array(pairs, dtype=np.uint32), groups


def _ups(rows):
    return S.updates_from([(u, v) for u, v, _ in rows], [t for _, _, t in rows])


def _handle():
    n, pairs, groups = _graph()
    g = S.Graph.from_edges(n, pairs)
    h = S.StreamGC(g, epoch_size=4096, histogram_threshold=64, max_batch=4096, exact_select=True)
    rep = h.repair()
    assert rep["proper"] == 1
    return g, h, groups


def _check_clean(h):
    st = h.stats()
    assert st["device_error"] == 0
    assert h.check_state()["bad_rows"] == 0


def test_reduction_left_to_the_pass_lands_on_the_freed_color():
    g, h, groups = _handle()
    try:
        col = h.colors().astype(np.int64)
        hubs = groups[0]
        a = max(hubs, key=lambda x: col[x])
        # a clique neighbor whose color no other neighbor of a holds (leaves take 1 or 2)
        b = next(x for x in hubs if x != a and 3 <= col[x] < col[a])
        before = h.stats()["hub_deferred"]
        h.apply(_ups([(a, b, DEL)]), S.MODE_CONCURRENT)
        h.synchronize()
        assert h.stats()["hub_deferred"] == before + 1
        after = h.colors()
        assert after[a] == col[b]  # moved down to the freed color
        assert after[b] == col[b]
        rep = h.publish()
        assert rep["proper"] == 1
        _check_clean(h)
    finally:
        h.close()


def test_conflict_loser_with_a_long_row_recolors_in_the_pass():
    g, h, groups = _handle()
    try:
        col = h.colors().astype(np.int64)
        by_color = {}
        for x in groups[1]:
            by_color.setdefault(int(col[x]), x)
        pair = next((x, by_color[int(col[x])]) for x in groups[0] if int(col[x]) in by_color)
        u, v = pair
        deg = g.degree
        loser = u if (deg[u], u) < (deg[v], v) else v
        before = h.stats()["hub_deferred"]
        h.apply(_ups([(u, v, ADD)]), S.MODE_CONCURRENT)
        h.synchronize()
        assert h.stats()["hub_deferred"] == before + 1
        after = h.colors()
        assert after[loser] != col[loser]  # left the shared color
        assert after[u] != after[v]
        rep = h.publish()
        assert rep["proper"] == 1
        _check_clean(h)
    finally:
        h.close()


def test_mixed_batches_publish_proper_snapshots_with_the_expected_rows():
    g, h, groups = _handle()
    rng = np.random.default_rng(7)
    try:
        rp, cl = g.row_ptr, g.col_idx
        present = set()
        for x in range(len(rp) - 1):
            for y in cl[rp[x]:rp[x + 1]].tolist():
                if x < y:
                    present.add((x, int(y)))
        hub_pairs = [(i, j) for hubs in groups for i in hubs for j in hubs if i < j]
        cross = [(i, j) for i in groups[0] for j in groups[1]]
        for _ in range(6):
            batch = []
            for _ in range(64):  # delete clique edges, add cross edges, and re-add deleted ones
                r = rng.random()
                if r < 0.45:
                    e = hub_pairs[rng.integers(len(hub_pairs))]
                    batch.append((e[0], e[1], DEL if e in present else ADD))
                    present.symmetric_difference_update({e})
                else:
                    e = cross[rng.integers(len(cross))]
                    batch.append((e[0], e[1], DEL if e in present else ADD))
                    present.symmetric_difference_update({e})
            h.apply(_ups(batch), S.MODE_CONCURRENT)
            rep = h.publish()
            assert rep["proper"] == 1
            snap = h.snapshot()
            v = O.validate_colors(h.row_ptr(), h.col(), snap)
            assert v["violations"] == 0 and v["uncolored_with_edges"] == 0
            _check_clean(h)
        assert h.stats()["hub_deferred"] > 0
        h.drain_and_compact()
        gr, gc = h.row_ptr(), h.col()
        want = {}
        for (x, y) in present:
            want.setdefault(x, []).append(y)
            want.setdefault(y, []).append(x)
        for x in (x for hubs in groups for x in hubs):  # the only rows the updates touch
            got = sorted(int(y) for y in gc[gr[x]:gr[x + 1]] if y < len(gr) - 1)
            assert got == sorted(want.get(x, [])), f"row {x}"
    finally:
        h.close()
