"""Known-answer tests the reference's unit tests pin, run against the oracle.

  color selection  algorithms/streamgc/test/unit/test_color_select.cu:62-276
  loser rule       algorithms/streamgc/test/unit/test_local_update.cu:162-269
  priority         algorithms/streamgc/test/unit/test_priority.cu:13-73
  pack / unpack    algorithms/streamgc/test/unit/test_vertex_state.cu:60-202
"""
import numpy as np
import pytest

from oracle import oracle as O


def one_vertex(deg=0, hd=False):
    """A vertex with no neighbors; degree above the threshold puts it in histogram mode."""
    rp = np.array([0, 0, 0], dtype=np.uint64)
    col = np.zeros(0, dtype=np.uint32)
    degree = np.array([65 if hd else deg, 0], dtype=np.uint32)
    return O.Oracle(rp, col, degree, hist_threshold=64)


@pytest.mark.parametrize("bitmap,expect", [(0, 1), (0x1, 2), (0b10111, 4), (0b11, 3)])
def test_bitmap_kats(bitmap, expect):
    g = one_vertex()
    g.set_bitmap(0, bitmap)
    assert g.fac(0) == expect


def test_bitmap_all_64_taken_falls_back_to_neighbor_scan():
    # The reference test asserts 65 here (test_color_select.cu:137-160), but the
    # reference code it exercises (color_select.cuh:20-52) falls back to scanning
    # neighbor colors when all 64 bits are set; an isolated vertex gets color 1.
    # Parity follows the code.
    g = one_vertex()
    g.set_bitmap(0, (1 << 64) - 1)
    assert g.fac(0) == 1


@pytest.mark.parametrize("counts,expect", [([], 1), ([3, 2, 1, 5, 4], 6), ([2, 1, 0, 3], 3)])
def test_histogram_kats(counts, expect):
    g = one_vertex(hd=True)
    g.set_hist_row(0, counts)
    assert g.fac(0) == expect


def test_histogram_full_returns_first_minimum():
    g = one_vertex(hd=True)
    h = np.full(1024, 7, dtype=np.uint32)
    h[10] = 3
    h[500] = 3
    g.set_hist_row(0, h)
    assert g.fac(0) == 11


def test_histogram_wrapped_counter_is_large():
    # uint32 counters can wrap below zero (color_select.cuh:151); a wrapped bin is
    # the largest value, never a minimum.
    g = one_vertex(hd=True)
    h = np.full(1024, 2, dtype=np.uint32)
    h[0] = 0xFFFFFFFF
    g.set_hist_row(0, h)
    assert g.fac(0) == 2


def two_vertices(cu, cv, du, dv):
    rp = np.array([0, 0, 0], dtype=np.uint64)
    g = O.Oracle(rp, np.zeros(0, dtype=np.uint32), np.array([du, dv], dtype=np.uint32))
    g.set_states(np.array([cu, cv], dtype=np.uint32))
    return g


def test_loser_rule_no_conflict():
    g = two_vertices(1, 2, 10, 5)
    g.apply(O.updates_from([[0, 1]]))
    s = g.states()
    assert (s & 0xFFFF).tolist() == [1, 2] and (s >> 16).tolist() == [0, 0]


def test_loser_rule_lower_degree_recolors():
    g = two_vertices(3, 3, 10, 5)
    g.apply(O.updates_from([[0, 1]]))
    s = g.states()
    assert s[0] & 0xFFFF == 3 and s[0] >> 16 == 0
    assert s[1] & 0xFFFF not in (0, 3) and s[1] >> 16 == 1


def test_loser_rule_equal_degree_higher_id_keeps():
    g = two_vertices(5, 5, 10, 10)
    g.apply(O.updates_from([[0, 1]]))
    s = g.states()
    assert s[1] & 0xFFFF == 5 and s[1] >> 16 == 0
    assert s[0] & 0xFFFF not in (0, 5) and s[0] >> 16 == 1


def test_uncolored_endpoints_get_distinct_colors_version_one():
    g = two_vertices(0, 0, 10, 5)
    g.apply(O.updates_from([[0, 1]]))
    s = g.states()
    assert (s & 0xFFFF).tolist() == [1, 2] and (s >> 16).tolist() == [1, 1]


def prio(deg, vid):
    return (deg << 32) | vid


def test_priority_order():
    assert prio(100, 1) > prio(50, 999)
    assert prio(100, 500) > prio(100, 200)
    assert prio(10, 1) != prio(10, 2) and prio(10, 1) != prio(11, 1)
    assert prio(1, 0) > prio(0, 42)
    p = prio(0xFFFFFFFF, 0xFFFFFFFF)
    assert p >> 32 == 0xFFFFFFFF and p & 0xFFFFFFFF == 0xFFFFFFFF


@pytest.mark.parametrize("c,v", [(42, 7), (0, 0), (0xFFFF, 0xFFFF), (0xFFFE, 100), (0xFFFF, 200)])
def test_pack_unpack(c, v):
    w = (v << 16) | c
    assert w & 0xFFFF == c and w >> 16 == v


def test_version_wraps_at_16_bits():
    # recolor writes version + 1 in a 16-bit field (recolor.cu:245-249)
    rp = np.array([0, 1, 2], dtype=np.uint64)
    g = O.Oracle(rp, np.array([1, 0], dtype=np.uint32), np.array([1, 2], dtype=np.uint32))
    g.set_states(np.array([(0xFFFF << 16) | 4, 4], dtype=np.uint32))
    g.apply(O.updates_from([[0, 1]]))  # equal colors, vertex 0 (degree 1) loses
    s = g.states()
    assert s[0] >> 16 == 0 and s[0] & 0xFFFF != 4
