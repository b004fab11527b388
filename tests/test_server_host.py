"""Host-side rules of the served form that need no GPU: the footprint the
admission control charges, and the queue before the first step."""
import pytest

import streamgc_b200 as S
from tests.golden import make_golden as MG


def test_footprint_counts_slack_slots_and_vertex_state():
    # rows get max(d + 3d, 8) slots of 4 bytes under alpha = 4
    assert S.Server.footprint(1000, 0) >= 1000 * 8 * 4
    a = S.Server.footprint(1 << 20, 10 << 20)
    b = S.Server.footprint(1 << 20, 20 << 20)
    assert b - a >= 4 * (40 << 20)  # 10M more entries -> 40M more slots of 4 bytes
    assert S.Server.footprint(1 << 20, 10 << 20, slack_pct=100) < a


def test_tenants_queue_until_a_step_and_can_leave():
    c = MG.build_case("delaunay2k")
    g = S.Graph(c["rp"], c["col"], c["deg"])
    srv = S.Server(hbm_budget_bytes=1 << 30, max_tick_updates=1 << 12)
    try:
        t0 = srv.add_tenant(g, epoch_size=1024)
        t1 = srv.add_tenant(g, epoch_size=1024)
        assert srv.state(t0) == srv.state(t1) == S.TENANT_QUEUED
        rid = srv.submit(t1, c["bench"][:10])
        assert rid > 0 and not srv.visible(rid)
        with pytest.raises(S.StreamGCError, match="max_tick_updates"):
            srv.submit(t1, c["bench"][:5000])
        srv.remove_tenant(t0)
        assert srv.state(t0) == S.TENANT_REMOVED
        with pytest.raises(S.StreamGCError, match="removed"):
            srv.submit(t0, c["bench"][:10])
        st = srv.stats()
        assert st["tenants_queued"] == 1 and st["tenants_resident"] == 0 and st["update_requests"] == 1
    finally:
        srv.close()


def test_queries_before_admission_answer_zero_and_are_counted():
    """A tenant that is not resident yet answers 0 for every vertex; each query
    is counted and timed (p50/p99 over the most recent queries)."""
    c = MG.build_case("delaunay2k")
    g = S.Graph(c["rp"], c["col"], c["deg"])
    srv = S.Server(hbm_budget_bytes=1 << 30, max_tick_updates=1 << 12)
    try:
        t = srv.add_tenant(g, epoch_size=1024)
        for k in range(25):
            out = srv.query(t, [0, 1, 2, k])
            assert out.tolist() == [0, 0, 0, 0]
        st = srv.stats()
        assert st["queries"] == 25 and st["query_vertices"] == 100
        assert 0.0 <= st["query_p50_ms"] <= st["query_p99_ms"]
        assert st["requests_visible"] == 0 and st["tenants_regrown"] == 0
    finally:
        srv.close()


def test_requests_of_a_removed_tenant_are_never_visible():
    c = MG.build_case("delaunay2k")
    g = S.Graph(c["rp"], c["col"], c["deg"])
    srv = S.Server(hbm_budget_bytes=1 << 30, max_tick_updates=1 << 12)
    try:
        t = srv.add_tenant(g, epoch_size=1024)
        ids = [srv.submit(t, c["bench"][k:k + 4]) for k in range(0, 40, 4)]
        assert ids == sorted(ids) and len(set(ids)) == len(ids)
        srv.remove_tenant(t)
        assert not any(srv.visible(i) for i in ids)
        assert not srv.visible(0) and not srv.visible(ids[-1] + 1)
    finally:
        srv.close()


def test_removed_tenant_requests_leave_the_state_window():
    """Requests of a removed tenant are resolved as dropped on every removal
    path, so the window of request states moves past them; the count of
    dropped requests is kept."""
    c = MG.build_case("delaunay2k")
    g = S.Graph(c["rp"], c["col"], c["deg"])
    srv = S.Server(hbm_budget_bytes=1 << 30, max_tick_updates=1 << 12)
    try:
        t0 = srv.add_tenant(g, epoch_size=1024)
        t1 = srv.add_tenant(g, epoch_size=1024)
        a = [srv.submit(t0, c["bench"][k:k + 4]) for k in range(0, 40, 4)]
        b = [srv.submit(t1, c["bench"][k:k + 4]) for k in range(0, 40, 4)]
        assert srv.stats()["requests_tracked"] == 20
        srv.remove_tenant(t1)  # its requests sit behind t0's unresolved ones
        st = srv.stats()
        assert st["requests_tracked"] == 20 and st["requests_dropped"] == 10
        srv.remove_tenant(t0)
        st = srv.stats()
        assert st["requests_tracked"] == 0 and st["requests_dropped"] == 20
        assert not any(srv.visible(i) for i in a + b)
    finally:
        srv.close()
