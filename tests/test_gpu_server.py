"""The served form (include/streamgc_server.h) on the GPU.

  - continuous batching keeps tenants apart: with stream-order groups each
    tenant's published colors are the same served alone and in the mix (same
    submissions, same steps) -- bit-exact;
  - admission follows the HBM budget: a tenant that does not fit waits and
    becomes resident once a group's tenants are removed;
  - requests become visible with the publish that includes them; latencies
    are recorded; queries answer while steps run on another thread."""
import threading

import numpy as np
import pytest

import streamgc_b200 as S
from tests.golden import make_golden as MG

pytestmark = pytest.mark.gpu

NAMES = ["delaunay2k", "rmat11", "overflow512"]
EPOCH = 1024


def _graph(c):
    return S.Graph(c["rp"], c["col"], c["deg"])


def _requests(c, steps, seed):
    """Per step, a few update requests of random sizes cut from the churn stream."""
    rng = np.random.default_rng(seed)
    ups, pos, out = c["bench"], 0, []
    for _ in range(steps):
        reqs = []
        for _ in range(int(rng.integers(1, 4))):
            m = int(rng.integers(1, 700))
            reqs.append(ups[pos:pos + m])
            pos += m
        out.append(reqs)
    return out


def test_served_alone_equals_mixed():
    cases = [MG.build_case(n) for n in NAMES]
    STEPS = 12
    plans = [_requests(c, STEPS, 100 + i) for i, c in enumerate(cases)]
    mixed = S.Server(stream_order=True)
    alone = [S.Server(stream_order=True) for _ in cases]
    try:
        tm = [mixed.add_tenant(_graph(c), epoch_size=EPOCH, histogram_threshold=c["thr"]) for c in cases]
        ta = [alone[i].add_tenant(_graph(c), epoch_size=EPOCH, histogram_threshold=c["thr"])
              for i, c in enumerate(cases)]
        for s in range(STEPS):
            for i in range(len(cases)):
                for r in plans[i][s]:
                    mixed.submit(tm[i], r)
                    alone[i].submit(ta[i], r)
            assert mixed.step()["proper"] == 1
            for i in range(len(cases)):
                assert alone[i].step()["proper"] == 1
                assert np.array_equal(mixed.snapshot(tm[i]), alone[i].snapshot(ta[i])), (NAMES[i], s)
        st = mixed.stats()
        assert st["tenants_resident"] == len(cases) and st["groups"] == 1
    finally:
        mixed.close()
        for a in alone:
            a.close()


def test_admission_waits_for_budget_and_frees_on_removal():
    c = MG.build_case("rmat11")
    g = _graph(c)
    fp = S.Server.footprint(g.n, g.nnz)
    staging = (1 << 16) * 64  # per-group staging the server reserves for max_tick_updates = 2^16
    budget = 2 * fp + staging + fp // 2  # two tenants fit, a third does not
    srv = S.Server(hbm_budget_bytes=budget, max_tick_updates=1 << 16)
    try:
        t = [srv.add_tenant(g, epoch_size=EPOCH) for _ in range(3)]
        assert all(srv.state(x) == S.TENANT_QUEUED for x in t)
        assert srv.step()["admitted"] == 2
        assert [srv.state(x) for x in t] == [S.TENANT_RESIDENT, S.TENANT_RESIDENT, S.TENANT_QUEUED]
        rid = srv.submit(t[2], c["bench"][:100])  # held while queued
        assert not srv.visible(rid)
        assert not srv.query(t[2], np.arange(10, dtype=np.uint32)).any()
        srv.remove_tenant(t[0])
        assert srv.step()["admitted"] == 0  # the group still holds tenant 1
        srv.remove_tenant(t[1])
        r = srv.step()  # frees the group, then admits tenant 2
        assert r["admitted"] == 1 and srv.state(t[2]) == S.TENANT_RESIDENT
        assert srv.visible(rid)  # admission publishes the tenant with its held updates
        snap = srv.snapshot(t[2])
        assert (snap[np.diff(c["rp"]) > 0] > 0).mean() > 0.99  # colored from scratch at admission
        st = srv.stats()
        assert st["tenants_resident"] == 1 and st["tenants_queued"] == 0 and st["resident_bytes"] <= budget
        assert st["groups"] == 1
    finally:
        srv.close()


def test_requests_become_visible_with_their_publish():
    c = MG.build_case("delaunay2k")
    srv = S.Server()
    try:
        t = srv.add_tenant(_graph(c), epoch_size=EPOCH)
        srv.step()  # admission: base graph colored and published
        ups = c["bench"]
        r1 = srv.submit(t, ups[:600])
        srv.step()
        assert not srv.visible(r1)  # 600 < epoch
        r2 = srv.submit(t, ups[600:1100])
        srv.step()
        assert srv.visible(r1) and srv.visible(r2)
        v = np.arange(0, len(c["deg"]), 3, dtype=np.uint32)
        assert np.array_equal(srv.query(t, v), srv.snapshot(t)[v])
        st = srv.stats()
        assert st["requests_visible"] == 2 and st["visible_p99_ms"] >= st["visible_p50_ms"] > 0
        assert st["queries"] == 1 and st["query_p50_ms"] > 0
    finally:
        srv.close()


def test_staleness_deadline_closes_epochs():
    c = MG.build_case("delaunay2k")
    srv = S.Server(max_staleness_us=1)
    try:
        t = srv.add_tenant(_graph(c), epoch_size=1 << 20)  # the count alone would never close it
        srv.step()
        rid = srv.submit(t, c["bench"][:50])
        srv.step()
        srv.step()
        assert srv.visible(rid)
    finally:
        srv.close()


def test_queries_and_submits_while_steps_run():
    """A stepping thread and a client thread: the client's queries answer from
    published snapshots during steps, and all its requests become visible."""
    c = MG.build_case("rmat11")
    srv = S.Server(max_staleness_us=200)
    t = srv.add_tenant(_graph(c), epoch_size=EPOCH)
    srv.step()
    stop = threading.Event()
    errors = []

    def stepper():
        try:
            while not stop.is_set():
                assert srv.step()["proper"] == 1
        except Exception as e:  # surfaced below
            errors.append(e)

    th = threading.Thread(target=stepper)
    th.start()
    try:
        ups = c["bench"]
        rids = []
        rng = np.random.default_rng(5)
        for i in range(40):
            rids.append(srv.submit(t, ups[i * 200:(i + 1) * 200]))
            q = srv.query(t, rng.integers(0, len(c["deg"]), 4).astype(np.uint32))
            assert q.shape == (4,)
        for _ in range(2000):
            if all(srv.visible(r) for r in rids):
                break
            threading.Event().wait(0.005)
    finally:
        stop.set()
        th.join()
    assert not errors, errors
    assert all(srv.visible(r) for r in rids)
    assert srv.stats()["queries"] == 40
    srv.close()
