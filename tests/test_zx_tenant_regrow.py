"""Served tenants whose rows fill up (options.regrow): a tenant whose inserts
no longer fit its rows loses entries at the drain, as the reference does; the
server then reads its live rows back, restores each surviving entry's mirror
and admits it again with rows sized from its current degrees. Afterwards its
rows hold every edge in both directions and its snapshot is proper."""
import time

import numpy as np
import pytest

import streamgc_b200 as S
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _mirror_complete(rp, col):
    n = len(rp) - 1
    x = np.repeat(np.arange(n, dtype=np.int64), np.diff(rp.astype(np.int64)))
    fwd = set(zip(x.tolist(), col.tolist()))
    return all((y, u) in fwd for u, y in fwd)


@pytest.mark.parametrize("regrow", [False, True])
def test_tenant_with_full_rows(regrow):
    g = S.Graph.delaunay(2000, seed=5)
    nbr0 = set(g.col_idx[g.row_ptr[0]:g.row_ptr[1]].tolist())
    star = [v for v in range(1, 2000) if v not in nbr0][:300]  # new edges at vertex 0: its row overflows
    ups = S.updates_from([[0, v] for v in star], [S.ADD] * len(star))
    with S.Server(max_tick_updates=1 << 16, slack_pct=0, regrow=regrow, max_staleness_us=1000) as srv:
        t = srv.add_tenant(g, epoch_size=64)
        assert srv.step()["admitted"] == 1
        for s0 in range(0, len(ups), 50):
            srv.submit(t, ups[s0:s0 + 50])
            for _ in range(3):
                assert srv.step()["proper"] == 1
        for _ in range(12):  # the staleness deadline publishes the last epoch's updates
            time.sleep(0.002)
            assert srv.step()["proper"] == 1
        st = srv.stats()
        assert st["requests_visible"] == st["update_requests"]
        assert st["drain_failed"] > 0 or st["tenants_regrown"] > 0
        rp, col = srv.rows(t)
        snap = srv.snapshot(t)
        v = O.validate_colors(rp, col, snap)
        assert v["violations"] == 0 and v["uncolored_with_edges"] == 0
        if regrow:
            assert st["tenants_regrown"] >= 1
            assert _mirror_complete(rp, col)
            row0 = set(col[rp[0]:rp[1]].tolist())
            assert all(v in row0 for v in star)  # every inserted edge, both directions
            q = np.array([0] + star[:10], dtype=np.uint32)
            assert np.array_equal(srv.query(t, q), snap[q])
        else:
            assert st["tenants_regrown"] == 0
