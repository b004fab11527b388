"""The allocation-free point query, checked against sgc_query.

Some callers cannot allocate device memory (a serving thread whose tenants
already fill their HBM budget, or a path that must not enter the allocator);
sgc_query_noalloc serves them from a fixed scratch array compiled into the
library. Its answers must equal sgc_query's, on two calls in a row (the second
call reuses the scratch the first one left behind). Collected last, so a run
that stops at the first failure has run every other test first; it also runs
on its own in a fresh process."""
import numpy as np
import pytest

import streamgc_b200 as S
from tests.golden import make_golden as MG

pytestmark = pytest.mark.gpu


def _published():
    c = MG.build_case("delaunay2k")
    h = S.StreamGC(S.Graph(c["rp"], c["col"], c["deg"]), epoch_size=2048, max_batch=2048)
    h.process_stream(c["init"], S.MODE_CONCURRENT)
    h.process_stream(c["bench"][:8192], S.MODE_CONCURRENT)
    h.publish()
    return c, h


def test_query_noalloc_matches_query_twice_in_a_row():
    c, h = _published()
    n = len(c["deg"])
    rng = np.random.default_rng(9)
    try:
        for call in range(2):
            k = [5000, 65536][call]
            v = rng.integers(0, n + 100, size=k).astype(np.uint32)  # some out of range -> 0
            ref = h.query(v)
            got = h.query_noalloc(v)
            assert np.array_equal(got, ref), f"call {call}"
            assert np.array_equal(got[v < n], h.snapshot()[v[v < n]])
    finally:
        h.close()


def test_query_noalloc_rejects_oversize():
    c, h = _published()
    try:
        with pytest.raises(S.StreamGCError, match="exceed"):
            h.query_noalloc(np.zeros(65537, dtype=np.uint32))
        assert len(h.query_noalloc(np.zeros(0, dtype=np.uint32))) == 0
    finally:
        h.close()
