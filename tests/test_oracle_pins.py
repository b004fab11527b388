"""Pins the oracle to the reference itself.

* Against the reference's own host code (stream_gen.cpp, graph_loader.cpp),
  compiled from its sources into oracle/_ref/libref_host.so when the reference
  tree was present at build time: loader, init stream and churn stream must be
  byte-identical.
* Against tests/golden/ref_epochs.json: SHA-256 of every state array at every
  epoch boundary of the reference's own kernels run as one warp in stream
  order (tests/golden/make_golden.py). The oracle must reproduce all of them.
"""
import json
import os

import numpy as np
import pytest

from oracle import oracle as O
from tests import _util
from tests.golden import make_golden as MG

HAVE_REF = O.ref_host_available()


def _write_mtx(path, rp, col, weights=False):
    n = len(rp) - 1
    with open(path, "w") as f:
        f.write("%%MatrixMarket matrix coordinate %s symmetric\n%% test\n" % ("real" if weights else "pattern"))
        lines = [(u + 1, int(col[j]) + 1) for u in range(n) for j in range(int(rp[u]), int(rp[u + 1]))
                 if col[j] < u]
        f.write(f"{n} {n} {len(lines) + 2}\n")
        for a, b in lines:
            f.write(f"{a} {b} 1.5\n" if weights else f"{a} {b}\n")
        f.write("3 3\n" if not weights else "3 3 2.0\n")   # self loop: dropped
        f.write(f"{lines[0][0]} {lines[0][1]}\n" if not weights else f"{lines[0][0]} {lines[0][1]} 1.0\n")  # duplicate


@pytest.mark.skipif(not HAVE_REF, reason="reference host library not built (no reference tree here)")
@pytest.mark.parametrize("weights", [False, True])
def test_loader_matches_reference(tmp_path, weights):
    rp, col, deg = MG.graph_delaunay(700, 11)
    path = str(tmp_path / "g.mtx")
    _write_mtx(path, rp, col, weights)
    a = O.load_mtx(path)
    b = O.ref_load_mtx(path)
    for x, y in zip(a, b):
        assert np.array_equal(x.astype(np.uint64), y.astype(np.uint64))


@pytest.mark.skipif(not HAVE_REF, reason="reference host library not built (no reference tree here)")
@pytest.mark.parametrize("name", ["delaunay2k", "rmat11", "overflow512"])
def test_streams_match_reference(name):
    c = MG.build_case(name)
    rp32 = c["rp"].astype(np.uint32)
    ri = O.ref_init_stream(rp32, c["col"], c["deg"])
    assert np.array_equal(O.init_stream(c["rp"], c["col"], c["deg"]), ri)
    size, pct = MG.CASES[name][1], MG.CASES[name][2]
    for seed in (42, 7):
        p1, t1 = O.bench_stream(c["rp"], c["col"], size, pct, seed)
        p2, t2 = O.ref_bench_stream(rp32, c["col"], c["deg"], size, pct, seed)
        assert np.array_equal(p1, p2) and np.array_equal(t1, t2)


GOLDEN = MG.GOLDEN_JSON


@pytest.mark.skipif(not os.path.exists(GOLDEN), reason="golden epoch fixtures not generated yet")
@pytest.mark.parametrize("name", list(MG.CASES))
def test_oracle_matches_reference_epochs(name):
    gold = json.load(open(GOLDEN))[name]
    c = MG.build_case(name)
    assert _util.sha(np.frombuffer(MG.case_bytes(c), dtype=np.uint8)) == gold["input_sha256"], "case input drifted"
    seen = 0
    for tag, arrays in _util.oracle_epochs(c):
        g = gold["epochs"][tag]
        for k in _util.ARRAY_NAMES:
            assert _util.sha(arrays[k]) == g[k], f"{name} {tag} {k}"
        seen += 1
    assert seen == len(gold["epochs"])


@pytest.mark.skipif(not os.path.exists(MG.GOLDEN_SCALE_JSON), reason="full-size epoch fixtures not generated yet")
@pytest.mark.parametrize("name", list(MG.SCALE_CASES))
def test_oracle_matches_reference_epochs_full_size(name):
    """The plain small workload at full size (Delaunay 2^17, 1 M churn, 43
    epoch boundaries): the oracle equals the reference's kernels at every one."""
    gold = json.load(open(MG.GOLDEN_SCALE_JSON))[name]
    c = MG.build_case(name)
    assert _util.sha(np.frombuffer(MG.case_bytes(c), dtype=np.uint8)) == gold["input_sha256"], "case input drifted"
    seen = 0
    for tag, arrays in _util.oracle_epochs(c):
        g = gold["epochs"][tag]
        for k in _util.ARRAY_NAMES:
            assert _util.sha(arrays[k]) == g[k], f"{name} {tag} {k}"
        seen += 1
    assert seen == len(gold["epochs"]) == 43
