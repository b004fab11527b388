"""Host side of the product library (no GPU needed): the library loads, exports
every entry point the public headers declare, and its graph / stream helpers
match the oracle (and, through it, the reference) byte for byte."""
import os
import re

import numpy as np
import pytest

import streamgc_b200 as S
from oracle import oracle as O
from tests.golden import make_golden as MG

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols(path):
    txt = open(path).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(sgc_[a-z0-9_]+)\s*\(", txt)) - {"sgc_default_config", "sgc_pack_state",
                                                                     "sgc_unpack_color", "sgc_unpack_version",
                                                                     "sgc_compute_priority"})


def test_library_exports_every_declared_symbol():
    L = S.lib()
    heads = [os.path.join(ROOT, "include", "streamgc_b200.h"),
             os.path.join(ROOT, "include", "streamgc_batch.h"),
             os.path.join(ROOT, "include", "streamgc_server.h"),
             os.path.join(ROOT, "streamgc_b200", "csrc", "sgc_host.h")]
    for h in heads:
        for name in header_symbols(h):
            assert hasattr(L, name), f"{name} declared in {os.path.basename(h)} but not exported"
            assert name in S.SIGNATURES, f"{name} has no Python binding"


def test_dropin_archive_exports_reference_kernel_symbols():
    import subprocess
    a = os.path.join(ROOT, "streamgc_b200", "lib", "libsgc_dropin.a")
    out = subprocess.run(["nm", "-C", a], capture_output=True, text=True, check=True).stdout
    for sig in ["local_update_kernel(EdgeUpdate*, unsigned int, GPUPartition*, unsigned int)",
                "epoch_snapshot_kernel(GPUPartition*, unsigned int)", "compact_csr_kernel(GPUPartition*)",
                "drain_overflow_local_kernel(GPUPartition*, unsigned int, unsigned int*)",
                "drain_overflow_ghost_kernel(GPUPartition*, unsigned int, unsigned int*)",
                "rebuild_bitmaps_kernel(GPUPartition*)",
                "conflict_repair_kernel(GPUPartition*, unsigned int, unsigned int*)"]:
        assert re.search(r" T " + re.escape(sig), out), sig


def test_version_string():
    assert "sm_100a" in S.version()


@pytest.mark.parametrize("name", ["delaunay2k", "rmat11", "overflow512"])
def test_streams_match_oracle(name):
    c = MG.build_case(name)
    g = S.Graph(c["rp"], c["col"], c["deg"])
    assert np.array_equal(g.init_stream(), O.updates_from(O.init_stream(c["rp"], c["col"], c["deg"])))
    size, pct = MG.CASES[name][1], MG.CASES[name][2]
    pairs, types = O.bench_stream(c["rp"], c["col"], size, pct, 42)
    assert np.array_equal(g.churn_stream(size, pct, 42), O.updates_from(pairs, types))


@pytest.mark.parametrize("pct", [10, 90])
def test_stream_with_unsorted_rows_matches_oracle(pct):
    """Rows given in descending order take the generator's full live-set path;
    the stream is the same as the oracle's."""
    c = MG.build_case("rmat11")
    rp, col = c["rp"], c["col"].copy()
    for u in range(len(rp) - 1):
        col[rp[u]:rp[u + 1]] = col[rp[u]:rp[u + 1]][::-1]
    g = S.Graph(rp, col, c["deg"])
    pairs, types = O.bench_stream(rp, col, 6000, pct, 7)
    assert np.array_equal(g.churn_stream(6000, pct, 7), O.updates_from(pairs, types))


def test_loader_matches_oracle(tmp_path):
    rp, col, deg = MG.graph_rmat(9, 8, 1)
    g = S.Graph(rp, col, deg)
    p = str(tmp_path / "r.mtx")
    g.write_mtx(p)
    a = S.Graph.load_mtx(p)
    b = O.load_mtx(p)
    assert np.array_equal(a.row_ptr, b[0]) and np.array_equal(a.col_idx, b[1]) and np.array_equal(a.degree, b[2])
    assert np.array_equal(a.row_ptr, rp) and np.array_equal(a.col_idx, col)


def test_loader_rejects_bad_ids(tmp_path):
    p = tmp_path / "bad.mtx"
    p.write_text("%%MatrixMarket matrix coordinate pattern symmetric\n3 3 2\n1 2\n0 3\n")
    with pytest.raises(S.StreamGCError):
        S.Graph.load_mtx(str(p))


def test_static_greedy_matches_oracle():
    rp, col, deg = MG.graph_rmat(10, 12, 2)
    assert S.Graph(rp, col, deg).static_greedy() == O.static_greedy(rp, col)


def test_kcore_stream_properties():
    g = S.Graph.rmat(11, 16, seed=4)
    ups, k, csize = g.kcore_stream(3000, 90.0, 42)
    core = g.core_numbers()
    inside = core >= k
    assert csize == int(inside.sum()) and 2 <= csize < g.n
    assert np.all(inside[ups["u"]]) and np.all(inside[ups["v"]])
    assert np.all(ups["u"] < ups["v"])
    # two inserts per delete; inserts are non-adjacent at the time, deletes are live
    assert (ups["type"] == 1).sum() == 3000 // 3
    live = set()
    for u in range(g.n):
        for j in range(int(g.row_ptr[u]), int(g.row_ptr[u + 1])):
            v = int(g.col_idx[j])
            if u < v and inside[u] and inside[v]:
                live.add((u, v))
    for u, v, t in zip(ups["u"].tolist(), ups["v"].tolist(), ups["type"].tolist()):
        if t == 0:
            assert (u, v) not in live
            live.add((u, v))
        else:
            assert (u, v) in live
            live.remove((u, v))
    again, _, _ = g.kcore_stream(3000, 90.0, 42)
    assert np.array_equal(ups, again)


def test_core_numbers_small():
    # triangle plus a pendant: cores 2,2,2,1
    g = S.Graph.from_edges(4, np.array([[0, 1], [1, 2], [0, 2], [2, 3]]))
    assert g.core_numbers().tolist() == [2, 2, 2, 1]


def test_generators_deterministic():
    a = S.Graph.rmat(10, 8, seed=9)
    b = S.Graph.rmat(10, 8, seed=9)
    assert np.array_equal(a.col_idx, b.col_idx)
    c = S.Graph.chung_lu(5000, 2.1, 17.0, 1000.0, seed=3)
    d = S.Graph.chung_lu(5000, 2.1, 17.0, 1000.0, seed=3)
    assert np.array_equal(c.col_idx, d.col_idx)
    assert 8 < c.nnz / c.n < 40
    for g in (a, c):
        rows = np.repeat(np.arange(g.n), np.diff(g.row_ptr).astype(np.int64))
        assert np.all(g.col_idx != rows)  # no self loops


def test_write_coloring_format(tmp_path):
    colors = np.array([1, 2, 0, 7], dtype=np.uint16)
    p = str(tmp_path / "x.coloring")
    S.write_coloring(p, colors)
    assert open(p, "rb").read() == colors.astype("<u2").tobytes()
    assert open(p + ".txt").read() == "# vertices: 4\n# colors: 7\n# algorithm: streamgc\n0 1\n1 2\n2 0\n3 7\n"


def test_symmetrize_restores_mirrors():
    """sgc_csr_symmetrize: rows that lost one direction of some edges (and hold
    a self loop and an out-of-range id) become the symmetric closure."""
    g = S.Graph.delaunay(500, seed=9)
    rp, col = g.row_ptr.astype(np.uint64), g.col_idx.copy()
    rng = np.random.default_rng(2)
    keep = rng.random(len(col)) > 0.2  # drop 20% of the directed entries
    rows = [col[rp[u]:rp[u + 1]][keep[rp[u]:rp[u + 1]]].tolist() for u in range(g.n)]
    rows[0] = rows[0] + [0, 10 ** 6]
    lrp = np.zeros(g.n + 1, dtype=np.uint64)
    lrp[1:] = np.cumsum([len(r) for r in rows])
    lcol = np.array([v for r in rows for v in r], dtype=np.uint32)
    h = S.Graph.symmetrized(lrp, lcol)
    want = set()
    for u, r in enumerate(rows):
        for v in r:
            if v != u and v < g.n:
                want.add((min(u, v), max(u, v)))
    got = {(u, int(v)) for u in range(h.n) for v in h.col_idx[h.row_ptr[u]:h.row_ptr[u + 1]] if u < v}
    assert got == want
    for u in range(h.n):
        row = h.col_idx[h.row_ptr[u]:h.row_ptr[u + 1]].astype(np.int64)
        assert np.all(np.diff(row) > 0)
        assert h.degree[u] == len(row)
