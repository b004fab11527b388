"""Golden epoch fixtures from the reference's own kernels.

Builds small deterministic cases (seeded graphs; update streams from the
oracle's restatement of the reference's stream generator, itself pinned
byte-for-byte against the reference's stream_gen.cpp), runs the reference's
kernels on them through oracle/_ref/ref_driver (one warp, stream order), and
records a SHA-256 of every state array at every epoch boundary and after each
drain_and_compact into tests/golden/ref_epochs.json.

    python tests/golden/make_golden.py --run OUT_DIR         # on a GPU box
    python tests/golden/make_golden.py --run-scale OUT_DIR   # the full-size case, on a GPU box
    python tests/golden/make_golden.py --list                # case summary

The JSONs are committed; tests rebuild the same cases and compare the oracle's
and the CUDA path's states against them. The full-size case (SCALE_CASES) is
the plain small workload at its real size: Delaunay of 131,072 points (seed
42), the reference's 50/50 churn stream of 1,000,000 updates (seed 42),
epochs of 32,768, threshold 64, alpha 4 -- 30 bench epochs and 12 init
epochs, each pinned to the reference's kernels (tests/golden/ref_epochs_c1.json).
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import struct
import subprocess
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from oracle import oracle as O  # noqa: E402

GOLDEN_JSON = os.path.join(os.path.dirname(os.path.abspath(__file__)), "ref_epochs.json")
GOLDEN_SCALE_JSON = os.path.join(os.path.dirname(os.path.abspath(__file__)), "ref_epochs_c1.json")
ARRAYS = ("states", "bitmaps", "col", "snapshot", "hist", "ovf_count")


def _csr_from_pairs(n, pairs):
    """Loader semantics: drop self loops, normalise, sort, unique, symmetric, sorted rows."""
    p = np.asarray(pairs, dtype=np.int64).reshape(-1, 2)
    p = p[p[:, 0] != p[:, 1]]
    p = np.sort(p, axis=1)
    key = np.unique(p[:, 0] * (1 << 32) + p[:, 1])
    a = (key >> 32).astype(np.int64)
    b = (key & 0xFFFFFFFF).astype(np.int64)
    src = np.concatenate([a, b])
    dst = np.concatenate([b, a])
    order = np.lexsort((dst, src))
    src, dst = src[order], dst[order]
    deg = np.bincount(src, minlength=n).astype(np.uint32)
    rp = np.zeros(n + 1, dtype=np.uint64)
    rp[1:] = np.cumsum(deg)
    return rp, dst.astype(np.uint32), deg


def graph_delaunay(n, seed):
    from scipy.spatial import Delaunay
    pts = np.random.default_rng(seed).random((n, 2))
    t = Delaunay(pts).simplices
    return _csr_from_pairs(n, np.concatenate([t[:, [0, 1]], t[:, [1, 2]], t[:, [0, 2]]]))


def graph_rmat(scale, ef, seed, a=0.57, b=0.19, c=0.19):
    rng = np.random.default_rng(seed)
    m = ef << scale
    u = np.zeros(m, dtype=np.int64)
    v = np.zeros(m, dtype=np.int64)
    for lvl in range(scale):
        r = rng.random(m)
        bit = 1 << (scale - 1 - lvl)
        v += np.where((r >= a) & (r < a + b), bit, 0) + np.where(r >= a + b + c, bit, 0)
        u += np.where(r >= a + b, bit, 0)
    return _csr_from_pairs(1 << scale, np.stack([u, v], axis=1))


def graph_sparse_ring(n, chords, seed):
    rng = np.random.default_rng(seed)
    ring = np.stack([np.arange(n), (np.arange(n) + 1) % n], axis=1)
    ch = rng.integers(0, n, size=(chords, 2))
    return _csr_from_pairs(n, np.concatenate([ring, ch]))


CASES = {
    # name: (graph builder, stream size, insert pct, hist threshold, epoch E, host batch, slack pct)
    "delaunay2k": (lambda: graph_delaunay(2048, 7), 24000, 50, 64, 2048, 2048, 300),
    "rmat11": (lambda: graph_rmat(11, 16, 3), 16000, 50, 64, 4096, 4096, 300),
    "overflow512": (lambda: graph_sparse_ring(512, 64, 5), 12000, 85, 64, 1024, 1024, 300),
    "rmat11_thr16_a2": (lambda: graph_rmat(11, 16, 3), 12000, 60, 16, 3000, 1500, 100),
}


SCALE_CASES = {
    "delaunay17_c1": (lambda: graph_delaunay(131072, 42), 1_000_000, 50, 64, 32768, 32768, 300),
}


def build_case(name):
    """Returns dict(rp, col, deg, init, bench, thr, E, batch, slack)."""
    gb, size, pct, thr, E, batch, slack = CASES[name] if name in CASES else SCALE_CASES[name]
    rp, col, deg = gb()
    init = O.updates_from(O.init_stream(rp, col, deg))
    pairs, types = O.bench_stream(rp, col, size, pct, 42)
    bench = O.updates_from(pairs, types)
    return dict(rp=rp, col=col, deg=deg, init=init, bench=bench, thr=thr, E=E, batch=batch, slack=slack)


def case_bytes(c):
    n = len(c["rp"]) - 1
    hdr = struct.pack("<IQIIIIQQ", n, len(c["col"]), c["thr"], c["E"], c["batch"], c["slack"], len(c["init"]),
                      len(c["bench"]))
    return b"".join([hdr, c["rp"].astype("<u4").tobytes(), c["col"].astype("<u4").tobytes(),
                     c["deg"].astype("<u4").tobytes(), c["init"].tobytes(), c["bench"].tobytes()])


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def parse_dump(path):
    """ref_driver output -> list of (tag, {array: bytes})."""
    out = []
    cur = None
    with open(path, "rb") as f:
        data = f.read()
    i = 0
    while i < len(data):
        tag = data[i:i + 16].split(b"\0", 1)[0].decode()
        (nb,) = struct.unpack("<Q", data[i + 16:i + 24])
        payload = data[i + 24:i + 24 + nb]
        i += 24 + nb
        if nb == 0 and tag not in ARRAYS:
            cur = (tag, {})
            out.append(cur)
        else:
            cur[1][tag] = payload
    return out


def epoch_tags(c):
    """Tags the driver emits, in order, for this case's protocol."""
    tags = []
    k = 0
    for phase, ups in (("init", c["init"]), ("bench", c["bench"])):
        since = 0
        for s in range(0, len(ups), c["batch"]):
            since += min(c["batch"], len(ups) - s)
            if since >= c["E"]:
                tags.append(f"{phase}_e{k}")
                k += 1
                since = 0
        tags.append(f"{phase}_dc")
    return tags


def run(out_dir, cases=CASES, out_name="ref_epochs.json"):
    driver = os.path.join(ROOT, "oracle", "_ref", "ref_driver")
    os.makedirs(out_dir, exist_ok=True)
    result = {}
    for name in cases:
        c = build_case(name)
        cin = os.path.join(out_dir, f"{name}.bin")
        cout = os.path.join(out_dir, f"{name}.dump")
        with open(cin, "wb") as f:
            f.write(case_bytes(c))
        subprocess.run([driver, "--in", cin, "--out", cout, "--launch", "det"], check=True)
        recs = parse_dump(cout)
        entry = {"input_sha256": hashlib.sha256(case_bytes(c)).hexdigest(), "epochs": {}}
        for tag, arrays in recs:
            if tag in ("timing", "final"):
                continue
            entry["epochs"][tag] = {k: hashlib.sha256(v).hexdigest() for k, v in arrays.items()}
            entry["epochs"][tag]["ovf_count_value"] = struct.unpack("<I", arrays["ovf_count"])[0]
        result[name] = entry
        os.remove(cout)  # the full-size dump is about 0.8 GB
    with open(os.path.join(out_dir, out_name), "w") as f:
        json.dump(result, f, indent=1, sort_keys=True)
    print("wrote", os.path.join(out_dir, out_name))


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--run", metavar="OUT_DIR")
    ap.add_argument("--run-scale", metavar="OUT_DIR")
    ap.add_argument("--list", action="store_true")
    a = ap.parse_args()
    if a.run:
        run(a.run)
    elif a.run_scale:
        run(a.run_scale, SCALE_CASES, "ref_epochs_c1.json")
    else:
        for name in CASES:
            c = build_case(name)
            print(name, "n=%d nnz=%d init=%d bench=%d tags=%d hd=%d" % (
                len(c["rp"]) - 1, len(c["col"]), len(c["init"]), len(c["bench"]), len(epoch_tags(c)),
                int((c["deg"] > c["thr"]).sum())))
