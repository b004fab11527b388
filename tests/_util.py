"""Shared drivers for parity tests: run one golden case through the oracle or
through the CUDA path with the reference's batch / epoch protocol, yielding the
state arrays at every epoch boundary and after each drain_and_compact."""
import hashlib

import numpy as np

from oracle import oracle as O

ARRAY_NAMES = ("states", "bitmaps", "col", "snapshot", "hist", "ovf_count")


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def _phases(c):
    return (("init", c["init"]), ("bench", c["bench"]))


def oracle_epochs(c):
    g = O.Oracle(c["rp"], c["col"], c["deg"], hist_threshold=c["thr"], slack_pct=c["slack"])
    k = 0

    def grab(g):
        return dict(states=g.states(), bitmaps=g.bitmaps(), col=g.col(), snapshot=g.snapshot(), hist=g.hist(),
                    ovf_count=np.array([g.overflow_count()], dtype=np.uint32))

    for phase, ups in _phases(c):
        since = 0
        for s in range(0, len(ups), c["batch"]):
            part = ups[s:s + c["batch"]]
            g.apply(part)
            since += len(part)
            if since >= c["E"]:
                g.epoch()
                yield f"{phase}_e{k}", grab(g)
                k += 1
                since = 0
        g.drain_and_compact()
        yield f"{phase}_dc", grab(g)


def gpu_epochs(c, mode=0):
    import streamgc_b200 as S
    graph = S.Graph(c["rp"], c["col"], c["deg"])
    h = S.StreamGC(graph, epoch_size=c["E"], histogram_threshold=c["thr"], slack_pct=c["slack"],
                   max_batch=max(c["batch"], 1))
    k = 0

    def grab():
        st = h.stats()
        return dict(states=h.states(), bitmaps=h.bitmaps(), col=h.col(), snapshot=h.snapshot(), hist=h.hist(),
                    ovf_count=np.array([st["overflow_pending"]], dtype=np.uint32))

    try:
        for phase, ups in _phases(c):
            since = 0
            for s in range(0, len(ups), c["batch"]):
                part = ups[s:s + c["batch"]]
                h.apply(part, mode)
                since += len(part)
                if since >= c["E"]:
                    h.epoch()
                    yield f"{phase}_e{k}", grab()
                    k += 1
                    since = 0
            h.drain_and_compact()
            yield f"{phase}_dc", grab()
    finally:
        h.close()
