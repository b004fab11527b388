"""The hole-count rule of concurrent row inserts (sgc_device.cuh::extend_row),
checked on a model of one row: inserts are split into their atomic steps (scan
for a free slot, compare-and-swap it, raise the high-water mark and account)
and deletes into theirs, and the steps of many operations interleave at
random. At quiescence the count must equal the free slots below the mark, and
every slot past the mark must be free. The earlier rule (a slot filled below
the old mark uncounts a hole, nothing else) fails the same check."""
import random

INV = None


def _run(seed, gap_rule):
    rnd = random.Random(seed)
    cap = 64
    row = [INV] * cap
    k0 = rnd.randint(0, 20)  # a compacted row: k0 live entries, mark k0, no holes
    for i in range(k0):
        row[i] = 1000 + i
    st = {"hw": k0, "holes": 0}

    def insert(v):
        frm = 0
        while True:
            p = next((i for i in range(frm, cap) if row[i] is INV), None)
            yield
            if p is None:
                return
            if row[p] is INV:
                row[p] = v
                yield
                prev = st["hw"]
                st["hw"] = max(prev, p + 1)
                if p < prev:
                    st["holes"] -= 1
                elif gap_rule and p > prev:
                    st["holes"] += p - prev
                return
            frm = p + 1

    def delete(v):
        p = next((i for i in range(cap) if row[i] == v), None)
        yield
        if p is not None and row[p] == v:
            row[p] = INV
            st["holes"] += 1

    present = [1000 + i for i in range(k0)]
    ops, nid = [], 5000
    for _ in range(rnd.randint(5, 40)):
        if present and rnd.random() < 0.4:
            ops.append(delete(present.pop(rnd.randrange(len(present)))))
        else:
            ops.append(insert(nid))
            nid += 1
    live = list(ops)
    while live:
        g = rnd.choice(live)
        try:
            next(g)
        except StopIteration:
            live.remove(g)
    free_inside = sum(1 for i in range(st["hw"]) if row[i] is INV)
    tail_free = all(row[i] is INV for i in range(st["hw"], cap))
    return st["holes"] == free_inside and tail_free


def test_gap_rule_keeps_the_count_exact():
    assert all(_run(s, gap_rule=True) for s in range(1500))


def test_earlier_rule_drifts():
    assert sum(not _run(s, gap_rule=False) for s in range(300)) > 100
