"""The per-row accounting of concurrent row edits (sgc_device.cuh::extend_row
and the delete paths), checked on a model of one row: inserts are split into
their atomic steps (scan for a free slot, compare-and-swap it, raise the
high-water mark, count the entry) and deletes into theirs (find, swap the
slot free, uncount), and the steps of many operations interleave at random.
At quiescence the mark minus the live count must equal the free slots below
the mark, and every slot past the mark must be free.

Rules modelled: "live" (the one the kernels use: every step a reduction whose
result nobody waits for), "gap" (a hole counter corrected from the mark the
raise returned, exact as well but it waits for that value) and "below_mark"
(uncount a hole only when the slot lay below the old mark, which drifts)."""
import random

INV = None


def _run(seed, rule):
    rnd = random.Random(seed)
    cap = 64
    row = [INV] * cap
    k0 = rnd.randint(0, 20)  # a compacted row: k0 live entries, mark k0, no holes
    for i in range(k0):
        row[i] = 1000 + i
    st = {"hw": k0, "holes": 0, "live": k0}

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
                if rule == "live":
                    st["hw"] = max(st["hw"], p + 1)  # reduction: max
                    yield
                    st["live"] += 1  # reduction: add
                    return
                prev = st["hw"]
                st["hw"] = max(prev, p + 1)
                if p < prev:
                    st["holes"] -= 1
                elif rule == "gap" and p > prev:
                    st["holes"] += p - prev
                return
            frm = p + 1

    def delete(v):
        p = next((i for i in range(cap) if row[i] == v), None)
        yield
        if p is not None and row[p] == v:
            row[p] = INV
            yield
            st["holes"] += 1
            st["live"] -= 1

    present = [1000 + i for i in range(k0)]
    ops, nid = [], 5000
    for _ in range(rnd.randint(5, 40)):
        if present and rnd.random() < 0.4:
            ops.append(delete(present.pop(rnd.randrange(len(present)))))
        else:
            ops.append(insert(nid))
            nid += 1
    pending = list(ops)
    while pending:
        g = rnd.choice(pending)
        try:
            next(g)
        except StopIteration:
            pending.remove(g)
    free_inside = sum(1 for i in range(st["hw"]) if row[i] is INV)
    tail_free = all(row[i] is INV for i in range(st["hw"], cap))
    holes = st["hw"] - st["live"] if rule == "live" else st["holes"]
    return holes == free_inside and tail_free


def test_live_count_is_exact():
    assert all(_run(s, "live") for s in range(1500))


def test_gap_rule_keeps_the_count_exact():
    assert all(_run(s, "gap") for s in range(1500))


def test_below_mark_rule_drifts():
    assert sum(not _run(s, "below_mark") for s in range(300)) > 100
