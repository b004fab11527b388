"""The same-edge ordering of the concurrent apply (sgc_kernels.cu
conc_prep_insert / conc_prep_prev / conc_apply_kernel), checked on a model:
updates push themselves onto their edge's list in an arbitrary order (the
atomic exchange of the prep kernel), each finds its previous and next update
of the same edge by walking that list, and the first update of each edge then
applies the edge's updates by following the next links. Every update is
applied exactly once, each edge's updates in stream order."""
import random

NONE = None


def _model(seed):
    rnd = random.Random(seed)
    n = rnd.randint(1, 300)
    keys = [rnd.randint(0, max(1, n // rnd.choice([1, 2, 5, 20]))) for _ in range(n)]
    head, nxt = {}, [NONE] * n
    for i in rnd.sample(range(n), n):  # pushes in any order
        nxt[i] = head.get(keys[i], NONE)
        head[keys[i]] = i
    prev, succ = [NONE] * n, [NONE] * n
    for i in range(n):  # each update walks its list
        j = head[keys[i]]
        while j is not NONE:
            if j < i and (prev[i] is NONE or j > prev[i]):
                prev[i] = j
            if j > i and (succ[i] is NONE or j < succ[i]):
                succ[i] = j
            j = nxt[j]
    applied = []
    for i in rnd.sample(range(n), n):  # tickets taken in any order; only first updates walk their edge
        if prev[i] is not NONE:
            continue
        j = i
        while j is not NONE:
            applied.append(j)
            j = succ[j]
    assert sorted(applied) == list(range(n))
    for k in set(keys):
        order = [j for j in applied if keys[j] == k]
        assert order == sorted(order)


def test_each_edge_applied_in_stream_order_once():
    for s in range(400):
        _model(s)
