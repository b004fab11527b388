"""Tier-2's ordered greedy (sgc_tier2.cu::ordered_greedy), checked on a model:
list vertices are recolored in rounds, a vertex going once no lower-id list
neighbor is pending; after a cap on the rounds the rest go in ascending order
on one warp. The colors equal those of the sequential ascending greedy, for
any cap."""
import random


def _greedy_color(v, adj, color):
    used = {color[w] for w in adj[v] if w != v and color[w]}
    c = 1
    while c in used:
        c += 1
    return c


def _sequential(L, adj, color):
    color = dict(color)
    for v in sorted(L):
        color[v] = _greedy_color(v, adj, color)
    return color


def _rounds(L, adj, color, cap):
    color = dict(color)
    inL, done = set(L), set()
    rem = sorted(L)
    rounds = 0
    while rem and rounds < cap:
        ready = [v for v in rem if not any(w < v and w in inL and w not in done for w in adj[v])]
        for v in ready:  # no two ready vertices are adjacent (the higher one waits for the lower)
            color[v] = _greedy_color(v, adj, color)
        done.update(ready)
        rem = [v for v in rem if v not in done]
        rounds += 1
    for v in rem:  # the tail, ascending
        color[v] = _greedy_color(v, adj, color)
    return color


def test_capped_rounds_match_the_sequential_greedy():
    rnd = random.Random(5)
    for t in range(120):
        n = rnd.randint(2, 80)
        adj = {v: set() for v in range(n)}
        for _ in range(rnd.randint(0, 4 * n)):
            a, b = rnd.randrange(n), rnd.randrange(n)
            if a != b:
                adj[a].add(b)
                adj[b].add(a)
        color = {v: rnd.randint(0, 4) for v in range(n)}
        L = rnd.sample(range(n), rnd.randint(1, n))
        want = _sequential(L, adj, color)
        for cap in (0, 1, 2, 5, 1024):
            assert _rounds(L, adj, color, cap) == want, (t, cap)
