"""Placement of independent graphs / tenants on the GPUs of a node (host
logic, no GPU): every item lands on exactly one rank, every rank computes the
same placement, and the shares are balanced by resident bytes."""
import random

import pytest

import streamgc_b200 as S
from streamgc_b200 import placement as P
from streamgc_b200 import workloads as W


def test_every_item_on_exactly_one_rank():
    fp = [random.Random(7).randint(1, 10**9) for _ in range(257)]
    for world in (1, 2, 3, 8):
        shares = P.place(fp, world)
        assert len(shares) == world
        got = sorted(i for s in shares for i in s)
        assert got == list(range(len(fp)))
        assert all(s == sorted(s) for s in shares)


def test_same_placement_on_every_rank():
    fp = [5, 5, 5, 9, 1, 1, 7, 7, 3]
    assert P.place(fp, 4) == P.place(list(fp), 4)
    # ties go to the lower rank, largest first
    assert P.place([4, 4, 4, 4], 2) == [[0, 2], [1, 3]]


def test_largest_first_bound():
    # greedy largest-first: no rank exceeds the mean by more than the largest item
    rng = random.Random(3)
    for _ in range(20):
        fp = [rng.randint(1, 1000) for _ in range(rng.randint(1, 60))]
        world = rng.randint(1, 8)
        loads = [sum(fp[i] for i in s) for s in P.place(fp, world)]
        assert max(loads) <= sum(fp) / world + max(fp)


def test_more_ranks_than_items():
    shares = P.place([10, 20], 4)
    assert sorted(len(s) for s in shares) == [0, 0, 1, 1]
    with pytest.raises(ValueError):
        P.place([1], 0)


def test_batched_specs_balance_on_eight_ranks():
    specs = W.batch_specs(256, seed=42)
    fp = [P.spec_footprint(sp) for sp in specs]
    assert P.imbalance(fp, P.place(fp, 8)) < 1.05


def test_expected_entries_and_footprint():
    assert P.expected_entries(dict(family="delaunay", n=1000)) == 6000
    assert P.expected_entries(dict(family="chung_lu", n=1000)) == 17000
    assert P.expected_entries(dict(family="rmat22", n=1 << 22, edge_factor=16)) == int(2 * 0.9 * 16 * (1 << 22))
    with pytest.raises(ValueError):
        P.expected_entries(dict(family="grid", n=4))
    assert P.footprint(1000, 6000) == S.Server.footprint(1000, 6000, 300)
    assert P.spec_footprint(dict(family="delaunay", n=1000)) == S.Server.footprint(1000, 6000, 300)
