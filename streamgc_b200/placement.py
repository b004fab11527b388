"""Placement of independent graphs (batched form) or tenants (served form) on
the GPUs of one node.

Graphs and tenants share nothing, so each GPU runs its own batched handle or
server over its share and no collective is on the data path; only the
metrics are combined on the host. Shares are balanced by resident bytes (the
served form's admission footprint, `sgc_tenant_footprint`): largest first,
each onto the GPU with the fewest bytes so far (ties to the lower rank), so
every rank computes the same placement from the same list.
"""

# Expected adjacency entries (2 x undirected edges) per vertex of the
# generators' families, for placing graphs before they are built.
_ENTRIES_PER_VERTEX = {
    "delaunay": 6.0,   # planar triangulation: average degree just under 6
    "chung_lu": 17.0,  # expected average degree 17
    "rmat": 82.0,      # edge factor 48, about 85 % distinct after symmetrizing
}


def expected_entries(spec):
    """Adjacency entries a workload spec (`workloads.batch_specs`) is expected
    to produce; R-MAT specs named `rmatS` with an explicit edge factor use it."""
    n = int(spec["n"])
    fam = spec["family"]
    if fam in _ENTRIES_PER_VERTEX:
        return int(_ENTRIES_PER_VERTEX[fam] * n)
    if fam.startswith("rmat"):
        ef = float(spec.get("edge_factor", 16))
        return int(2 * 0.9 * ef * n)
    raise ValueError(f"unknown family {fam!r}")


def footprint(n, entries, slack_pct=300):
    """Resident bytes of a graph of n vertices and `entries` adjacency entries
    (the served form's admission formula)."""
    import streamgc_b200 as S
    return int(S.Server.footprint(n, entries, slack_pct))


def spec_footprint(spec, slack_pct=300):
    return footprint(int(spec["n"]), expected_entries(spec), slack_pct)


def place(footprints, world):
    """Indices of `footprints` per rank (each list ascending): largest first onto
    the least-loaded rank."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(footprints)), key=lambda i: (-footprints[i], i))
    load = [0] * world
    out = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        out[r].append(i)
        load[r] += footprints[i]
    return [sorted(x) for x in out]


def imbalance(footprints, shares):
    """Largest share over the mean share (1.0 = perfectly balanced)."""
    loads = [sum(footprints[i] for i in s) for s in shares]
    mean = sum(loads) / len(loads)
    return max(loads) / mean if mean else 1.0
