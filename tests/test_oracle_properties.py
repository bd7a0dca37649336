"""Invariants of the oracle's coarsening on random graphs (CPU only).

The oracle is the checker every GPU parity test compares against, so its own
contraction and aggregation are held to the properties the reference's
--verify checks state (coarsen.cu:1835-1902): a contracted level is a
symmetric CSR with sorted, duplicate-free rows and no self loops, its edge
weight is the fine weight between different clusters, its vertex weights are
the clusters' sums; an aggregation map covers every coarse id and keeps every
cluster within the returned cap (max(heaviest vertex, average cap), so a
singleton never exceeds it).  Hypothesis draws the graphs derandomized: the
same examples every run."""
import numpy as np
from hypothesis import assume, given, settings, strategies as st

import pyoracle as O


def random_symmetric(n, density, seed, weighted):
    """Symmetric CSR without self loops; weights equal in both directions."""
    rng = np.random.default_rng(seed)
    pairs = rng.random((n, n)) < density
    upper = np.triu(pairs, 1)
    sym = upper | upper.T
    w = rng.integers(1, 50, size=(n, n)) if weighted else np.ones((n, n), np.int64)
    w = np.triu(w, 1)
    w = w + w.T
    off = np.zeros(n + 1, np.int64)
    nbr, ew = [], []
    for v in range(n):
        row = np.nonzero(sym[v])[0]
        off[v + 1] = off[v] + len(row)
        nbr.extend(row.tolist())
        ew.extend(w[v, row].tolist())
    vw = rng.integers(1, 5, size=n) if weighted else None
    return O.Graph(off, np.array(nbr, np.int32), np.array(ew, np.uint64) if weighted else None,
                   None if vw is None else vw.astype(np.uint64))


def edge_weights(g):
    return g.ew if g.ew is not None else np.ones(len(g.nbr), np.uint64)


def vertex_weights(g):
    return g.vw if g.vw is not None else np.ones(g.n, np.uint64)


def assert_valid_level(g):
    """Symmetric (equal reverse weights), rows strictly ascending, no self loops."""
    w = edge_weights(g)
    entries = {}
    for v in range(g.n):
        row = g.nbr[g.off[v]:g.off[v + 1]]
        assert np.all(np.diff(row) > 0), f"row {v} not strictly ascending"
        assert not np.any(row == v), f"self loop at {v}"
        for j, u in enumerate(row):
            entries[(v, int(u))] = int(w[g.off[v] + j])
    for (v, u), x in entries.items():
        assert entries.get((u, v)) == x, f"edge {v}-{u} not symmetric"


@settings(max_examples=40, deadline=None, derandomize=True)
@given(n=st.integers(2, 60), density=st.floats(0.02, 0.4), seed=st.integers(0, 10**6),
       groups=st.integers(1, 20), weighted=st.booleans())
def test_contraction_invariants(n, density, seed, groups, weighted):
    g = random_symmetric(n, density, seed, weighted)
    rng = np.random.default_rng(seed + 1)
    c = min(groups, n)
    mp = rng.integers(0, c, size=n).astype(np.int32)
    mp[:c] = np.arange(c)                     # every coarse id is used
    cg = O.contract(g, mp, c)
    assert cg.n == c
    assert_valid_level(cg)
    src = np.repeat(mp, np.diff(g.off))
    dst = mp[g.nbr]
    crossing = int(edge_weights(g)[src != dst].sum())
    assert int(edge_weights(cg).sum()) == crossing
    assert np.array_equal(vertex_weights(cg), np.bincount(mp, weights=vertex_weights(g), minlength=c).astype(np.uint64))


@settings(max_examples=30, deadline=None, derandomize=True)
@given(n=st.integers(4, 80), density=st.floats(0.02, 0.3), seed=st.integers(0, 10**6),
       parts=st.sampled_from([2, 4, 8, 32]), weighted=st.booleans())
def test_aggregation_invariants(n, density, seed, parts, weighted):
    g = random_symmetric(n, density, seed, weighted)
    mp, cn, cap = O.aggregate(g, parts, seed % 7, 0)
    assert 1 <= cn <= n
    assert mp.min() >= 0 and mp.max() == cn - 1
    assert len(np.unique(mp)) == cn                # every coarse id covers a cluster
    weights = np.bincount(mp, weights=vertex_weights(g), minlength=cn)
    assert weights.max() <= cap                    # no cluster above the cap
    assert_valid_level(O.contract(g, mp, cn))


@settings(max_examples=25, deadline=None, derandomize=True)
@given(n=st.integers(64, 220), density=st.floats(0.02, 0.12), seed=st.integers(0, 10**6),
       parts=st.sampled_from([2, 4, 8]), weighted_edges=st.booleans())
def test_partition_invariants(n, density, seed, parts, weighted_edges):
    """The oracle's whole pipeline: labels in [0, k), every part within the
    capacity floor(1.03 n / k) (unit vertex weights, n >= 8k, and only the n
    whose capacities hold the total), the reported cut equal to an exact
    recount; a further
    refinement from its result never raises the cut and keeps the capacity."""
    # integer capacities can fall short of the total (n = 121, k = 8: 8 x 15);
    # the reference rejects those inputs (the capacity tests check that), so
    # only the totals its capacity rule accepts are drawn
    try:
        cap = O.partition_capacity(n, parts, 1.03)
    except O.OracleError:
        assume(False)
    g = random_symmetric(n, density, seed, False)
    if weighted_edges:
        g = O.Graph(g.off, g.nbr, random_symmetric(n, density, seed, True).ew, None)
    labels, cut = O.partition(g, parts, seed=seed % 5)
    assert labels.min() >= 0 and labels.max() < parts
    directed, loads = O.recount(g, labels, parts)
    assert directed // 2 == cut
    assert loads.max() <= cap
    again, st_ = O.refine(g, labels, parts)
    d2, loads2 = O.recount(g, again, parts)
    assert d2 // 2 == st_.final_cut <= st_.initial_cut == cut
    assert loads2.max() <= cap
