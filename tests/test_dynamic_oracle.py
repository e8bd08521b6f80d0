"""CPU: the DSL's own batch arithmetic for DynTC and DynCF (oracle/dynamic_dsl.py, a
restatement of dynamicBatchTCV2 and dynamicBatchClustering) against exact recounts.
On the batches that the library's incremental paths count (a symmetric graph, each
undirected update given in both directions) with every deletion naming an edge and
every addition a new one, DynTC's count1/2 + count2/4 + count3/6 is exact, which is
the weighting sp_tc_dynamic uses. The DSL departs from the recount on deletions of
absent edges and on additions of present ones, which the library does not follow, and
DynCF moves each vertex once per direction of an update, twice per triangle."""
import numpy as np
import pytest

from oracle import dynamic_dsl as D
from oracle import oracle as O


def _graph(rng, V, m):
    edges = set()
    while len(edges) < 2 * m:
        a, b = (int(x) for x in rng.integers(0, V, 2))
        if a != b:
            edges |= {(a, b), (b, a)}
    return edges


def _clean_batch(rng, V, edges, n):
    """n undirected updates, both directions: deletions of held edges, additions of
    absent ones, no pair twice, no self-loops."""
    held = sorted((a, b) for a, b in edges if a < b)
    seen, batch = set(), []
    while len(seen) < n:
        if rng.integers(0, 2) and held:
            a, b = held[rng.integers(0, len(held))]
            t = "d"
        else:
            a, b = sorted(int(x) for x in rng.integers(0, V, 2))
            if a == b or (a, b) in edges:
                continue
            t = "a"
        if (a, b) in seen:
            continue
        seen.add((a, b))
        batch += [(t, a, b), (t, b, a)]
    return batch


def _tc(V, edges):
    off, adj = D.csr(V, edges)
    return O.tc(off, adj)


@pytest.mark.parametrize("seed", range(6))
def test_dsl_dyntc_is_exact_on_clean_symmetric_batches(seed):
    rng = np.random.default_rng(seed)
    V = 40
    edges = _graph(rng, V, 160)
    count = _tc(V, edges)
    for n in (1, 5, 30):
        batch = _clean_batch(rng, V, edges, n)
        count, edges = D.dyn_tc_dsl(V, edges, count, batch)
        assert count == _tc(V, edges)


def test_dsl_dyntc_counts_a_deletion_of_an_absent_edge():
    # (0, 1) is absent, but 0 and 1 share the neighbour 2: the DSL's Decremental still
    # walks it and removes a triangle that never existed
    edges = {(0, 2), (2, 0), (1, 2), (2, 1), (2, 3), (3, 2), (0, 3), (3, 0)}
    V = 4
    count = _tc(V, edges)
    got, new = D.dyn_tc_dsl(V, edges, count, [("d", 0, 1), ("d", 1, 0)])
    assert new == edges and _tc(V, new) == count
    assert got == count - 1


@pytest.mark.parametrize("seed", range(4))
def test_dsl_dyncf_moves_vertices_twice_per_triangle(seed):
    # one undirected update, given in both directions: every triangle through it is found
    # once from each direction, so the DSL moves cf by twice the exact change (the library
    # moves it once per triangle)
    rng = np.random.default_rng(seed)
    V = 30
    edges = _graph(rng, V, 120)
    off, adj = D.csr(V, edges)
    cf = O.lcc(off, adj)
    for _ in range(4):
        batch = _clean_batch(rng, V, edges, 1)
        got, new = D.dyn_cf_dsl(V, edges, cf.tolist(), batch)
        off, adj = D.csr(V, new)
        exact = O.lcc(off, adj)
        assert np.array_equal(np.array(got) - cf, 2 * (exact - cf))
        cf, edges = exact, new
