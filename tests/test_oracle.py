"""CPU tests: the oracle against independent computations (networkx, dense
numpy) and against the reference's own graph.hpp / check_if_nbr where the
reference-compiled harness is present."""
import numpy as np
import pytest

from oracle import oracle as O
from starplat_b200 import generators as G

from graphs import clique, directed_zoo, path, star, undirected_zoo

nx = pytest.importorskip("networkx")


def to_nx(g, directed=False, weights=None):
    H = nx.DiGraph() if directed else nx.Graph()
    H.add_nodes_from(range(g.V))
    off, adj = g.indexofNodes, g.edgeList
    for u in range(g.V):
        for e in range(off[u], off[u + 1]):
            if weights is None:
                H.add_edge(u, int(adj[e]))
            else:
                H.add_edge(u, int(adj[e]), weight=int(weights[e]))
    return H


def tc_formula(g):
    """The DSL formula by brute force over edge sets (small graphs only)."""
    off, adj = g.indexofNodes, g.edgeList
    nbr = [set(adj[off[v]:off[v + 1]].tolist()) for v in range(g.V)]
    c = 0
    for v in range(g.V):
        for u in nbr[v]:
            if u < v:
                for w in nbr[v]:
                    if w > v and w in nbr[u]:
                        c += 1
    return c


@pytest.mark.parametrize("gi", range(6))
def test_tc_oracle_vs_networkx(gi):
    g = undirected_zoo()[gi]
    if g.V > 5000:
        pytest.skip("large")
    H = to_nx(g)
    assert O.tc(g.indexofNodes, g.edgeList) == sum(nx.triangles(H).values()) // 3


def test_tc_oracle_directed_formula():
    for g in directed_zoo():
        if g.E > 60000:
            continue
        assert O.tc(g.indexofNodes, g.edgeList) == tc_formula(g)


def test_tc_omp_form_equals_exact():
    g = G.rmat(10, 8, seed=11)
    assert O.tc_omp(g.indexofNodes, g.edgeList) == O.tc(g.indexofNodes, g.edgeList)


def test_tc_reference_harness():
    if O.ref_lib() is None:
        pytest.skip("reference harness not built (no reference checkout)")
    for g in [G.rmat(10, 8, seed=11), clique(12), G.rmat(9, 8, seed=2, directed=True)]:
        assert O.ref_tc(g.indexofNodes, g.edgeList) == O.tc(g.indexofNodes, g.edgeList)


def dense_pagerank(g, beta, delta, max_iter):
    V = g.V
    A = np.zeros((V, V))
    od = g.out_degree()
    for u in range(V):
        for e in range(g.indexofNodes[u], g.indexofNodes[u + 1]):
            A[g.edgeList[e], u] += 1.0 / od[u]
    pr = np.full(V, 1.0 / V)
    it = 0
    while True:
        nxt = (1 - delta) / V + delta * (A @ pr)
        diff = np.abs(nxt - pr).sum()
        pr = nxt
        it += 1
        if not (diff > beta and it < max_iter):
            break
    return pr, it


@pytest.mark.parametrize("gi", [0, 3])
def test_pagerank_oracle_vs_dense(gi):
    g = directed_zoo()[gi]
    g.ensure_reverse()
    pr, it, _ = O.pagerank(g.indexofNodes, g.rev_indexofNodes, g.srcList, 1e-6, 0.85, 100)
    ref, rit = dense_pagerank(g, 1e-6, 0.85, 100)
    assert it == rit
    assert np.abs(pr - ref).sum() < 1e-12


def test_pagerank_omp_form_close():
    g = directed_zoo()[0]
    g.ensure_reverse()
    pr, it, _ = O.pagerank(g.indexofNodes, g.rev_indexofNodes, g.srcList, 1e-6, 0.85, 100)
    pf, itf = O.pagerank_omp(g.indexofNodes, g.rev_indexofNodes, g.srcList, 1e-6, 0.85, 100)
    assert abs(it - itf) <= 2
    assert np.abs(pf.astype(np.float64) - pr).sum() < 1e-4
