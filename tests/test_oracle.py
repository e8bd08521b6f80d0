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


def test_lcc_reference_harness_and_identities():
    # per-vertex counts of the clustering_coeff loop: the reference's own check_if_nbr
    # loop agrees (when it was built here), every triple found adds three, and each
    # vertex of a clique K_n lies in C(n-1, 2) triangles
    for g in [G.rmat(10, 8, seed=11), clique(12), G.rmat(9, 8, seed=2, directed=True)]:
        cf = O.lcc(g.indexofNodes, g.edgeList)
        assert int(cf.astype(np.int64).sum()) == 3 * O.tc(g.indexofNodes, g.edgeList)
        if O.ref_lib() is not None:
            assert np.array_equal(O.ref_lcc(g.indexofNodes, g.edgeList), cf)
    assert np.all(O.lcc(clique(12).indexofNodes, clique(12).edgeList) == 55)


def test_closeness_known_answers():
    # path 0-1-2-3 (both directions), weights 1, 2, 3: weighted sums from 0 and 3 are
    # 1+3+6 = 10 and 3+5+6 = 14; BFS level sums 1+2+3 = 6 from either end; vertex 4 is
    # isolated (sum 0 -> +inf); non-sources stay 0
    from graphs import from_pairs

    g = from_pairs(5, [[0, 1], [1, 2], [2, 3]], symmetrize=True, name="path")
    w = np.zeros(g.E, np.int32)
    for u in range(g.V):
        for e in range(g.indexofNodes[u], g.indexofNodes[u + 1]):
            w[e] = min(u, g.edgeList[e]) + 1
    cc = O.closeness(g.indexofNodes, g.edgeList, w, [0, 3, 4])
    assert cc[0] == np.float32(1.0 / 10) and cc[3] == np.float32(1.0 / 14) and np.isinf(cc[4])
    assert cc[1] == 0 and cc[2] == 0
    cu = O.closeness_unweighted(g.indexofNodes, g.edgeList, [0, 3])
    assert cu[0] == np.float32(1.0 / 6) and cu[3] == np.float32(1.0 / 6) and cu[1] == 0
    assert np.array_equal(O.degree(g.indexofNodes), [1, 2, 2, 1, 0])


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
