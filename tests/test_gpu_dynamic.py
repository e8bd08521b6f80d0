"""GPU: batches of edge updates applied to the device mirror (sp_graph_update, the
role of graph::updateCSRDel / updateCSRAdd). The updated CSR equals the one built from
the edge set on the host (deletions first, then additions, duplicate additions summed),
and every algorithm then runs on it and matches the oracle."""
import numpy as np
import pytest

from oracle import oracle as O
from starplat_b200 import _lib
from starplat_b200 import generators as G
from starplat_b200.device import DeviceGraph

from graphs import from_pairs

pytestmark = pytest.mark.gpu


def _edges(off, adj, w):
    src = np.repeat(np.arange(len(off) - 1), np.diff(off))
    return {(int(a), int(b)): int(c) for a, b, c in zip(src, adj, w)}


def _apply(edges, types, src, dst, w):
    out = dict(edges)
    for t, a, b in zip(types, src, dst):
        if t == "d":
            out.pop((int(a), int(b)), None)
    for t, a, b, c in zip(types, src, dst, w):
        if t == "a":
            out[(int(a), int(b))] = out.get((int(a), int(b)), 0) + int(c)
    return out


def _csr(V, edges):
    keys = sorted(edges)
    off = np.zeros(V + 1, np.int32)
    for a, _ in keys:
        off[a + 1] += 1
    off = np.cumsum(off).astype(np.int32)
    adj = np.array([b for _, b in keys], np.int32)
    w = np.array([edges[k] for k in keys], np.int32)
    return off, adj, w


def _batch(rng, V, edges, n):
    ex = list(edges)
    types, src, dst, w = [], [], [], []
    for _ in range(n):
        kind = rng.integers(0, 4)
        if kind == 0 and ex:  # delete an existing edge
            a, b = ex[rng.integers(0, len(ex))]
            types.append("d")
        elif kind == 1:  # delete an edge that may not exist
            a, b = rng.integers(0, V, 2)
            types.append("d")
        elif kind == 2 and ex:  # add an existing edge (weights summed)
            a, b = ex[rng.integers(0, len(ex))]
            types.append("a")
        else:  # add a new edge, self-loops included
            a, b = rng.integers(0, V, 2)
            types.append("a")
        src.append(int(a))
        dst.append(int(b))
        w.append(int(rng.integers(1, 50)))
    return "".join(types), np.array(src, np.int32), np.array(dst, np.int32), np.array(w, np.int32)


def test_update_batches_match_the_host_edge_set():
    rng = np.random.default_rng(11)
    g = G.rmat(12, 8, seed=3, directed=True)
    g.edgeLen = G.hash_weights(g, 3, 1, 50, False)
    edges = _edges(g.indexofNodes, g.edgeList, g.edgeLen)
    with DeviceGraph.from_csr(g) as dg:
        for step in range(4):
            t, s, d, w = _batch(rng, g.V, edges, [1, 50, 700, 3000][step])
            dg.update(t, s, d, w)
            edges = _apply(edges, t, s, d, w)
            off, adj, ww = _csr(g.V, edges)
            got = dg.export()
            assert np.array_equal(got["indexofNodes"], off) and np.array_equal(got["edgeList"], adj)
            assert np.array_equal(got["edgeLen"], ww)
            # the reverse CSR is rebuilt from the new forward CSR
            rs = np.argsort(adj, kind="stable")
            assert np.array_equal(got["srcList"], np.repeat(np.arange(g.V), np.diff(off))[rs])
            # algorithms run on the updated graph
            src = int(s[0])
            dist, _ = dg.sssp(src)
            assert np.array_equal(dist, O.sssp(off, adj, ww, src))
            roff = np.zeros(g.V + 1, np.int32)
            roff[1:] = np.cumsum(np.bincount(adj, minlength=g.V))
            radj = np.repeat(np.arange(g.V), np.diff(off))[rs].astype(np.int32)
            pr, it, _ = dg.pagerank(1e-6, 0.85, 100)
            ref, rit, _ = O.pagerank(off, roff, radj, 1e-6, 0.85, 100)
            assert abs(it - rit) <= 2 and np.abs(pr.astype(np.float64) - ref).sum() < 1e-5
            assert dg.tc() == O.tc(off, adj)


def test_update_undirected_keeps_symmetry_and_counts():
    # adding and deleting both directions of undirected edges: triangles, BC and
    # Louvain see the updated symmetric graph
    g = G.rmat(11, 8, seed=5)
    edges = _edges(g.indexofNodes, g.edgeList, np.ones(g.E, np.int32))
    rng = np.random.default_rng(2)
    pairs = rng.integers(0, g.V, (300, 2))
    t = "d" * 150 + "a" * 150
    src = np.concatenate([pairs[:150, 0], pairs[:150, 1], pairs[150:, 0], pairs[150:, 1]]).astype(np.int32)
    dst = np.concatenate([pairs[:150, 1], pairs[:150, 0], pairs[150:, 1], pairs[150:, 0]]).astype(np.int32)
    types = "d" * 300 + "a" * 300
    with DeviceGraph.from_csr(g, with_weights=False) as dg:
        assert dg.tc() == O.tc(g.indexofNodes, g.edgeList)
        dg.update(types, src, dst)
        w1 = np.ones(src.shape[0], np.int32)
        edges = _apply(edges, types, src, dst, w1)
        off, adj, _ = _csr(g.V, edges)
        got = dg.export()
        assert np.array_equal(got["indexofNodes"], off) and np.array_equal(got["edgeList"], adj)
        assert "edgeLen" not in got  # a graph without weights stays without
        assert dg.tc() == O.tc(off, adj)
        srcs = G.pick_sources(g, 20, seed=3)
        bc = dg.bc(srcs).astype(np.float64)
        rbc = O.bc(off, adj, srcs)
        assert np.all(np.abs(bc - rbc) <= 1e-5 * np.abs(rbc) + 1e-6)
        assert np.array_equal(dg.clustering_coeff(), O.lcc(off, adj))
    del t


def test_update_edge_cases():
    g = from_pairs(4, [[0, 1], [1, 2], [2, 3]], name="path4")
    g.edgeLen = np.array([5, 6, 7], np.int32)
    with DeviceGraph.from_csr(g) as dg:
        dg.update("", [], [])  # an empty batch changes nothing
        assert dg.E == 3
        # delete every edge, then add them back in another order with new weights
        dg.update("ddd", [0, 1, 2], [1, 2, 3])
        assert dg.E == 0
        assert np.array_equal(dg.export()["indexofNodes"], [0, 0, 0, 0, 0])
        dg.update("aaaa", [2, 0, 1, 0], [3, 1, 2, 1], [1, 2, 3, 4])
        got = dg.export()
        assert got["edgeList"].tolist() == [1, 2, 3] and got["edgeLen"].tolist() == [6, 3, 1]
        # a deletion and an addition of the same edge in one batch: deleted first, then added
        dg.update("ad", [0, 0], [1, 1], [9, 0])
        assert dg.export()["edgeLen"].tolist() == [9, 3, 1]
        dist, _ = dg.sssp(0)
        assert dist.tolist() == [0, 9, 12, 13]
        # bad batches are rejected whole and leave the graph as it was
        for t, s, d in (("a", [4], [0]), ("d", [0], [-1]), ("x", [0], [1])):
            with pytest.raises(_lib.SPError):
                dg.update(t, s, d)
        assert dg.export()["edgeLen"].tolist() == [9, 3, 1]


def test_sssp_dynamic_additions_resume_and_deletions_repair():
    # DynSSSP's batch: additions resume from the old distances (and relax far fewer
    # edges than a fresh solve); a batch with deletions repairs through parents (weights
    # >= 1 here); exact every way
    rng = np.random.default_rng(4)
    g = G.rmat(14, 8, seed=9, directed=True)
    g.edgeLen = G.hash_weights(g, 9, 1, 100, False)
    edges = _edges(g.indexofNodes, g.edgeList, g.edgeLen)
    source = int(G.pick_sources(g, 1, seed=4)[0])
    with DeviceGraph.from_csr(g) as dg:
        dist, _ = dg.sssp(source)
        full = dg.tune_get("sssp.last_relaxed")
        for step in range(6):
            n = [1, 10, 200, 2000, 50, 400][step]
            if step % 3 == 2:  # mixed batch: deletions force a new solve
                t, s, d, w = _batch(rng, g.V, edges, n)
            else:  # additions only
                s = rng.integers(0, g.V, n).astype(np.int32)
                d = rng.integers(0, g.V, n).astype(np.int32)
                w = rng.integers(1, 100, n).astype(np.int32)
                t = "a" * n
            resumed = dg.sssp_dynamic(t, s, d, w, source, dist)
            held = any((int(a), int(b)) in edges for a, b in zip(s, d))
            path = dg.tune_get("sssp.last_incremental")
            if "d" in t:  # repaired, or solved again when the repair would reset > V / 4
                assert path in (0, 2) and resumed == (path == 2)
            else:
                assert resumed == (not held) and path == (1 if not held else 0)
            edges = _apply(edges, t, s, d, w)
            off, adj, ww = _csr(g.V, edges)
            assert np.array_equal(dist, O.sssp(off, adj, ww, source)), step
            if resumed and n <= 10:
                assert dg.tune_get("sssp.last_relaxed") < full // 10
    # device distances, and the errors
    import torch

    with DeviceGraph.from_csr(g) as dg:
        dd = torch.empty(g.V, dtype=torch.int32, device="cuda")
        dg.sssp(source, out=dd)
        far = int(np.argmax(np.where(O.sssp(g.indexofNodes, g.edgeList, g.edgeLen, source) == 2**31 - 1, -1,
                                     O.sssp(g.indexofNodes, g.edgeList, g.edgeLen, source))))
        assert dg.sssp_dynamic("a", [source], [far], [1], source, dd)
        e2 = _apply(_edges(g.indexofNodes, g.edgeList, g.edgeLen), "a", [source], [far], [1])
        off, adj, ww = _csr(g.V, e2)
        assert np.array_equal(dd.cpu().numpy(), O.sssp(off, adj, ww, source))
        with pytest.raises(_lib.SPError):
            dg.sssp_dynamic("a", [0], [g.V], [1], source, dd)
    h = from_pairs(3, [[0, 1], [1, 2]], name="noweights")
    with DeviceGraph.from_csr(h, with_weights=False) as dh:
        with pytest.raises(_lib.SPError):
            dh.sssp_dynamic("a", [0], [2], [1], 0, np.zeros(3, np.int32))


def test_sssp_dynamic_readding_a_held_tree_edge_solves_again():
    # an additions-only batch that adds an edge the graph already holds makes it longer
    # (the weights are summed), so distances through it rise: the call must not resume
    g = G.rmat(12, 8, seed=5, directed=True)
    g.edgeLen = G.hash_weights(g, 5, 1, 100, False)
    source = int(G.pick_sources(g, 1, seed=5)[0])
    edges = _edges(g.indexofNodes, g.edgeList, g.edgeLen)
    ref = O.sssp(g.indexofNodes, g.edgeList, g.edgeLen, source)
    # tree edges out of the source: d(v) == w(source, v), and no other edge reaches v as short
    tree = [(source, int(v)) for v in g.edgeList[g.indexofNodes[source]:g.indexofNodes[source + 1]]
            if ref[v] == edges[(source, int(v))] and int(v) != source]
    assert tree
    with DeviceGraph.from_csr(g) as dg:
        dist, _ = dg.sssp(source)
        s = np.array([a for a, _ in tree], np.int32)
        d = np.array([b for _, b in tree], np.int32)
        w = np.full(len(tree), 1000, np.int32)
        resumed = dg.sssp_dynamic("a" * len(tree), s, d, w, source, dist)
        assert not resumed
        edges = _apply(edges, "a" * len(tree), s, d, w)
        off, adj, ww = _csr(g.V, edges)
        new = O.sssp(off, adj, ww, source)
        assert np.array_equal(dist, new)
        assert (new[d] > ref[d]).any()  # some distance did rise
        # a fresh edge in the next batch resumes again
        far = int(np.argmax(np.where(new == 2**31 - 1, -1, new)))
        if (source, far) not in edges:
            assert dg.sssp_dynamic("a", [source], [far], [1], source, dist)
            edges = _apply(edges, "a", [source], [far], [1])
            off, adj, ww = _csr(g.V, edges)
            assert np.array_equal(dist, O.sssp(off, adj, ww, source))


def _tight(off, adj, w, dist):
    """(u, v) edges with dist[u] + w == dist[v]: the tight edges of the distances."""
    out = []
    for u in range(len(off) - 1):
        if dist[u] == 2**31 - 1:
            continue
        for k in range(off[u], off[u + 1]):
            v = int(adj[k])
            if int(dist[u]) + int(w[k]) == int(dist[v]):
                out.append((u, v))
    return out


@pytest.mark.parametrize("case", ["grid", "rmat"])
def test_sssp_dynamic_decremental_repair_through_parents(case):
    # deletions of tight (tree) edges reset whole subtrees, which are lowered again from
    # their unmarked in-neighbours; batches mix deletions of tree edges, other deletions,
    # lengthened tree edges (additions to held edges) and new edges; exact every batch
    import torch

    rng = np.random.default_rng(11)
    if case == "grid":
        g = G.grid(60, 70)
        g.edgeLen = G.hash_weights(g, 3, 1, 50, True)
    else:
        g = G.rmat(13, 8, seed=3, directed=True)
        g.edgeLen = G.hash_weights(g, 3, 1, 100, False)
    source = int(G.pick_sources(g, 1, seed=2)[0])
    edges = _edges(g.indexofNodes, g.edgeList, g.edgeLen)
    paths = []
    with DeviceGraph.from_csr(g) as dg:
        dg.tune_set("sssp.repair", 1)  # whatever the rounds of the first solve
        dd = torch.empty(g.V, dtype=torch.int32, device="cuda")
        dg.sssp(source, out=dd)
        for step in range(5):
            off, adj, ww = _csr(g.V, edges)
            tight = _tight(off, adj, ww, dd.cpu().numpy())
            pick = rng.choice(len(tight), min(len(tight), [5, 40, 200, 3, 60][step]), replace=False)
            dels = [tight[i] for i in pick]
            keys = list(edges)
            others = [keys[i] for i in rng.choice(len(keys), 20, replace=False)]
            longer = [tight[i] for i in rng.choice(len(tight), 5, replace=False)]
            fresh = [(int(a), int(b)) for a, b in rng.integers(0, g.V, (10, 2))]
            t = "d" * (len(dels) + len(others)) + "a" * (len(longer) + len(fresh))
            s_ = np.array([a for a, _ in dels + others + longer + fresh], np.int32)
            d_ = np.array([b for _, b in dels + others + longer + fresh], np.int32)
            w_ = np.concatenate([np.ones(len(dels) + len(others), np.int32),
                                 rng.integers(1, 30, len(longer) + len(fresh)).astype(np.int32)])
            repaired = dg.sssp_dynamic(t, s_, d_, w_, source, dd)
            paths.append(dg.tune_get("sssp.last_incremental"))
            assert paths[-1] in (0, 2) and repaired == (paths[-1] == 2)
            edges = _apply(edges, t, s_, d_, w_)
            off, adj, ww = _csr(g.V, edges)
            assert np.array_equal(dd.cpu().numpy(), O.sssp(off, adj, ww, source)), (case, step, paths[-1])
    assert 2 in paths, paths  # the repair ran (larger resets solve again)


def test_sssp_dynamic_repair_edge_cases():
    # every out-edge of the source deleted (all else unreachable), then re-added; and a
    # graph with a zero weight, where the parents need not form a forest: solve again
    g = G.grid(20, 20)
    g.edgeLen = G.hash_weights(g, 5, 1, 9, True)
    source = 210
    edges = _edges(g.indexofNodes, g.edgeList, g.edgeLen)
    outs = [(source, int(v)) for v in g.edgeList[g.indexofNodes[source]:g.indexofNodes[source + 1]]]
    with DeviceGraph.from_csr(g) as dg:
        dist, _ = dg.sssp(source)
        s_ = np.array([a for a, _ in outs], np.int32)
        d_ = np.array([b for _, b in outs], np.int32)
        ones = np.ones(len(outs), np.int32)
        dg.sssp_dynamic("d" * len(outs), s_, d_, ones, source, dist)  # resets everything: solves again
        assert dg.tune_get("sssp.last_incremental") == 0
        assert dist[source] == 0 and np.all(np.delete(dist, source) == 2**31 - 1)
        edges = _apply(edges, "d" * len(outs), s_, d_, ones)
        w_ = np.full(len(outs), 4, np.int32)
        assert dg.sssp_dynamic("a" * len(outs), s_, d_, w_, source, dist)
        edges = _apply(edges, "a" * len(outs), s_, d_, w_)
        off, adj, ww = _csr(g.V, edges)
        assert np.array_equal(dist, O.sssp(off, adj, ww, source))
    z = G.grid(12, 12)
    z.edgeLen = G.hash_weights(z, 6, 0, 5, True)
    assert (z.edgeLen == 0).any()
    ez = _edges(z.indexofNodes, z.edgeList, z.edgeLen)
    with DeviceGraph.from_csr(z) as dz:
        dist, _ = dz.sssp(0)
        k = list(ez)[:30]
        s_ = np.array([a for a, _ in k], np.int32)
        d_ = np.array([b for _, b in k], np.int32)
        ones = np.ones(len(k), np.int32)
        assert not dz.sssp_dynamic("d" * len(k), s_, d_, ones, 0, dist)
        assert dz.tune_get("sssp.last_marked") == -1
        ez = _apply(ez, "d" * len(k), s_, d_, ones)
        off, adj, ww = _csr(z.V, ez)
        assert np.array_equal(dist, O.sssp(off, adj, ww, 0))
    # the knob: sssp.repair = 0 solves again on a batch with deletions
    g2 = G.grid(16, 16)
    g2.edgeLen = G.hash_weights(g2, 8, 1, 9, True)
    e2 = _edges(g2.indexofNodes, g2.edgeList, g2.edgeLen)
    with DeviceGraph.from_csr(g2) as d2:
        dist, _ = d2.sssp(0)
        d2.tune_set("sssp.repair", 0)
        k = list(e2)[5:9]
        s_ = np.array([a for a, _ in k], np.int32)
        d_ = np.array([b for _, b in k], np.int32)
        assert not d2.sssp_dynamic("dddd", s_, d_, np.ones(4, np.int32), 0, dist)
        e2 = _apply(e2, "dddd", s_, d_, np.ones(4, np.int32))
        off, adj, ww = _csr(g2.V, e2)
        assert np.array_equal(dist, O.sssp(off, adj, ww, 0))
        d2.tune_set("sssp.repair", -1)
        with pytest.raises(_lib.SPError):
            d2.tune_set("sssp.repair", 2)


def test_sssp_dynamic_repair_policy_follows_the_rounds_of_the_last_solve():
    # by default (sssp.repair = -1) a batch with deletions repairs when the last solve
    # took at least 32 rounds, and solves again otherwise; exact either way
    chain = np.array([[i, i + 1] for i in range(399)] + [[i + 1, i] for i in range(399)], np.int32)
    p = from_pairs(400, chain, name="path400")
    p.edgeLen = G.hash_weights(p, 2, 1, 9, True)
    ep = _edges(p.indexofNodes, p.edgeList, p.edgeLen)
    with DeviceGraph.from_csr(p) as dp:
        assert dp.tune_get("sssp.repair") == -1
        dp.tune_set("sssp.delta", 1)  # one distance per bucket: hundreds of rounds
        dist, rounds = dp.sssp(0)
        assert rounds >= 32
        s_, d_ = np.array([300], np.int32), np.array([301], np.int32)
        assert dp.sssp_dynamic("d", s_, d_, np.ones(1, np.int32), 0, dist)
        assert dp.tune_get("sssp.last_incremental") == 2 and dp.tune_get("sssp.last_marked") > 0
        ep = _apply(ep, "d", s_, d_, np.ones(1, np.int32))
        off, adj, ww = _csr(p.V, ep)
        assert np.array_equal(dist, O.sssp(off, adj, ww, 0))
    g = G.rmat(12, 8, seed=7, directed=True)
    g.edgeLen = G.hash_weights(g, 7, 1, 100, False)
    eg = _edges(g.indexofNodes, g.edgeList, g.edgeLen)
    source = int(G.pick_sources(g, 1, seed=7)[0])
    with DeviceGraph.from_csr(g) as dg:
        dist, rounds = dg.sssp(source)
        k = list(eg)[:20]
        s_ = np.array([a for a, _ in k], np.int32)
        d_ = np.array([b for _, b in k], np.int32)
        dg.sssp_dynamic("d" * 20, s_, d_, np.ones(20, np.int32), source, dist)
        assert dg.tune_get("sssp.last_incremental") == (2 if rounds >= 32 else 0)
        eg = _apply(eg, "d" * 20, s_, d_, np.ones(20, np.int32))
        off, adj, ww = _csr(g.V, eg)
        assert np.array_equal(dist, O.sssp(off, adj, ww, source))


def test_update_rejects_weight_sums_outside_int32():
    g = from_pairs(3, [[0, 1], [1, 2]], name="w")
    g.edgeLen = np.array([2**31 - 10, 5], np.int32)
    with DeviceGraph.from_csr(g) as dg:
        with pytest.raises(_lib.SPError):  # held edge + addition wraps
            dg.update("a", [0], [1], [100])
        with pytest.raises(_lib.SPError):  # two additions of one new edge wrap
            dg.update("aa", [2, 2], [0, 0], [2**31 - 1, 2**31 - 1])
        # rejected batches leave the graph as it was
        assert dg.export()["edgeLen"].tolist() == [2**31 - 10, 5]
        dg.update("a", [0], [1], [9])
        assert dg.export()["edgeLen"].tolist() == [2**31 - 1, 5]


def _pagerank_fixed_point(V, edges):
    """FP64 PageRank of the edge set, iterated to its fixed point (the oracle)."""
    off, adj, _ = _csr(V, edges)
    rev = sorted((b, a) for a, b in edges)
    roff = np.searchsorted(np.array([b for b, _ in rev], np.int64), np.arange(V + 1)).astype(np.int32)
    radj = np.array([a for _, a in rev], np.int32)
    ref, _, _ = O.pagerank(off, roff, radj, 0.0, 0.85, 300)
    return ref


def test_pagerank_dynamic_reaches_the_new_fixed_point():
    # DynPR's Batch block: ranks carried across batches (host and device arrays) end at
    # the updated graph's PageRank, like a cold start, within L1 1e-6
    import torch

    rng = np.random.default_rng(5)
    g = G.rmat(12, 8, seed=9, directed=True)
    g.edgeLen = G.hash_weights(g, 3, 1, 50, False)
    edges = _edges(g.indexofNodes, g.edgeList, g.edgeLen)
    with DeviceGraph.from_csr(g) as dg:
        pr, _, _ = dg.pagerank(beta=1e-9)
        for step, n in enumerate((16, 400, 3000)):
            t, s, d, w = _batch(rng, g.V, edges, n)
            ranks = pr if step != 1 else torch.from_numpy(pr).cuda()
            ranks, it, _ = dg.pagerank_dynamic(t, s, d, w, ranks, beta=1e-9)
            pr = ranks if step != 1 else ranks.cpu().numpy()
            edges = _apply(edges, t, s, d, w)
            assert 1 <= it <= 100
            assert np.abs(pr.astype(np.float64) - _pagerank_fixed_point(g.V, edges)).sum() < 1e-6


def test_pagerank_dynamic_warm_start_takes_fewer_iterations():
    rng = np.random.default_rng(5)
    g = G.rmat(12, 8, seed=9, directed=True)
    g.edgeLen = G.hash_weights(g, 3, 1, 50, False)
    edges = _edges(g.indexofNodes, g.edgeList, g.edgeLen)
    with DeviceGraph.from_csr(g) as dg:
        pr, _, _ = dg.pagerank()
        before = pr.copy()
        # no updates: converged ranks stay within the stop test after at most two sweeps
        _, it, diff = dg.pagerank_dynamic("", [], [], None, pr)
        assert it <= 2 and diff <= 1e-6 and np.abs(pr - before).sum() <= 2e-6
        t, s, d, w = _batch(rng, g.V, edges, 16)
        _, it_warm, _ = dg.pagerank_dynamic(t, s, d, w, pr)
        cold, it_cold, _ = dg.pagerank()
        # FP64 restatement on this graph: 14 warm against 52 cold sweeps
        assert it_warm < it_cold
        # both stop at L1 diff <= 1e-6, which bounds each one's distance to the fixed point
        # by 0.85 / 0.15 * 1e-6 in L1
        assert np.abs(pr.astype(np.float64) - cold).sum() < 2 * 5.7e-6 + 1e-7


def test_pagerank_dynamic_rejects_bad_arguments():
    g = G.rmat(8, 4, seed=2, directed=True)
    with DeviceGraph.from_csr(g) as dg:
        with pytest.raises(ValueError):
            dg.pagerank_dynamic("a", [0], [1], None, np.zeros(g.V - 1, np.float32))
        with pytest.raises(ValueError):
            dg.pagerank_dynamic("a", [0], [1], None, np.zeros(g.V, np.float64))
        with pytest.raises(_lib.SPError):
            dg.pagerank_dynamic("x", [0], [1], None, np.zeros(g.V, np.float32))
        with pytest.raises(_lib.SPError):
            dg.pagerank_dynamic("a", [0], [g.V], None, np.zeros(g.V, np.float32))


def _sym_batch(rng, V, edges, n):
    """n / 2 undirected updates, each given in both directions (kinds as in _batch)."""
    t, s, d, w = _batch(rng, V, edges, n // 2)
    return (t + t, np.concatenate([s, d]), np.concatenate([d, s]), np.concatenate([w, w]))


def test_tc_dynamic_counts_only_the_batch_on_symmetric_graphs():
    rng = np.random.default_rng(21)
    g = G.rmat(12, 16, seed=5)  # undirected
    g.edgeLen = G.hash_weights(g, 5, 1, 50, True)
    edges = _edges(g.indexofNodes, g.edgeList, g.edgeLen)
    with DeviceGraph.from_csr(g) as dg:
        count = dg.tc()
        for n in (2, 60, 800, 6000):
            t, s, d, w = _sym_batch(rng, g.V, edges, n)
            count, incremental = dg.tc_dynamic(t, s, d, w, count)
            edges = _apply(edges, t, s, d, w)
            off, adj, _ = _csr(g.V, edges)
            assert incremental
            assert count == O.tc(off, adj) == dg.tc()


def test_tc_dynamic_edge_deleted_and_added_in_one_batch():
    # deletions apply first: the edge is gone, then back, and so are its triangles
    g = G.rmat(10, 16, seed=3)
    with DeviceGraph.from_csr(g) as dg:
        before = dg.tc()
        a = int(np.argmax(np.diff(g.indexofNodes)))
        b = int(g.edgeList[g.indexofNodes[a]])
        count, incremental = dg.tc_dynamic("ddaa", [a, b, a, b], [b, a, b, a], None, before)
        assert incremental and count == before == dg.tc()
        # an added edge that is already there changes nothing either
        count, incremental = dg.tc_dynamic("aa", [a, b], [b, a], None, count)
        assert incremental and count == before


def test_tc_dynamic_counts_again_otherwise():
    rng = np.random.default_rng(22)
    for g, sym in ((G.rmat(11, 8, seed=2), False), (G.rmat(11, 8, seed=2, directed=True), True)):
        g.edgeLen = G.hash_weights(g, 2, 1, 50, g.is_symmetric())
        edges = _edges(g.indexofNodes, g.edgeList, g.edgeLen)
        with DeviceGraph.from_csr(g) as dg:
            count = dg.tc()
            t, s, d, w = (_sym_batch if sym else _batch)(rng, g.V, edges, 300)
            count, incremental = dg.tc_dynamic(t, s, d, w, count)
            edges = _apply(edges, t, s, d, w)
            off, adj, _ = _csr(g.V, edges)
            assert not incremental  # an unsymmetric batch, or a directed graph
            assert count == O.tc(off, adj)


def test_tc_dynamic_rejects_a_bad_batch_unchanged():
    g = G.rmat(9, 8, seed=4)
    with DeviceGraph.from_csr(g) as dg:
        before, E = dg.tc(), dg.E
        for t, s, d in (("ax", [0, 1], [1, 0]), ("aa", [0, g.V], [g.V, 0])):
            with pytest.raises(_lib.SPError):
                dg.tc_dynamic(t, s, d, None, before)
        assert dg.E == E and dg.tc() == before


def test_clustering_coeff_dynamic_matches_the_oracle():
    # symmetric batches: per-vertex triangle counts moved by the changed triangles only;
    # an unsymmetric batch: counted again; host and device arrays
    import torch

    rng = np.random.default_rng(23)
    g = G.rmat(12, 16, seed=7)
    edges = _edges(g.indexofNodes, g.edgeList, np.ones(g.E, np.int32))
    with DeviceGraph.from_csr(g) as dg:
        cf = dg.clustering_coeff()
        for step, (n, sym) in enumerate(((2, True), (50, True), (900, True), (4000, True), (100, False))):
            t, s, d, w = (_sym_batch if sym else _batch)(rng, g.V, edges, n)
            x = torch.from_numpy(cf).cuda() if step == 2 else cf
            incremental = dg.clustering_coeff_dynamic(t, s, d, w, x)
            cf = x.cpu().numpy() if step == 2 else x
            edges = _apply(edges, t, s, d, w)
            off, adj, _ = _csr(g.V, edges)
            assert incremental == sym
            assert np.array_equal(cf, O.lcc(off, adj)), step


def test_degree_dynamic_gives_the_new_out_degrees():
    rng = np.random.default_rng(24)
    g = G.rmat(11, 8, seed=3, directed=True)
    edges = _edges(g.indexofNodes, g.edgeList, np.ones(g.E, np.int32))
    with DeviceGraph.from_csr(g, with_weights=False) as dg:
        for n in (1, 300):
            t, s, d, w = _batch(rng, g.V, edges, n)
            deg = dg.degree_dynamic(t, s, d, None)
            edges = _apply(edges, t, s, d, w)
            off, _, _ = _csr(g.V, edges)
            assert np.array_equal(deg, np.diff(off))


def test_bc_dynamic_matches_the_oracle_on_the_new_graph():
    rng = np.random.default_rng(25)
    g = G.rmat(11, 8, seed=6)
    edges = _edges(g.indexofNodes, g.edgeList, np.ones(g.E, np.int32))
    srcs = G.pick_sources(g, 40, seed=3)
    with DeviceGraph.from_csr(g, with_weights=False) as dg:
        for n, sym in ((2, True), (400, True), (100, False)):
            t, s, d, w = (_sym_batch if sym else _batch)(rng, g.V, edges, n)
            bc = dg.bc_dynamic(t, s, d, None, srcs).astype(np.float64)
            edges = _apply(edges, t, s, d, w)
            off, adj, _ = _csr(g.V, edges)
            ref = O.bc(off, adj, srcs)
            assert np.all(np.abs(bc - ref) <= 1e-5 * np.abs(ref) + 1e-9 * max(1.0, ref.max()))
        # a seed outside the graph is rejected before the batch is applied
        E = dg.E
        a = next(v for v in range(1, g.V) if (0, v) not in edges)
        with pytest.raises(_lib.SPError):
            dg.bc_dynamic("aa", [0, a], [a, 0], None, [0, g.V])
        dg._refresh_size()
        assert dg.E == E


def test_dsl_dynamic_programs_run_batch_by_batch():
    # DynTC, DynPR, DynSSSP, DynCF, DynDegree and DynBC (starplat_b200.algorithms) over 30
    # update records in batches of 8, each undirected update given in both directions
    # next to each other; results against the oracle on the edge set replayed batch by batch
    from starplat_b200 import algorithms as A

    def fresh():
        g = G.rmat(10, 8, seed=8)
        g.edgeLen = G.hash_weights(g, 8, 1, 40, True)
        return g

    rng = np.random.default_rng(26)
    g0 = fresh()
    edges = _edges(g0.indexofNodes, g0.edgeList, g0.edgeLen)
    t, s, d, w = _batch(rng, g0.V, edges, 15)
    updates = []
    for i in range(len(t)):
        updates += [(t[i], int(s[i]), int(d[i]), int(w[i])), (t[i], int(d[i]), int(s[i]), int(w[i]))]
    for k in range(0, len(updates), 8):
        chunk = updates[k:k + 8]
        edges = _apply(edges, "".join(u[0] for u in chunk), [u[1] for u in chunk], [u[2] for u in chunk],
                       [u[3] for u in chunk])
    off, adj, ww = _csr(g0.V, edges)
    V = g0.V

    assert A.DynTC(fresh(), updates, 8) == O.tc(off, adj)
    # the programs leave g and its cached mirror as they were before the batches
    g1 = fresh()
    before = A.Compute_TC(g1)
    assert A.DynTC(g1, updates, 8) == O.tc(off, adj)
    assert A.Compute_TC(g1) == before == O.tc(g1.indexofNodes, g1.edgeList)
    A.invalidate(g1)
    pr = np.zeros(V, np.float32)
    A.DynPR(fresh(), 1e-9, 0.85, 100, pr, updates, 8)
    assert np.abs(pr.astype(np.float64) - _pagerank_fixed_point(V, edges)).sum() < 1e-6
    src = int(G.pick_sources(g0, 1, seed=1)[0])
    dist = np.zeros(V, np.int32)
    A.DynSSSP(fresh(), dist, None, None, updates, 8, src)
    assert np.array_equal(dist, O.sssp(off, adj, ww, src))
    cf = np.zeros(V, np.int32)
    A.DynCF(fresh(), updates, cf, 8)
    assert np.array_equal(cf, O.lcc(off, adj))
    deg = np.zeros(V, np.int32)
    A.DynDegree(fresh(), updates, deg, 8)
    assert np.array_equal(deg, np.diff(off))
    seeds = set(int(x) for x in G.pick_sources(g0, 20, seed=2))
    bc = np.zeros(V, np.float32)
    A.DynBC(fresh(), bc, seeds, updates, 8)
    ref = O.bc(off, adj, np.array(sorted(seeds), np.int32))
    assert np.all(np.abs(bc.astype(np.float64) - ref) <= 1e-5 * np.abs(ref) + 1e-9 * max(1.0, ref.max()))
    with pytest.raises(ValueError):
        A.DynSSSP(fresh(), dist, np.zeros(V, np.int32), None, updates, 8, src)
