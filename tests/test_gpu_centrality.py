"""GPU parity for the algorithms built on the same kernels: per-vertex triangle counts
(staticClusteringCoeff), out-degrees (Degree) and closeness (Compute_CC weighted,
Compute_CC_Unweighted). Integer outputs are bit-exact against the oracle; closeness is
1.0 / an exact integer sum, so it is bit-exact too."""
import numpy as np
import pytest

from oracle import oracle as O
from starplat_b200 import _lib
from starplat_b200 import generators as G
from starplat_b200.algorithms import (Compute_CC, Compute_CC_Unweighted, Degree, device_graph,
                                      staticClusteringCoeff)

from graphs import directed_zoo, from_pairs, star, undirected_zoo

pytestmark = pytest.mark.gpu


def _lcc_graphs():
    # V <= 65536 (shared-memory bitmap) and above (hash tables, heavy anchors), directed
    # (literal formula) and undirected (oriented), hubs
    return (directed_zoo()[:3] + undirected_zoo()[:5] +
            [G.rmat(17, 16, seed=4), G.rmat(14, 16, seed=6, directed=True), star(3000, directed_in=False)])


@pytest.mark.parametrize("variant", [_lib.SP_TC_TUNED, _lib.SP_TC_PLAIN])
def test_clustering_coeff_matches_oracle(variant):
    for g in _lcc_graphs():
        out = device_graph(g).clustering_coeff(variant=variant)
        ref = O.lcc(g.indexofNodes, g.edgeList)
        assert np.array_equal(out, ref), (g.name, int((out != ref).sum()))
        if variant == _lib.SP_TC_TUNED and g.is_symmetric():
            assert int(out.astype(np.int64).sum()) == 3 * device_graph(g).tc()


def test_clustering_coeff_large_anchor_set():
    # a directed graph whose vertex 5000 has 5,500 higher neighbours (its S, above the
    # 4,096 counted in shared memory, so its hits go straight to global counts) and
    # 5,000 lower ones, each with edges into S; plus small anchors counted in shared memory
    pairs = [[5000, u] for u in range(5000)] + [[5000, w] for w in range(5001, 10501)]
    pairs += [[u, 5001 + (u * 7) % 5500] for u in range(5000)]
    pairs += [[u, 5001 + (u * 13 + 1) % 5500] for u in range(0, 5000, 3)]
    pairs += [[u, u + 1] for u in range(10501, 11999)] + [[u, u + 2] for u in range(10501, 11998)]
    g = from_pairs(12000, np.array(pairs, np.int32), name="big_anchor")
    for variant in (_lib.SP_TC_TUNED, _lib.SP_TC_PLAIN):
        out = device_graph(g).clustering_coeff(variant=variant)
        assert np.array_equal(out, O.lcc(g.indexofNodes, g.edgeList)), variant
    assert O.lcc(g.indexofNodes, g.edgeList)[5000] > 0


def test_clustering_coeff_entry_point_twice_and_device_output():
    import torch

    g = G.rmat(12, 16, seed=2)
    cf = np.full(g.V, -7, np.int32)  # overwritten, not accumulated
    staticClusteringCoeff(g, cf)
    staticClusteringCoeff(g, cf)
    assert np.array_equal(cf, O.lcc(g.indexofNodes, g.edgeList))
    out = torch.empty(g.V, dtype=torch.int32, device="cuda")
    device_graph(g).clustering_coeff(out=out)
    assert np.array_equal(out.cpu().numpy(), cf)


def test_degree():
    for g in directed_zoo()[:2] + undirected_zoo()[:2] + [from_pairs(5, [[0, 1], [0, 2], [3, 1]], name="tiny")]:
        deg = np.empty(g.V, np.int32)
        Degree(g, deg)
        assert np.array_equal(deg, O.degree(g.indexofNodes))


def _weighted(g, lo, hi, seed=3):
    g.edgeLen = G.hash_weights(g, seed, lo, hi, g.is_symmetric())
    return g


def test_closeness_weighted_matches_oracle():
    cases = [_weighted(directed_zoo()[0], 1, 100), _weighted(undirected_zoo()[1], 1, 1000),
             _weighted(G.grid(30, 40), 1, 1000), _weighted(G.rmat(13, 8, seed=2, directed=True), 1, 100)]
    for g in cases:
        srcs = G.pick_sources(g, 9, seed=5)
        cc = np.empty(g.V, np.float32)
        Compute_CC(g, cc, set(int(s) for s in srcs))
        ref = O.closeness(g.indexofNodes, g.edgeList, g.edgeLen, np.sort(srcs))
        assert np.array_equal(cc, ref), g.name
        assert np.count_nonzero(cc) <= len(srcs)


def test_closeness_unweighted_matches_oracle():
    # more than one 64-source pass, and directed / undirected graphs
    for g in [directed_zoo()[1], undirected_zoo()[0], G.grid(20, 25), G.rmat(12, 16, seed=8)]:
        srcs = G.pick_sources(g, min(g.V, 150), seed=7)
        cc = np.empty(g.V, np.float32)
        Compute_CC_Unweighted(g, cc, set(int(s) for s in srcs))
        ref = O.closeness_unweighted(g.indexofNodes, g.edgeList, np.sort(srcs))
        assert np.array_equal(cc, ref), g.name


def test_closeness_edge_cases():
    # an isolated source (sum 0 -> +inf, as 1.0 / 0 gives in the generated C++), a
    # source set with every vertex, an empty source set, and bad sources
    g = from_pairs(5, [[0, 1], [1, 2], [2, 0]], name="tri_iso")
    g.edgeLen = np.array([2, 3, 4], np.int32)
    cc = np.empty(g.V, np.float32)
    Compute_CC(g, cc, {4})
    assert np.isinf(cc[4]) and cc[4] > 0 and np.count_nonzero(cc[:4]) == 0
    Compute_CC(g, cc, set(range(g.V)))
    assert np.array_equal(cc, O.closeness(g.indexofNodes, g.edgeList, g.edgeLen, np.arange(g.V)))
    Compute_CC_Unweighted(g, cc, set(range(g.V)))
    assert np.array_equal(cc, O.closeness_unweighted(g.indexofNodes, g.edgeList, np.arange(g.V)))
    Compute_CC(g, cc, set())
    assert not cc.any()
    dg = device_graph(g)
    with pytest.raises(_lib.SPError):
        dg.closeness(np.array([1, 1], np.int32))
    with pytest.raises(_lib.SPError):
        dg.closeness_unweighted(np.array([5], np.int32))


@pytest.mark.parametrize("nparts", [1, 2, 3, 8])
def test_triangle_parts_sum_to_the_whole(nparts):
    # sp_tc_part / sp_clustering_coeff_part: every triangle falls in exactly one part of
    # the anchor order, so the parts add up to the oracle's figures exactly
    for g in _lcc_graphs():
        dg = device_graph(g)
        tcs = [dg.tc_part(r, nparts) for r in range(nparts)]
        cfs = [dg.clustering_coeff_part(r, nparts).astype(np.int64) for r in range(nparts)]
        ref_tc = O.tc(g.indexofNodes, g.edgeList)
        assert sum(tcs) == ref_tc, g.name
        assert np.array_equal(np.sum(cfs, axis=0), O.lcc(g.indexofNodes, g.edgeList)), g.name
    if nparts > 1:  # R-MAT 17: every part holds a share
        g = G.rmat(17, 16, seed=4)
        parts = [device_graph(g).tc_part(r, nparts) for r in range(nparts)]
        assert all(0 < p < sum(parts) for p in parts)


def test_triangle_parts_under_every_small_graph_kernel():
    from starplat_b200.device import DeviceGraph

    g = G.rmat(12, 16, seed=9)
    ref_tc = O.tc(g.indexofNodes, g.edgeList)
    ref_cf = O.lcc(g.indexofNodes, g.edgeList)
    with DeviceGraph.from_csr(g) as dg:
        for warps in (0, 2, 4, 8, 16):  # 0: the per-warp bitmap kernel
            dg.tune_set("tc.cta_warps", warps)
            assert sum(dg.tc_part(r, 3) for r in range(3)) == ref_tc, warps
        cf = sum(dg.clustering_coeff_part(r, 3).astype(np.int64) for r in range(3))
        assert np.array_equal(cf, ref_cf)


def test_triangle_parts_beyond_the_vertex_count_and_bad_parts():
    g = from_pairs(3, [[0, 1], [1, 2], [0, 2]], symmetrize=True)
    dg = device_graph(g)
    parts = [dg.tc_part(r, 5) for r in range(5)]
    assert sum(parts) == 1 and parts[3] == 0 and parts[4] == 0
    cf = sum(dg.clustering_coeff_part(r, 5).astype(np.int64) for r in range(5))
    assert np.array_equal(cf, [1, 1, 1])
    for part, nparts in ((2, 2), (0, 0), (-1, 3)):
        with pytest.raises(_lib.SPError):
            dg.tc_part(part, nparts)
        with pytest.raises(_lib.SPError):
            dg.clustering_coeff_part(part, nparts)
