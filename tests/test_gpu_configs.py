"""GPU parity at the benchmark configurations themselves, each against the oracle
(never against another GPU form):

* PageRank, directed R-MAT 22 ef16 (the headline): L1 < 1e-6 against FP64 PageRank
  at the same iteration count (semantics: staticDSLCodes/PageRankDSLV3:1-25);
* SSSP, directed R-MAT 23 ef16 with weights U[1,100], and the 4096 x 4096 grid with
  symmetric weights U[1,1000]: distances bit-exact (sssp_dslV3:1-26);
* BC, undirected R-MAT 20 ef16, the first 64 of the benchmark's 256 sources (one full
  source batch): BFS levels and path counts bit-exact for a few sources, BC within
  1e-5 relative of FP64 Brandes (bc_dslV2:1-21); and the 1000 Erdos-Renyi graphs run
  as one batch, every 20th graph checked;
* Louvain, the 1,048,576-vertex planted partition: the returned partition has the
  returned modularity, at least that of the reference's own CUDA Louvain on this graph
  (a committed fixture) minus 1e-3.

Each graph is built by the same seeded generator call as bench.py."""
import numpy as np
import pytest

from oracle import oracle as O
from starplat_b200 import generators as G
from starplat_b200.device import DeviceGraph

pytestmark = pytest.mark.gpu
INT_MAX = np.iinfo(np.int32).max


def bc_within(got, ref):
    got = np.asarray(got, np.float64)
    bar = 1e-5 * np.abs(ref) + 1e-9 * max(1.0, float(ref.max(initial=0.0)))
    return bool(np.all(np.abs(got - ref) <= bar)), float((np.abs(got - ref) / bar).max(initial=0.0))


def test_pagerank_rmat22_against_fp64():
    g = G.rmat(22, 16, seed=1, directed=True)
    with DeviceGraph.from_csr(g, with_weights=False) as dg:
        pr, it, diff = dg.pagerank(1e-6, 0.85, 100)
    assert 1 < it < 100 and diff <= 1e-6
    exact, _, _ = O.pagerank(g.indexofNodes, g.rev_indexofNodes, g.srcList, 0.0, 0.85, it, nthreads=O.num_threads())
    l1 = float(np.abs(pr.astype(np.float64) - exact).sum())
    assert l1 < 1e-6, l1
    # the stop test agrees with the FP64 run's own (same iteration, or one apart inside
    # the FP32 quantisation window of the last rank changes)
    _, it64, _ = O.pagerank(g.indexofNodes, g.rev_indexofNodes, g.srcList, 1e-6, 0.85, 100,
                            nthreads=O.num_threads())
    assert abs(it64 - it) <= 1, (it, it64)


def test_sssp_rmat23_bit_exact():
    g = G.rmat(23, 16, seed=1, directed=True)
    g.edgeLen = G.hash_weights(g, 23, 1, 100, False)
    src = int(G.pick_sources(g, 1, seed=23)[0])
    with DeviceGraph.from_csr(g) as dg:
        dist, _ = dg.sssp(src)
    ref, _ = O.sssp_omp(g.indexofNodes, g.edgeList, g.edgeLen, src, nthreads=O.num_threads())
    assert np.array_equal(dist, ref), int((dist != ref).sum())
    assert (dist < INT_MAX).sum() > g.V // 4


def test_sssp_grid4096_bit_exact():
    g = G.grid(4096, 4096)
    g.edgeLen = G.hash_weights(g, 4096, 1, 1000, True)
    src = int(np.random.default_rng(4096).integers(0, g.V))
    with DeviceGraph.from_csr(g) as dg:
        dist, _ = dg.sssp(src)
    ref = O.sssp(g.indexofNodes, g.edgeList, g.edgeLen, src)
    assert np.array_equal(dist, ref), int((dist != ref).sum())


def test_bc_rmat20_one_full_batch():
    g = G.rmat(20, 16, seed=1)
    srcs = G.pick_sources(g, 256, seed=20)[:64]
    with DeviceGraph.from_csr(g, with_weights=False) as dg:
        bc = dg.bc(srcs)
        lv, sg = dg.bfs_sigma(srcs[:4])
    for k in range(4):
        rl, rs, _ = O.bfs_sigma(g.indexofNodes, g.edgeList, int(srcs[k]))
        assert np.array_equal(lv[k], rl) and np.array_equal(sg[k], rs), k
    ref = O.bc(g.indexofNodes, g.edgeList, srcs, nthreads=O.num_threads())
    ok, worst = bc_within(bc, ref)
    assert ok, worst


def test_bc_er1000_batched():
    gs = G.er_batch(1000, 1000, 50000, 8, 32, seed=11)
    voff = np.zeros(len(gs) + 1, np.int64)
    eoff = np.zeros(len(gs) + 1, np.int64)
    for k, g in enumerate(gs):
        voff[k + 1] = voff[k] + g.V
        eoff[k + 1] = eoff[k] + g.E
    V, E = int(voff[-1]), int(eoff[-1])
    off = np.empty(V + 1, np.int32)
    adj = np.empty(E, np.int32)
    srcs, soff = [], [0]
    for k, g in enumerate(gs):
        off[voff[k]:voff[k + 1]] = g.indexofNodes[:-1] + eoff[k]
        adj[eoff[k]:eoff[k + 1]] = g.edgeList + voff[k]
        s = G.pick_sources(g, 16, seed=k)
        srcs.append(s + voff[k])
        soff.append(soff[-1] + len(s))
    off[V] = E
    srcs = np.concatenate(srcs).astype(np.int32)
    soff = np.array(soff, np.int32)
    voff32 = voff.astype(np.int32)
    with DeviceGraph(off, adj, None, off, adj) as dg:
        bc = dg.bc_graphs(voff32, soff, srcs)
    for k in range(0, len(gs), 20):
        ref = O.bc(gs[k].indexofNodes, gs[k].edgeList, srcs[soff[k]:soff[k + 1]] - voff32[k],
                   nthreads=O.num_threads())
        ok, worst = bc_within(bc[voff32[k]:voff32[k + 1]], ref)
        assert ok, (k, worst)


def test_louvain_sbm1m_against_the_reference_louvain():
    # the reference's CUDA Louvain reaches the committed fixture's modularity on this
    # graph; this library's partition must reach at least that minus 1e-3, and have the
    # modularity it returns
    import json
    import os

    g = G.sbm(1 << 20, 256, exponent=2.0, avg_degree=32, p_in=0.8, seed=1)
    with DeviceGraph.from_csr(g, with_weights=False) as dg:
        q, comm, _ = dg.louvain(None, 1e-4)
    assert abs(O.modularity(g.indexofNodes, g.edgeList, comm) - q) < 1e-9
    fx = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_gpu", "louvain.json")
    ref = json.load(open(fx))["sbm1m"]["reference_q"]
    assert q >= ref - 1e-3, (q, ref)
