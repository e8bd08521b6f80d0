"""GPU parity: SSSP distances are bit-exact against the oracle (Dijkstra, or
queue Bellman-Ford when weights are negative), for every schedule (delta) and
both variants."""
import numpy as np
import pytest

from oracle import oracle as O
from starplat_b200 import _lib
from starplat_b200 import generators as G
from starplat_b200.algorithms import Compute_SSSP, device_graph
from starplat_b200.device import DeviceGraph

from graphs import directed_zoo, from_pairs, undirected_zoo

pytestmark = pytest.mark.gpu
INT_MAX = np.iinfo(np.int32).max


def weighted(g, lo, hi, seed=3, symmetric=None):
    if symmetric is None:
        symmetric = g.is_symmetric()
    g.edgeLen = G.hash_weights(g, seed, lo, hi, symmetric)
    return g


def check(g, src, **kw):
    dg = device_graph(g)
    out, rounds = dg.sssp(src, **kw)
    ref = O.sssp(g.indexofNodes, g.edgeList, g.edgeLen, src)
    assert np.array_equal(out, ref), (g.name, src, int((out != ref).sum()))
    return rounds


@pytest.mark.parametrize("gi", range(4))
def test_sssp_directed(gi):
    g = weighted(directed_zoo()[gi], 1, 100)
    for src in G.pick_sources(g, 3, seed=gi):
        check(g, int(src))


@pytest.mark.parametrize("gi", range(8))
def test_sssp_undirected(gi):
    g = weighted(undirected_zoo()[gi], 1, 1000)
    check(g, 0)
    check(g, g.V - 1)


@pytest.mark.parametrize("delta", [1, 3, 50, 1000, 10**6, 2**31 - 1])
def test_sssp_any_delta_is_exact(delta):
    g = weighted(G.rmat(12, 16, seed=5, directed=True), 1, 100)
    check(g, int(G.pick_sources(g, 1, seed=1)[0]), delta=delta)
    gg = weighted(G.grid(40, 50), 1, 1000)
    check(gg, 0, delta=delta)


@pytest.mark.parametrize("hub_deg,chunk", [(2048, 256), (128, 64), (1, 1), (3, 1000), (0, 0)])
def test_sssp_hub_splitting_knobs_keep_distances_exact(hub_deg, chunk):
    from graphs import star

    for g in (weighted(G.rmat(13, 16, seed=8, directed=True), 1, 100), weighted(star(5000, directed_in=False), 1, 9),
              weighted(G.grid(40, 50), 1, 1000)):
        dg = device_graph(g)
        dg.tune_set("sssp.hub_deg", hub_deg)
        dg.tune_set("sssp.hub_chunk", chunk)
        for src in (0, g.V // 2):
            check(g, src)
        dg.tune_set("sssp.hub_deg", 0)
        dg.tune_set("sssp.hub_chunk", 0)


@pytest.mark.parametrize("local", [0, 1, 2, 64, 65536])
def test_sssp_warp_cascade_budget_keeps_distances_exact(local):
    # the cascade ring (256 entries per warp) overflows into the stamped queue on the
    # star and R-MAT; the grid cascades for many hops; budget 1 stops after one step
    from graphs import star

    cases = [(weighted(G.rmat(13, 16, seed=8, directed=True), 1, 100), None),
             (weighted(star(5000, directed_in=False), 1, 9), None),
             (weighted(G.grid(64, 80), 1, 1000), None), (weighted(G.grid(64, 80), 1, 1000), 2**31 - 1),
             (weighted(G.grid(64, 80), 1, 1000), 1)]
    for g, delta in cases:
        dg = device_graph(g)
        dg.tune_set("sssp.local", local)
        assert dg.tune_get("sssp.local") == local
        for src in (0, g.V // 2):
            check(g, src, **({} if delta is None else {"delta": delta}))
        dg.tune_set("sssp.hub_deg", 3)  # hubs popped from a ring go to the hub list
        check(g, g.V - 1, **({} if delta is None else {"delta": delta}))
        dg.tune_set("sssp.hub_deg", 0)
        dg.tune_set("sssp.local", 64)


@pytest.mark.parametrize("flt", [0, 1])
def test_sssp_atomic_filter_knob_keeps_distances_exact(flt):
    # 0: every candidate goes straight to atomicMin (no dist load first); also with
    # negative weights (Bellman-Ford mode) and in the batched multi-source form
    from graphs import star

    cases = [weighted(G.rmat(13, 16, seed=8, directed=True), 1, 100), weighted(star(5000, directed_in=False), 1, 9),
             weighted(G.grid(64, 80), 1, 1000), weighted(undirected_zoo()[3], 1, 1000)]
    for g in cases:
        dg = device_graph(g)
        dg.tune_set("sssp.filter", flt)
        assert dg.tune_get("sssp.filter") == flt
        for src in (0, g.V // 2):
            check(g, src)
        check(g, g.V - 1, delta=2**31 - 1)
        srcs = np.array([0, g.V // 3, g.V - 1], np.int32)
        rows = dg.sssp_batch(srcs)
        for k, s in enumerate(srcs):
            assert np.array_equal(rows[k], O.sssp(g.indexofNodes, g.edgeList, g.edgeLen, int(s))), (g.name, int(s))
        dg.tune_set("sssp.filter", -1)
    rng = np.random.default_rng(4)
    n = 300
    pairs = np.array([(i, j) for i in range(n) for j in rng.choice(n, 4) if i < j], np.int32)
    gn = from_pairs(n, pairs, name="dag_filter")
    gn.edgeLen = rng.integers(-40, 100, gn.E).astype(np.int32)
    dn = device_graph(gn)
    dn.tune_set("sssp.filter", flt)
    check(gn, 0)


def test_sssp_cascade_with_negative_weights():
    rng = np.random.default_rng(2)
    n = 400
    pairs = np.array([(i, j) for i in range(n) for j in rng.choice(n, 5) if i < j], np.int32)
    g = from_pairs(n, pairs, name="dag2")
    g.edgeLen = rng.integers(-50, 100, g.E).astype(np.int32)
    dg = device_graph(g)
    for local in (0, 4, 1000):
        dg.tune_set("sssp.local", local)
        check(g, 0)
    c = from_pairs(3, [[0, 1], [1, 2], [2, 0]], name="negcycle2")
    c.edgeLen = np.array([1, -5, 1], np.int32)
    dc = device_graph(c)
    dc.tune_set("sssp.local", 1000)
    with pytest.raises(_lib.SPError) as ei:
        dc.sssp(0)
    assert ei.value.status == -6


def test_sssp_tuned_delta_knob():
    g = weighted(G.grid(30, 30), 1, 1000)
    dg = device_graph(g)
    for d in (0, 17, 5000):
        dg.tune_set("sssp.delta", d)
        assert dg.tune_get("sssp.delta") == d
        check(g, 5)
    dg.tune_set("sssp.delta", 0)


def test_sssp_plain_variant():
    for g in (weighted(G.rmat(11, 8, seed=3, directed=True), 1, 100), weighted(G.grid(20, 20), 1, 1000)):
        check(g, 0, variant=_lib.SP_SSSP_PLAIN)


def test_sssp_unreachable_and_zero_weights():
    g = from_pairs(7, [[0, 1], [1, 2], [2, 3], [4, 5]], name="chain")
    g.edgeLen = np.zeros(g.E, np.int32)
    out, _ = device_graph(g).sssp(0)
    assert out.tolist() == [0, 0, 0, 0, INT_MAX, INT_MAX, INT_MAX]
    out, _ = device_graph(g).sssp(6)  # isolated source
    assert out.tolist() == [INT_MAX] * 6 + [0]


def test_sssp_negative_weights_and_cycle():
    # a DAG with negative weights: exact via the queue Bellman-Ford oracle
    rng = np.random.default_rng(1)
    n = 300
    pairs = np.array([(i, j) for i in range(n) for j in rng.choice(n, 4) if i < j], np.int32)
    g = from_pairs(n, pairs, name="dag")
    g.edgeLen = rng.integers(-50, 100, g.E).astype(np.int32)
    check(g, 0)
    # a reachable negative cycle has no fixed point
    c = from_pairs(3, [[0, 1], [1, 2], [2, 0]], name="negcycle")
    c.edgeLen = np.array([1, -5, 1], np.int32)
    with pytest.raises(_lib.SPError) as ei:
        device_graph(c).sssp(0)
    assert ei.value.status == -6


def test_sssp_large_weights_no_overflow():
    # 2^30 + (2^30 - 1) = INT_MAX: a sum reaching INT_MAX is never stored (the
    # reference's `dist[nbr] > dist_new` test fails there too), so 2 and 3 stay unreachable
    g = from_pairs(4, [[0, 1], [1, 2], [2, 3]], name="big")
    g.edgeLen = np.array([2**30, 2**30 - 1, 2**30], np.int32)
    out, _ = device_graph(g).sssp(0)
    assert out.tolist() == [0, 2**30, INT_MAX, INT_MAX]
    assert np.array_equal(out, O.sssp(g.indexofNodes, g.edgeList, g.edgeLen, 0))


def test_sssp_entry_point_and_device_weights():
    import torch

    g = weighted(G.rmat(11, 16, seed=8, directed=True), 1, 100)
    w = g.edgeLen.copy()
    g.edgeLen = None  # weights passed per call, as the generated signature does
    dist = np.zeros(g.V, np.int32)
    Compute_SSSP(g, dist, w, 3)
    assert np.array_equal(dist, O.sssp(g.indexofNodes, g.edgeList, w, 3))
    t = [torch.from_numpy(a).cuda() for a in (g.indexofNodes, g.edgeList)]
    with DeviceGraph(t[0], t[1]) as dg:
        out = torch.empty(g.V, dtype=torch.int32, device="cuda")
        dg.sssp(3, weight=torch.from_numpy(w).cuda(), out=out)
        assert np.array_equal(out.cpu().numpy(), dist)


def test_sssp_bad_source():
    g = weighted(G.grid(5, 5), 1, 10)
    with pytest.raises(_lib.SPError):
        device_graph(g).sssp(25)


@pytest.mark.parametrize("case", ["rmat17", "rmat20", "grid1024"])
def test_sssp_at_scale(case):
    # sizes where phases of different CTAs overlap in time (the small graphs above
    # finish each phase before a second CTA starts)
    if case.startswith("rmat"):
        g = weighted(G.rmat(int(case[4:]), 16, seed=1, directed=True), 1, 100, seed=23)
        src = int(G.pick_sources(g, 1, seed=23)[0])
    else:
        g = weighted(G.grid(1024, 1024), 1, 1000, seed=4096)
        src = 123457
    check(g, src)
    check(g, src, variant=_lib.SP_SSSP_PLAIN)


@pytest.mark.parametrize("batch", [1, 3, 16, 64])
def test_sssp_batch_one_launch_per_batch_is_exact(batch):
    # many sources, each on its own CTA group of one cooperative launch per batch:
    # every row equals the single-source distances, for any batch size
    graphs = [weighted(G.rmat(12, 16, seed=5, directed=True), 1, 100), weighted(G.grid(40, 50), 1, 1000),
              weighted(G.rmat(11, 8, seed=3), 1, 50)]
    for g in graphs:
        srcs = G.pick_sources(g, 21, seed=batch)
        with DeviceGraph.from_csr(g) as dg:
            dg.tune_set("sssp.batch", batch)
            rows = dg.sssp_batch(srcs)
            assert dg.tune_get("sssp.last_batch") == min(batch, len(srcs))
        for k, s in enumerate(srcs):
            ref = O.sssp(g.indexofNodes, g.edgeList, g.edgeLen, int(s))
            assert np.array_equal(rows[k], ref), (g.name, batch, k)


def test_sssp_batch_device_rows_negative_weights_and_errors():
    import torch

    # negative weights without negative cycles: every group runs queue Bellman-Ford
    g = from_pairs(5, [[0, 1], [1, 2], [0, 2], [2, 3], [3, 4], [1, 4]], name="neg")
    g.edgeLen = np.array([4, -2, 3, 1, 2, 7], np.int32)
    with DeviceGraph.from_csr(g) as dg:
        rows = dg.sssp_batch(np.array([0, 1, 2, 4], np.int32))
        for k, s in enumerate([0, 1, 2, 4]):
            assert np.array_equal(rows[k], O.sssp(g.indexofNodes, g.edgeList, g.edgeLen, s))
    g = weighted(G.rmat(13, 8, seed=2, directed=True), 1, 100)
    srcs = G.pick_sources(g, 40, seed=2)
    with DeviceGraph.from_csr(g) as dg:
        out = torch.empty((len(srcs), g.V), dtype=torch.int32, device="cuda")
        dg.sssp_batch(torch.from_numpy(srcs).cuda(), out=out)
        got = out.cpu().numpy()
        for k in (0, 17, 39):
            assert np.array_equal(got[k], O.sssp(g.indexofNodes, g.edgeList, g.edgeLen, int(srcs[k])))
        with pytest.raises(_lib.SPError):
            dg.sssp_batch(np.array([0, g.V], np.int32))
        with pytest.raises(_lib.SPError):
            dg.tune_set("sssp.batch", 5000)
