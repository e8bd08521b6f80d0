"""GPU parity: Brandes BC within 1e-5 relative of the FP64 oracle; BFS levels and
path counts (sigma) bit-exact."""
import numpy as np
import pytest

from oracle import oracle as O
from starplat_b200 import _lib
from starplat_b200 import generators as G
from starplat_b200.algorithms import Compute_BC, device_graph
from starplat_b200.device import DeviceGraph

from graphs import clique, directed_zoo, from_pairs, path, star, undirected_zoo

pytestmark = pytest.mark.gpu


def assert_bc_close(out, ref, name=""):
    out = out.astype(np.float64)
    scale = max(1.0, float(np.abs(ref).max()))
    err = np.abs(out - ref)
    # relative error 1e-5 per vertex, with an absolute floor for values near zero
    bad = err > 1e-5 * np.abs(ref) + 1e-9 * scale
    assert not bad.any(), (name, int(bad.sum()), float((err / np.maximum(np.abs(ref), 1e-30))[bad].max()))


@pytest.mark.parametrize("gi", range(8))
def test_bc_undirected(gi):
    g = undirected_zoo()[gi]
    srcs = G.pick_sources(g, min(100, g.V), seed=gi, min_out_degree=0)
    out = device_graph(g).bc(srcs)
    assert_bc_close(out, O.bc(g.indexofNodes, g.edgeList, srcs), g.name)


@pytest.mark.parametrize("gi", range(4))
def test_bc_directed(gi):
    g = directed_zoo()[gi]
    srcs = G.pick_sources(g, min(70, g.V), seed=gi, min_out_degree=0)
    out = device_graph(g).bc(srcs)
    assert_bc_close(out, O.bc(g.indexofNodes, g.edgeList, srcs), g.name)


@pytest.mark.parametrize("batch", [1, 7, 32, 33, 64])
def test_bc_batch_knob(batch):
    g = G.rmat(11, 16, seed=4)
    srcs = G.pick_sources(g, 150, seed=2)
    dg = device_graph(g)
    dg.tune_set("bc.batch", batch)
    out = dg.bc(srcs)
    dg.tune_set("bc.batch", 0)
    assert_bc_close(out, O.bc(g.indexofNodes, g.edgeList, srcs))


@pytest.mark.parametrize("hub_deg,chunk", [(4096, 256), (64, 64), (1, 1), (1, 7), (16, 1000)])
def test_bc_entry_splitting_knobs(hub_deg, chunk):
    # how level-list entries are cut into shared pieces changes the work split, not the
    # result: BC within the tolerance, BFS levels and sigma exact
    for g in (G.rmat(12, 16, seed=4), star(300, directed_in=False), G.grid(9, 11)):
        srcs = G.pick_sources(g, 70, seed=1, min_out_degree=0)
        dg = device_graph(g)
        dg.tune_set("bc.hub_deg", hub_deg)
        dg.tune_set("bc.hub_chunk", chunk)
        assert (dg.tune_get("bc.hub_deg"), dg.tune_get("bc.hub_chunk")) == (hub_deg, chunk)
        out = dg.bc(srcs)
        lvl, sig = dg.bfs_sigma(srcs[:64])
        dg.tune_set("bc.hub_deg", 0)
        dg.tune_set("bc.hub_chunk", 0)
        assert_bc_close(out, O.bc(g.indexofNodes, g.edgeList, srcs), g.name)
        for k, s in enumerate(srcs[:64]):
            rl, rs, _ = O.bfs_sigma(g.indexofNodes, g.edgeList, int(s))
            assert np.array_equal(lvl[k], rl) and np.array_equal(sig[k], rs)


def test_bc_all_sources_small_graphs():
    # the reference driver passes every vertex as a source (bc_dslV2main.cpp:50-53)
    for g in (clique(10), path(40), star(50, directed_in=False), G.grid(7, 9)):
        srcs = np.arange(g.V, dtype=np.int32)
        out = device_graph(g).bc(srcs)
        assert_bc_close(out, O.bc(g.indexofNodes, g.edgeList, srcs), g.name)


def test_bc_plain_variant():
    g = G.rmat(10, 8, seed=3)
    srcs = G.pick_sources(g, 20, seed=1)
    out = device_graph(g).bc(srcs, variant=_lib.SP_BC_PLAIN)
    assert_bc_close(out, O.bc(g.indexofNodes, g.edgeList, srcs))


def test_bc_entry_point_and_errors():
    g = G.rmat(10, 8, seed=9)
    BC = np.zeros(g.V, np.float32)
    Compute_BC(g, BC, {3, 1, 4, 15, 92})
    assert_bc_close(BC, O.bc(g.indexofNodes, g.edgeList, np.array([1, 3, 4, 15, 92], np.int32)))
    with pytest.raises(_lib.SPError):
        device_graph(g).bc(np.array([1, 1], np.int32))
    with pytest.raises(_lib.SPError):
        device_graph(g).bc(np.array([g.V], np.int32))
    assert not device_graph(g).bc(np.zeros(0, np.int32)).any()


def test_bfs_levels_and_sigma_bit_exact():
    for g in (G.rmat(12, 16, seed=6), G.rmat(11, 8, seed=2, directed=True), G.grid(12, 15)):
        srcs = G.pick_sources(g, 64, seed=5)
        lvl, sig = device_graph(g).bfs_sigma(srcs)
        for k, s in enumerate(srcs):
            rl, rs, _ = O.bfs_sigma(g.indexofNodes, g.edgeList, int(s))
            assert np.array_equal(lvl[k], rl)
            assert np.array_equal(sig[k], rs)  # integers below 2^53: exact


@pytest.mark.parametrize("cluster", [1, 2, 4, 8])
def test_bc_many_graphs_one_launch(cluster):
    # each graph taken by one CTA or by a cluster of CTAs with cluster barriers
    gs = G.er_batch(12, 200, 3000, 4, 12, seed=3)
    offs = [0]
    src_all, soff = [], [0]
    pairs_s, pairs_d = [], []
    for k, g in enumerate(gs):
        b = offs[-1]
        u = np.repeat(np.arange(g.V, dtype=np.int32), np.diff(g.indexofNodes))
        pairs_s.append(u + b)
        pairs_d.append(g.edgeList + b)
        src_all.append(G.pick_sources(g, 16, seed=k) + b)
        soff.append(soff[-1] + src_all[-1].shape[0])
        offs.append(b + g.V)
    V = offs[-1]
    union = from_pairs(V, np.stack([np.concatenate(pairs_s), np.concatenate(pairs_d)], 1), name="union")
    with DeviceGraph.from_csr(union) as dg:
        dg.tune_set("bc.cluster", cluster)
        assert dg.tune_get("bc.cluster") == cluster
        out = dg.bc_graphs(np.array(offs, np.int32), np.array(soff, np.int32), np.concatenate(src_all))
    for k, g in enumerate(gs):
        ref = O.bc(g.indexofNodes, g.edgeList, src_all[k] - offs[k])
        assert_bc_close(out[offs[k]:offs[k + 1]], ref, f"graph{k}")


def test_bc_at_scale():
    g = G.rmat(17, 16, seed=1)
    srcs = G.pick_sources(g, 96, seed=20)
    out = device_graph(g).bc(srcs)
    assert_bc_close(out, O.bc(g.indexofNodes, g.edgeList, srcs), "rmat17")


@pytest.mark.parametrize("policy", [1, 2, 3])
def test_bc_forward_direction_per_level_keeps_results(policy):
    # pull levels (bottom-up over in-edges, hubs in shared pieces) and push levels mixed by
    # the rule, by a seeded random choice, or pull everywhere: BFS levels and path counts
    # stay bit-exact and BC within its tolerance, on undirected and directed graphs and
    # on a star whose hub has more in-edges than a pull piece
    from graphs import star

    graphs = [G.rmat(13, 16, seed=3), G.rmat(12, 8, seed=5, directed=True), G.grid(30, 40),
              star(5000, directed_in=False)]
    for g in graphs:
        srcs = G.pick_sources(g, 40, seed=policy)
        with DeviceGraph.from_csr(g, with_weights=False) as dg:
            dg.tune_set("bc.dir", policy)
            for seed in (1, 2):
                dg.tune_set("bc.dir_seed", seed)
                out = dg.bc(srcs)
                assert_bc_close(out, O.bc(g.indexofNodes, g.edgeList, srcs), g.name)
                lvl, sig = dg.bfs_sigma(srcs[:8])
                for k, s in enumerate(srcs[:8]):
                    rl, rs, _ = O.bfs_sigma(g.indexofNodes, g.edgeList, int(s))
                    assert np.array_equal(lvl[k], rl) and np.array_equal(sig[k], rs), (g.name, policy, k)


def test_bc_level_trace_records_the_directions():
    import ctypes

    from starplat_b200._lib import check, lib

    g = G.rmat(14, 16, seed=2)
    srcs = G.pick_sources(g, 64, seed=4)
    with DeviceGraph.from_csr(g, with_weights=False) as dg:
        dg.tune_set("bc.dir", 2)
        dg.tune_set("bc.trace", 1)
        dg.bc(srcs)
        rec = np.zeros((4096, 16), np.float32)
        t = np.zeros(4097, np.uint64)
        n = ctypes.c_int32()
        check("sp_bc_level_trace", lib().sp_bc_level_trace(dg.handle, rec.ctypes.data, t.ctypes.data, 4096,
                                                           ctypes.byref(n)))
    k = int(n.value)
    assert k > 3
    pull = rec[:k, _lib.SP_MLP_IN]
    assert set(pull.tolist()) <= {0.0, 1.0} and pull.sum() > 0
    assert np.array_equal(rec[:k, 10], pull)  # the direction input of the level model
    assert (np.diff(t[:k + 1].astype(np.int64)) >= 0).all()
    assert (rec[:k, 4] > 0).all()  # log2(1 + entries of the level)


def test_bc_level_model_direction_keeps_results_and_matches_the_network():
    # a loaded level model (random weights: the device evaluation is what is checked)
    # decides each level's direction; results stay exact, and every traced level's
    # direction is the argmin of the network's two scores computed by the forward kernel
    import ctypes

    from starplat_b200 import scheduler as S
    from starplat_b200._lib import check, lib

    p = S.init_params(21)
    mean = np.zeros(_lib.SP_MLP_IN, np.float32)
    scale = np.full(_lib.SP_MLP_IN, 0.4, np.float32)
    check("sp_sched_level_load", lib().sp_sched_level_load(p.ctypes.data, mean.ctypes.data, scale.ctypes.data))
    try:
        g = G.rmat(14, 16, seed=6)
        srcs = G.pick_sources(g, 64, seed=2)
        with DeviceGraph.from_csr(g, with_weights=False) as dg:
            assert dg.tune_get("bc.dir") == -1  # default: the model when one is loaded
            dg.tune_set("bc.trace", 1)
            out = dg.bc(srcs)
            x, pull, ns = S.level_trace(dg)
        assert_bc_close(out, O.bc(g.indexofNodes, g.edgeList, srcs), g.name)
        assert x.shape[0] > 3
        rows = np.repeat(x, 2, axis=0)
        rows[0::2, 10], rows[1::2, 10] = 0.0, 1.0
        rows[:, 11] = rows[:, 10] * rows[:, 7]
        rows[:, 12] = rows[:, 10] * rows[:, 4]
        y = S.mlp_forward(p, (rows - mean) * scale).reshape(-1, 2)
        best = np.argmin(y, axis=1)
        taken = pull.astype(np.int64)
        gap = y[np.arange(len(y)), taken] - y[np.arange(len(y)), best]
        assert np.all(gap <= 1e-4 * np.maximum(1.0, np.abs(y).max(axis=1))), gap.max()
    finally:
        S.unload_level()
