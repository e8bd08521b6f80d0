"""GPU: learned kernel variants of PageRank, TC, BC and Louvain.

* every candidate of each table gives the oracle's results (TC counts exact, PageRank
  L1 < 1e-6 against FP64, BC within 1e-5 relative, Louvain the same partition quality);
* with a model loaded, the candidate a call runs is the argmin of the network's scores
  over the applicable candidates, recomputed on the host from the library's inputs;
* Louvain's level trace records one entry per level with the inputs of the candidate
  that ran;
* a shipped model is no slower than the fixed defaults on graphs outside its training
  set.
"""
import numpy as np
import pytest

from oracle import oracle as O
from starplat_b200 import generators as G
from starplat_b200 import scheduler, variants
from starplat_b200.device import DeviceGraph

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def _no_models():
    variants.unload()
    yield
    variants.unload()


def _bc_close(out, ref):
    out = out.astype(np.float64)
    return np.all(np.abs(out - ref) <= 1e-5 * np.abs(ref) + 1e-9 * max(1.0, ref.max()))


def _pr_l1(dg, g):
    out, it, _ = dg.pagerank(1e-6, 0.85, 100)
    ref, _, _ = O.pagerank(g.indexofNodes, g.rev_indexofNodes, g.srcList, 1e-6, 0.85, 100, fixed_iters=it)
    return np.abs(out.astype(np.float64) - ref).sum()


def test_variant_tables_and_knobs():
    g = G.rmat(10, 8, seed=1)
    with DeviceGraph.from_csr(g) as dg:
        for algo, key in variants.KNOB.items():
            n = variants.count(algo)
            assert n >= 4
            assert dg.tune_get(key + ".variant") == -1
            assert dg.tune_get(key + ".last_variant") == -1
            with pytest.raises(RuntimeError):
                dg.tune_set(key + ".variant", n)
            with pytest.raises(RuntimeError):
                dg.tune_set(key + ".variant", -3)
        with pytest.raises(RuntimeError):
            dg.tune_set("tc.unroll", 3)
        with pytest.raises(RuntimeError):
            dg.tune_set("lv.cta_slots", 1000)


@pytest.mark.parametrize("directed", [True, False])
def test_pagerank_every_candidate_matches_oracle(directed):
    g = G.rmat(15, 16, seed=21, directed=directed)
    g.ensure_reverse()
    with DeviceGraph.from_csr(g) as dg:
        X, ok = variants.features(dg, "pagerank")
        assert ok.all() and np.isfinite(X).all()
        for k in range(variants.count("pagerank")):
            dg.tune_set("pr.variant", k)
            l1 = _pr_l1(dg, g)
            assert dg.tune_get("pr.last_variant") == k
            assert l1 < 1e-6, (k, l1)


def test_tc_every_candidate_exact():
    small = G.rmat(13, 16, seed=22)
    big = G.rmat(17, 8, seed=23)
    for g, path in ((small, 1), (big, 0)):
        ref = O.tc(g.indexofNodes, g.edgeList)
        with DeviceGraph.from_csr(g) as dg:
            X, ok = variants.features(dg, "tc")
            assert ok.sum() >= 3 and np.isfinite(X).all()
            for k in range(variants.count("tc")):
                if not ok[k]:
                    assert X[k, 8] != path
                    with pytest.raises(RuntimeError):
                        dg.tune_set("tc.variant", k)
                        dg.tc()
                    dg.tune_set("tc.variant", -1)
                    continue
                dg.tune_set("tc.variant", k)
                assert dg.tc() == ref, k
                assert dg.tune_get("tc.last_variant") == k


def test_bc_every_candidate_within_tolerance():
    g = G.rmat(14, 16, seed=24)
    srcs = G.pick_sources(g, 40, seed=5)
    ref = O.bc(g.indexofNodes, g.edgeList, srcs)
    with DeviceGraph.from_csr(g) as dg:
        for k in range(variants.count("bc")):
            dg.tune_set("bc.variant", k)
            assert _bc_close(dg.bc(srcs), ref), k
            assert dg.tune_get("bc.last_variant") == k


def test_louvain_every_candidate_same_partition_and_trace():
    # R-MAT hubs reach the CTA bins, and the small tables push some of them to the
    # global-table bin; with unit weights every bin computes the same gains.
    g = G.rmat(15, 16, seed=25)
    with DeviceGraph.from_csr(g) as dg:
        dg.tune_set("lv.trace", 1)
        q0, comm0, lv0 = dg.louvain()
        xs0, cs0, ms0 = variants.louvain_trace(dg)
        assert len(xs0) == lv0 and (ms0 > 0).all()
        assert (cs0 == variants.DEFAULT_CANDIDATE["louvain"]).all()
        X, ok = variants.features(dg, "louvain")
        np.testing.assert_allclose(xs0[0], X[variants.DEFAULT_CANDIDATE["louvain"]], rtol=1e-6)
        assert abs(q0 - O.modularity(g.indexofNodes, g.edgeList, comm0)) < 1e-6
        for k in range(variants.count("louvain")):
            dg.tune_set("lv.variant", k)
            q, comm, lv = dg.louvain()
            xs, cs, ms = variants.louvain_trace(dg)
            assert (cs == k).all() and len(cs) == lv
            assert np.array_equal(comm, comm0) and q == q0, k


def _random_model(seed):
    rng = np.random.default_rng(seed)
    return (scheduler.init_params(seed), rng.normal(0, 1, variants.IN).astype(np.float32),
            np.full(variants.IN, 0.3, np.float32))


@pytest.mark.parametrize("seed", [1, 2])
def test_learned_pick_is_network_argmin(seed):
    g = G.rmat(14, 16, seed=26)
    g.ensure_reverse()
    srcs = G.pick_sources(g, 24, seed=6)
    with DeviceGraph.from_csr(g) as dg:
        for algo in ("pagerank", "tc", "bc", "louvain"):
            p, mu, sc = _random_model(seed + 10 * variants.ALGOS[algo])
            variants.load_params(algo, p, mu, sc)
            if algo == "pagerank":
                dg.pagerank(1e-6, 0.85, 100)
            elif algo == "tc":
                dg.tc()
            elif algo == "bc":
                dg.bc(srcs)
            else:
                dg.tune_set("lv.trace", 1)
                dg.louvain()
            key = variants.KNOB[algo] + ".last_variant"
            if algo == "louvain":
                # level 0 is the input graph, whose inputs the library gives for every
                # candidate; later levels record only the candidate that ran
                xs, cs, _ = variants.louvain_trace(dg)
                X, _ = variants.features(dg, algo)
                np.testing.assert_allclose(xs[0], X[int(cs[0])], rtol=1e-6)
                y = scheduler.mlp_forward(p, (X - mu) * sc)
                assert int(cs[0]) == int(np.argmin(y)) or abs(y[int(cs[0])] - y.min()) < 1e-4
                assert ((cs >= 0) & (cs < variants.count(algo))).all()
                assert dg.tune_get(key) == int(cs[-1])
            else:
                X, ok = variants.features(dg, algo, len(srcs) if algo == "bc" else 1)
                y = scheduler.mlp_forward(p, (X - mu) * sc)
                y[~ok] = np.inf
                pick = dg.tune_get(key)
                assert ok[pick]
                assert pick == int(np.argmin(y)) or abs(y[pick] - y.min()) < 1e-4, (algo, pick, y)
            # -2: the fixed defaults even with a model loaded
            dg.tune_set(variants.KNOB[algo] + ".variant", -2)
            if algo == "pagerank":
                dg.pagerank(1e-6, 0.85, 100)
                assert dg.tune_get(key) == -1
            dg.tune_set(variants.KNOB[algo] + ".variant", -1)
            variants.unload([algo])


def test_margin_keeps_the_defaults():
    # a margin no prediction can beat: every call runs the defaults' candidate
    g = G.rmat(14, 16, seed=27)
    g.ensure_reverse()
    srcs = G.pick_sources(g, 24, seed=7)
    with DeviceGraph.from_csr(g) as dg:
        for algo in ("pagerank", "tc", "bc", "louvain"):
            p, mu, sc = _random_model(3 + variants.ALGOS[algo])
            variants.load_params(algo, p, mu, sc, margin=1e6)
            if algo == "pagerank":
                dg.pagerank(1e-6, 0.85, 100)
            elif algo == "tc":
                dg.tc()
            elif algo == "bc":
                dg.bc(srcs)
            else:
                dg.louvain()
            assert dg.tune_get(variants.KNOB[algo] + ".last_variant") == variants.default_candidate(dg, algo)
            variants.unload([algo])
    with pytest.raises(RuntimeError):
        variants.load_params("tc", p, mu, sc, margin=-1.0)


@pytest.mark.parametrize("algo", ["pagerank", "tc", "bc", "louvain"])
def test_shipped_model_not_slower_on_unseen_graphs(algo):
    import torch

    if not variants.load([algo]):
        pytest.skip(f"no shipped {algo} variant model")
    cases = {
        "pagerank": [G.rmat(19, 16, seed=77, directed=True), G.erdos_renyi(1 << 19, 12, seed=78)],
        "tc": [G.rmat(14, 24, seed=79), G.rmat(18, 12, seed=80)],
        "bc": [G.rmat(17, 16, seed=81), G.grid(768, 768)],
        "louvain": [G.sbm(1 << 17, 96, seed=82), G.rmat(16, 16, seed=83)],
    }[algo]
    tl = tf = 0.0
    for g in cases:
        g.ensure_reverse()
        args = {"sources": G.pick_sources(g, 64, seed=4)} if algo == "bc" else {}
        with DeviceGraph.from_csr(g) as dg:
            dg.set_stream(torch.cuda.current_stream())
            tf += variants.time_variant(dg, algo, -2, args, reps=5)
            tl += variants.time_variant(dg, algo, -1, args, reps=5)
    print(f"{algo}: fixed {tf:.3f} ms, learned {tl:.3f} ms, gain x{tf / tl:.3f}")
    assert tl <= 1.05 * tf, (tl, tf)
