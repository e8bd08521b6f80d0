"""GPU: the learned scheduler. The network's CUDA kernels agree with the FP64
oracle (forward, gradient); the fused training kernel fits; a loaded model keeps
SSSP exact; and on graphs it was not trained on, the learned schedule is compared
with the fixed heuristic (the gain is printed; the learned one must not lose)."""
import math
import os

import numpy as np
import pytest

from oracle import mlp_oracle as M
from oracle import oracle as O
from starplat_b200 import _lib
from starplat_b200 import generators as G
from starplat_b200 import scheduler as S
from starplat_b200.device import DeviceGraph

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True)
def no_model_after_each_test():
    yield
    S.unload()


def data(n=300, seed=1):
    rng = np.random.default_rng(seed)
    X = rng.normal(0, 1, (n, M.IN)).astype(np.float32)
    T = (np.sin(X[:, 0]) + 0.5 * X[:, 1] * X[:, 2] - 0.3 * X[:, 3] ** 2).astype(np.float32)
    return X, T


def test_forward_matches_oracle():
    p = S.init_params(3)
    X, _ = data()
    y = S.mlp_forward(p, X)
    ref, _, _ = M.forward(p.astype(np.float64), X.astype(np.float64))
    assert np.allclose(y, ref, rtol=1e-4, atol=1e-5)


def test_gradient_matches_oracle():
    rng = np.random.default_rng(2)
    p = (rng.normal(0, 0.3, _lib.SP_MLP_PARAMS)).astype(np.float32)
    X, T = data(517)  # not a multiple of the warp size
    loss, g = S.mlp_grad(p, X, T)
    L, gr = M.loss_grad(p.astype(np.float64), X.astype(np.float64), T.astype(np.float64))
    assert abs(loss - L) <= 1e-4 * max(1.0, L)
    err = np.linalg.norm(g - gr) / np.linalg.norm(gr)
    assert err < 1e-4, err
    assert np.allclose(g, gr, rtol=1e-3, atol=1e-6 * np.abs(gr).max())


def test_fused_training_fits():
    X, T = data(800)
    p0 = S.init_params(0)
    L0, _ = M.loss_grad(p0.astype(np.float64), X, T)
    p, loss = S.mlp_train(p0, X, T, steps=1500, lr=3e-3)
    L1, _ = M.loss_grad(p.astype(np.float64), X, T)
    # `loss` is the kernel's loss at the start of its last step (before the last update)
    assert L1 < 0.1 * L0 and loss < 0.1 * L0


def _small_model():
    """A model trained on random rows (schedule choice arbitrary but valid)."""
    rng = np.random.default_rng(5)
    X = rng.normal(0, 1, (256, M.IN)).astype(np.float32)
    T = rng.normal(0, 1, 256).astype(np.float32)
    p, _ = S.mlp_train(S.init_params(1), X, T, steps=50, lr=1e-3)
    mean = np.zeros(M.IN, np.float32)
    scale = np.ones(M.IN, np.float32)
    return p, mean, scale


def test_loaded_model_keeps_sssp_exact():
    p, mean, scale = _small_model()
    S.unload()  # settles the shipped model's lazy load, which would replace this one
    _lib.check("sp_sched_load", _lib.lib().sp_sched_load(p.ctypes.data, mean.ctypes.data, scale.ctypes.data))
    for g in (G.rmat(13, 16, seed=2, directed=True), G.grid(60, 70)):
        g.edgeLen = G.hash_weights(g, 9, 1, 100, g.is_symmetric())
        with DeviceGraph.from_csr(g) as dg:
            out, _ = dg.sssp(1)
            assert dg.tune_get("sssp.last_delta") >= 1 and dg.tune_get("sssp.last_ctas") in (1, 2, 4)
        assert np.array_equal(out, O.sssp(g.indexofNodes, g.edgeList, g.edgeLen, 1))


def test_learned_choice_is_reused_only_for_the_same_inputs():
    # the network's inputs are the graph and the weight range: a second call with the
    # same range reuses the choice, a new range or a new model scores again, and
    # without a model the fixed heuristic runs; distances stay exact throughout
    g = G.rmat(13, 8, seed=4, directed=True)
    w = G.hash_weights(g, 4, 1, 100, False)
    ref = O.sssp(g.indexofNodes, g.edgeList, w, 0)
    p, mean, scale = _small_model()
    with DeviceGraph.from_csr(g) as dg:
        S.unload()  # settles the shipped model's lazy load, which would replace this one
        _lib.check("sp_sched_load", _lib.lib().sp_sched_load(p.ctypes.data, mean.ctypes.data, scale.ctypes.data))

        def run(weights):
            out, _ = dg.sssp(0, weight=weights)
            return out, (dg.tune_get("sssp.last_delta"), dg.tune_get("sssp.last_ctas"))

        out1, c1 = run(w)
        out2, c2 = run(w)
        assert c1 == c2 and np.array_equal(out1, ref) and np.array_equal(out2, ref)
        assert c1[0] % int(w.max()) == 0
        w10 = (w * 10).astype(np.int32)
        out3, c3 = run(w10)
        assert c3[0] % int(w10.max()) == 0  # scored again: a multiple of the new largest weight
        assert np.array_equal(out3, O.sssp(g.indexofNodes, g.edgeList, w10, 0))
        # another model (negated scores reverse the ranking) must not reuse the old choice
        q = p.copy()
        q[-1 - _lib.SP_MLP_HIDDEN:] *= -1
        _lib.check("sp_sched_load", _lib.lib().sp_sched_load(q.ctypes.data, mean.ctypes.data, scale.ctypes.data))
        out4, c4 = run(w)
        assert np.array_equal(out4, ref)
        S.unload()
        out5, c5 = run(w)
        assert c5 == (int(w.max()), 4) and np.array_equal(out5, ref)


def test_unload_is_not_undone_by_the_lazy_model_load():
    # in a fresh process the first sssp call loads the shipped model, unless the caller
    # already chose: after an explicit unload the fixed heuristic must run
    import subprocess
    import sys

    code = (
        "from starplat_b200 import generators as G, scheduler as S\n"
        "from starplat_b200.device import DeviceGraph\n"
        "g = G.rmat(12, 8, seed=3, directed=True)\n"
        "w = G.hash_weights(g, 3, 1, 100, False)\n"
        "S.unload()\n"
        "with DeviceGraph.from_csr(g) as dg:\n"
        "    dg.sssp(0, weight=w)\n"
        "    print(dg.tune_get('sssp.last_delta'), dg.tune_get('sssp.last_ctas'), int(w.max()))\n")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    out = subprocess.run([sys.executable, "-c", code], cwd=root, capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    delta, ctas, wmax = map(int, out.stdout.split())
    assert (delta, ctas) == (wmax, 4)


def test_learned_schedule_gain_on_unseen_graphs():
    if not os.path.exists(S.MODEL_PATH):
        pytest.skip("no trained model (python -m starplat_b200.scheduler train)")
    import torch

    held_out = []
    g = G.rmat(19, 16, seed=77, directed=True)
    g.edgeLen = G.hash_weights(g, 77, 1, 100, False)
    held_out.append(("rmat19", g, int(G.pick_sources(g, 1, seed=77)[0])))
    g = G.grid(1536, 1536)
    g.edgeLen = G.hash_weights(g, 78, 1, 1000, True)
    held_out.append(("grid1536", g, 777))
    g = G.erdos_renyi(1 << 19, 6, seed=79)
    g.edgeLen = G.hash_weights(g, 79, 1, 100, True)
    held_out.append(("er19_d6", g, 5))
    total_fixed = total_learned = 0.0
    lines = []
    for name, g, src in held_out:
        with DeviceGraph.from_csr(g) as dg:
            dg.set_stream(torch.cuda.current_stream())

            def run():
                out = torch.empty(g.V, dtype=torch.int32, device="cuda")
                dg.sssp(src, out=out)
                a = torch.cuda.Event(enable_timing=True)
                b = torch.cuda.Event(enable_timing=True)
                best = None
                for _ in range(3):
                    a.record()
                    dg.sssp(src, out=out)
                    b.record()
                    torch.cuda.synchronize()
                    best = a.elapsed_time(b) if best is None else min(best, a.elapsed_time(b))
                return best, out.cpu().numpy()

            S.unload()
            t_fixed, d_fixed = run()
            assert S.load()
            t_learned, d_learned = run()
            choice = (dg.tune_get("sssp.last_delta"), dg.tune_get("sssp.last_ctas"))
        assert np.array_equal(d_fixed, d_learned)
        total_fixed += t_fixed
        total_learned += t_learned
        lines.append(f"{name}: fixed {t_fixed:.2f} ms, learned {t_learned:.2f} ms (delta, ctas = {choice})")
    print("\n".join(lines) + f"\ntotal: fixed {total_fixed:.2f} ms, learned {total_learned:.2f} ms, "
          f"gain x{total_fixed / total_learned:.2f}")
    assert total_learned <= 1.05 * total_fixed


def _load_random_epoch_model(seed=5):
    # a random epoch model (the device inference is what is checked, not its quality)
    p = S.init_params(seed)
    mean = np.zeros(_lib.SP_MLP_IN, np.float32)
    scale = np.full(_lib.SP_MLP_IN, 0.3, np.float32)
    from starplat_b200._lib import check, lib

    check("sp_sched_epoch_load", lib().sp_sched_epoch_load(p.ctypes.data, mean.ctypes.data, scale.ctypes.data))
    return p, mean, scale


def test_per_epoch_widths_keep_sssp_exact():
    # any per-epoch width sequence gives the exact distances: seeded random factors
    # (exploration) and a loaded epoch model, single-source and batched
    _load_random_epoch_model()
    for g in (G.rmat(13, 16, seed=4, directed=True), G.grid(60, 70), G.rmat(12, 8, seed=9)):
        g.edgeLen = G.hash_weights(g, 2, 1, 500, g.is_symmetric())
        srcs = G.pick_sources(g, 3, seed=1)
        refs = [O.sssp(g.indexofNodes, g.edgeList, g.edgeLen, int(s)) for s in srcs]
        with DeviceGraph.from_csr(g) as dg:
            for pol, seed in ((2, 1), (2, 7), (1, 0), (0, 0)):
                dg.tune_set("sssp.epoch", pol)
                dg.tune_set("sssp.epoch_seed", seed)
                for s, ref in zip(srcs, refs):
                    d, _ = dg.sssp(int(s))
                    assert np.array_equal(d, ref), (g.name, pol, seed)
                    assert dg.tune_get("sssp.last_epolicy") == pol
                rows = dg.sssp_batch(srcs)
                for k in range(len(srcs)):
                    assert np.array_equal(rows[k], refs[k]), (g.name, pol, "batch")


def test_in_kernel_epoch_choice_matches_the_network():
    # the factor every CTA picked at each advance is the argmin of the network's scores
    # for that epoch's inputs, computed again by the forward kernel
    p, mean, scale = _load_random_epoch_model(11)
    g = G.grid(200, 200)
    g.edgeLen = G.hash_weights(g, 3, 1, 1000, True)
    with DeviceGraph.from_csr(g) as dg:
        dg.tune_set("sssp.epoch", 1)
        dg.tune_set("sssp.trace", 1)
        d, _ = dg.sssp(0)
        assert np.array_equal(d, O.sssp(g.indexofNodes, g.edgeList, g.edgeLen, 0))
        x, f, adv, ns = S.epoch_trace(dg)
    assert x.shape[0] > 5 and (adv > 0).all()
    y = S.epoch_scores(p, mean, scale, x)
    picked = np.array([S.EPOCH_FACTORS.index(float(v)) for v in f])
    best = np.argmin(y, axis=1)
    # equal up to near-ties between the kernel's fused evaluation and the forward kernel
    gap = y[np.arange(len(y)), picked] - y[np.arange(len(y)), best]
    assert np.all(gap <= 1e-4 * np.maximum(1.0, np.abs(y).max(axis=1))), gap.max()


@pytest.mark.skipif(not os.path.exists(S.EPOCH_MODEL_PATH), reason="no trained epoch model shipped")
def test_per_epoch_width_gain_on_unseen_graphs():
    # graphs outside the training set: the shipped epoch model against fixed widths (the
    # per-call choice stays loaded for both); printed, and the learned total must not
    # lose by more than 5%
    S.load()
    tot = {0: 0.0, 1: 0.0}
    for g in (G.rmat(19, 16, seed=77, directed=True), G.grid(1536, 1536), G.erdos_renyi(1 << 19, 8, seed=5)):
        g.edgeLen = G.hash_weights(g, 9, 1, 1000 if g.is_symmetric() else 100, g.is_symmetric())
        src = int(G.pick_sources(g, 1, seed=3)[0])
        with DeviceGraph.from_csr(g) as dg:
            t0 = S.time_policy(dg, src, 0)
            t1 = S.time_policy(dg, src, 1)
        print(f"{g.name}: fixed widths {t0:.3f} ms, learned per epoch {t1:.3f} ms")
        tot[0] += t0
        tot[1] += t1
    print(f"total gain x{tot[0] / tot[1]:.3f}")
    assert tot[1] <= 1.05 * tot[0]
