"""Learned schedule selection for SSSP (bucket width, CTAs per SM, warp cascades).

The network (csrc/sp_mlp.cu) predicts the log run time of SSSP on a graph under a
candidate schedule from 13 inputs the library builds itself (sp_sssp_features:
graph size, degree skew, symmetry, weight range, the candidate). It is trained on
timings this method generates (``collect`` times every candidate on a set of
training graphs with CUDA events) by the project's own fused training kernel
(``sp_mlp_train``), and loaded with ``sp_sched_load``; from then on sp_sssp with no
explicit delta scores all 42 candidates on the GPU and runs the best one. Warp
cascades (the sssp.local knob) pay on thin, high-diameter frontiers and cost on
skewed ones, so they are part of the choice. Without a model the fixed heuristic
(delta = largest weight, 4 CTAs per SM, cascades of 64 steps) runs. Schedules change
speed only: distances are exact either way.

    python -m starplat_b200.scheduler train     # collect, train, write sched_model.json
"""
from __future__ import annotations

import ctypes
import json
import math
import os
import sys
import time

import numpy as np

from . import _lib
from ._lib import check, lib

_HERE = os.path.dirname(os.path.abspath(__file__))
MODEL_PATH = os.path.join(_HERE, "sched_model.json")
MULTS = (1, 2, 4, 8, 16, 32, 64)
CTAS = (1, 2, 4)
LOCALS = (0, 64)  # warp cascade budget per round (sssp.local), off or the default
CANDIDATES = [(m, c, l) for m in MULTS for c in CTAS for l in LOCALS]
IN, P = _lib.SP_MLP_IN, _lib.SP_MLP_PARAMS

f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")


def _fp(a):
    return np.ascontiguousarray(a, np.float32).ctypes.data


def init_params(seed: int = 0) -> np.ndarray:
    """Glorot-uniform weights, zero biases, in the kernel's parameter layout."""
    rng = np.random.default_rng(seed)
    H = _lib.SP_MLP_HIDDEN

    def glorot(o, i):
        a = math.sqrt(6.0 / (o + i))
        return rng.uniform(-a, a, size=(o, i))

    p = np.concatenate([glorot(H, IN).ravel(), np.zeros(H), glorot(H, H).ravel(), np.zeros(H),
                        glorot(1, H).ravel(), [0.0]])
    assert p.shape[0] == P
    return p.astype(np.float32)


def mlp_forward(params, X) -> np.ndarray:
    X = np.ascontiguousarray(X, np.float32)
    y = np.empty(X.shape[0], np.float32)
    check("sp_mlp_forward", lib().sp_mlp_forward(_fp(params), X.ctypes.data, X.shape[0], y.ctypes.data))
    return y


def mlp_grad(params, X, T):
    X = np.ascontiguousarray(X, np.float32)
    T = np.ascontiguousarray(T, np.float32)
    g = np.empty(P, np.float32)
    loss = np.zeros(1, np.float32)
    p = np.ascontiguousarray(params, np.float32)
    check("sp_mlp_grad", lib().sp_mlp_grad(p.ctypes.data, X.ctypes.data, T.ctypes.data, X.shape[0], g.ctypes.data,
                                           loss.ctypes.data))
    return float(loss[0]), g


def mlp_train(params, X, T, steps: int, lr: float):
    """Full-batch Adam on the GPU, all steps in one fused launch; returns (params, loss)."""
    p = np.array(params, np.float32, copy=True)
    X = np.ascontiguousarray(X, np.float32)
    T = np.ascontiguousarray(T, np.float32)
    loss = np.zeros(1, np.float32)
    check("sp_mlp_train", lib().sp_mlp_train(p.ctypes.data, X.ctypes.data, T.ctypes.data, X.shape[0], steps, lr,
                                             loss.ctypes.data))
    return p, float(loss[0])


def features(dg, mult: float, ctas: int, local: int = 64, weight=None) -> np.ndarray:
    from .device import _ptr

    x = np.empty(IN, np.float32)
    check("sp_sssp_features", lib().sp_sssp_features(dg.handle, _ptr(weight), float(mult), int(ctas), int(local),
                                                     x.ctypes.data))
    return x


# ----------------------------------------------------------------------------- model file

def _settle_auto_load() -> None:
    """An explicit load() or unload() decides: the first DeviceGraph.sssp of the process
    must not load the shipped model over it afterwards."""
    from . import device

    device._SCHED_TRIED = True


def load(path: str = MODEL_PATH) -> bool:
    """Load the model into the library; False (fixed heuristic stays) if absent."""
    _settle_auto_load()
    if not os.path.exists(path):
        return False
    d = json.load(open(path))
    p = np.asarray(d["params"], np.float32)
    mean = np.asarray(d["feat_mean"], np.float32)
    scale = np.asarray(d["feat_scale"], np.float32)
    if p.shape[0] != P or mean.shape[0] != IN:
        raise ValueError(f"{path}: model shape does not match this library")
    check("sp_sched_load", lib().sp_sched_load(p.ctypes.data, mean.ctypes.data, scale.ctypes.data))
    return True


def unload() -> None:
    """Back to the fixed heuristic, also for later calls in this process."""
    _settle_auto_load()
    check("sp_sched_load", lib().sp_sched_load(None, None, None))


# ----------------------------------------------------------------------------- data collection

def training_graphs():
    """(name, graph with edgeLen, source) — sizes below the benchmark configs, which
    the model never sees while training."""
    from . import generators as G

    out = []

    def add(name, g, wlo, whi, sym, seed):
        g.edgeLen = G.hash_weights(g, seed, wlo, whi, sym)
        src = int(G.pick_sources(g, 1, seed=seed)[0])
        out.append((name, g, src))

    for sc in (14, 16, 18, 20, 21, 22):
        add(f"rmat{sc}d_w100", G.rmat(sc, 16, seed=sc, directed=True), 1, 100, False, sc)
    add("rmat17d_ef8_w1000", G.rmat(17, 8, seed=5, directed=True), 1, 1000, False, 5)
    for sc in (15, 17):
        add(f"rmat{sc}u_w100", G.rmat(sc, 16, seed=sc + 100), 1, 100, True, sc)
    for n in (128, 256, 512, 1024, 2048, 3072):
        add(f"grid{n}_w1000", G.grid(n, n), 1, 1000, True, n)
    add("grid512_w100", G.grid(512, 512), 1, 100, True, 7)
    add("er16_d4", G.erdos_renyi(1 << 16, 4, seed=3), 1, 100, True, 3)
    add("er18_d8", G.erdos_renyi(1 << 18, 8, seed=4), 1, 100, True, 4)
    add("er16_d16", G.erdos_renyi(1 << 16, 16, seed=6), 1, 1000, True, 6)
    return out


def time_sssp(dg, src, mult, ctas, wmax, reps=3, local=64):
    import torch

    dg.tune_set("sssp.delta", max(1, int(round(mult * wmax))))
    dg.tune_set("sssp.ctas_per_sm", ctas)
    dg.tune_set("sssp.local", local)
    out = torch.empty(dg.V, dtype=torch.int32, device="cuda")
    dg.sssp(src, out=out)  # warm-up
    best = None
    for _ in range(reps):
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(torch.cuda.current_stream())
        dg.sssp(src, out=out)
        b.record(torch.cuda.current_stream())
        torch.cuda.synchronize()
        t = a.elapsed_time(b)
        best = t if best is None else min(best, t)
    dg.tune_set("sssp.delta", 0)
    dg.tune_set("sssp.ctas_per_sm", 0)
    dg.tune_set("sssp.local", 64)
    return best


def collect(graphs, reps: int = 3, log=print):
    from .device import DeviceGraph

    import torch

    rows, targets, meta = [], [], []
    for name, g, src in graphs:
        wmax = int(g.edgeLen.max()) if g.E else 1
        with DeviceGraph.from_csr(g) as dg:
            dg.set_stream(torch.cuda.current_stream())
            for m, c, l in CANDIDATES:
                ms = time_sssp(dg, src, m, c, wmax, reps, l)
                rows.append(features(dg, m, c, l))
                targets.append(math.log(ms))
                meta.append((name, m, c, l, ms))
        best = min((x for x in meta if x[0] == name), key=lambda x: x[4])
        log(f"  {name}: best delta={best[1]}x ctas={best[2]} local={best[3]} {best[4]:.3f} ms")
    return np.array(rows, np.float32), np.array(targets, np.float32), meta


def fit(X, T, steps=4000, lr=3e-3, seed=0):
    mean = X.mean(0)
    std = X.std(0)
    scale = np.where(std > 1e-6, 1.0 / np.maximum(std, 1e-6), 0.0).astype(np.float32)
    Xn = (X - mean) * scale
    params, loss = mlp_train(init_params(seed), Xn, T, steps, lr)
    return params, mean.astype(np.float32), scale, loss


def regret(params, mean, scale, X, T, meta):
    """Per graph: time of the predicted-best candidate / time of the true best."""
    y = mlp_forward(params, (X - mean) * scale)
    out = {}
    names = sorted(set(m[0] for m in meta), key=[m[0] for m in meta].index)
    for name in names:
        idx = [i for i, m in enumerate(meta) if m[0] == name]
        pick = idx[int(np.argmin(y[idx]))]
        best = idx[int(np.argmin(T[idx]))]
        out[name] = float(math.exp(T[pick] - T[best]))
    return out


def main(argv=None):
    import torch

    argv = sys.argv[1:] if argv is None else argv
    if not argv or argv[0] != "train":
        print(__doc__)
        return 1
    out = argv[1] if len(argv) > 1 else MODEL_PATH
    torch.cuda.set_device(0)
    t0 = time.time()
    graphs = training_graphs()
    print(f"collecting timings on {len(graphs)} graphs x {len(CANDIDATES)} schedules")
    X, T, meta = collect(graphs)
    # leave-one-graph-out check of how well the network ranks schedules
    names = sorted(set(m[0] for m in meta), key=[m[0] for m in meta].index)
    loo = {}
    for name in names:
        tr = np.array([m[0] != name for m in meta])
        p, mu, sc, _ = fit(X[tr], T[tr])
        te = ~tr
        loo[name] = regret(p, mu, sc, X[te], T[te], [m for m in meta if m[0] == name])[name]
    params, mean, scale, loss = fit(X, T)
    d = {"params": params.tolist(), "feat_mean": mean.tolist(), "feat_scale": scale.tolist(),
         "candidates": CANDIDATES, "train_loss": loss, "samples": int(X.shape[0]),
         "leave_one_graph_out_regret": loo, "train_regret": regret(params, mean, scale, X, T, meta),
         "timings_ms": [[m[0], m[1], m[2], m[3], round(m[4], 4)] for m in meta],
         "gpu": torch.cuda.get_device_name(0), "collect_and_train_s": round(time.time() - t0, 1)}
    with open(out, "w") as f:
        json.dump(d, f, indent=1)
    print(f"trained: loss {loss:.4f}; leave-one-graph-out regret "
          f"{np.mean(list(loo.values())):.3f} (1.0 = always the best schedule); wrote {out}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
