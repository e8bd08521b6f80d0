"""Learned schedule selection for SSSP (bucket width, CTAs per SM, warp cascades).

The network (csrc/sp_mlp.cu) predicts the log run time of SSSP on a graph under a
candidate schedule from 13 inputs the library builds itself (sp_sssp_features:
graph size, degree skew, symmetry, weight range, the candidate). It is trained on
timings this method generates (``collect`` times every candidate on a set of
training graphs with CUDA events) by the project's own fused training kernel
(``sp_mlp_train``), and loaded with ``sp_sched_load``; from then on sp_sssp with no
explicit delta scores all 63 candidates on the GPU and runs the best one. Warp
cascades (the sssp.local knob) pay on thin, high-diameter frontiers and cost on
skewed ones, so they are part of the choice. Without a model the fixed heuristic
(delta = largest weight, 4 CTAs per SM, cascades of 64 steps) runs. Schedules change
speed only: distances are exact either way.

    python -m starplat_b200.scheduler train     # collect, train, write sched_model.json

A second network with the same shape makes a decision per iteration inside the
kernel: at every bucket advance of a delta-stepping solve it scores six width factors
(1/4 .. 8 times the call's delta) from inputs the kernel reads on the device (far-pile
size, rounds and relaxations of the previous epoch, progress, the previous factor) and
widens or narrows the next bucket accordingly (knob sssp.epoch). Its training data are
traces of solves that pick a seeded random factor per epoch (sssp.epoch = 2): per epoch
the chosen factor's inputs and the measured device time per unit of distance advanced.

    python -m starplat_b200.scheduler train-epoch   # collect traces, train, write sched_epoch_model.json

A third network of the same shape decides BC's forward direction per level inside the
kernel (push along the level's out-edges, or pull over the in-edges of the vertices not
yet reached by every source): it predicts the level's log time in each direction from
the level's statistics, and every CTA takes the direction with the lower prediction.
Its training data are traces of runs with a seeded random direction per level (bc.dir = 2).

    python -m starplat_b200.scheduler train-level   # collect BC traces, train, write sched_level_model.json
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
EPOCH_MODEL_PATH = os.path.join(_HERE, "sched_epoch_model.json")
EPOCH_FACTORS = (0.25, 0.5, 1.0, 2.0, 4.0, 8.0)  # the kernel's width candidates (kFacNum / 4)
LEVEL_MODEL_PATH = os.path.join(_HERE, "sched_level_model.json")
MULTS = (1, 2, 4, 8, 16, 32, 64)
CTAS = (1, 2, 4)
LOCALS = (0, 64, 256)  # warp cascade budget per round (sssp.local): off, the default, long
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


def load(path: str = MODEL_PATH, epoch_path: str = EPOCH_MODEL_PATH, level_path: str = LEVEL_MODEL_PATH) -> bool:
    """Load the model (and the per-epoch width and per-level direction models, when their
    files exist, and the shipped kernel-variant models of variants.py) into the library;
    False (fixed heuristic stays) if the SSSP model file is absent."""
    _settle_auto_load()
    if epoch_path and os.path.exists(epoch_path):
        load_epoch(epoch_path)
    if level_path and os.path.exists(level_path):
        load_level(level_path)
    from . import variants

    variants.load()  # the kernel-variant models marked shipped
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
    """Back to the fixed heuristic (and fixed bucket widths and kernel variants), also for
    later calls in this process."""
    _settle_auto_load()
    check("sp_sched_load", lib().sp_sched_load(None, None, None))
    check("sp_sched_epoch_load", lib().sp_sched_epoch_load(None, None, None))
    check("sp_sched_level_load", lib().sp_sched_level_load(None, None, None))
    from . import variants

    variants.unload()


def _load_packed(path, call) -> bool:
    if not os.path.exists(path):
        return False
    d = json.load(open(path))
    p = np.asarray(d["params"], np.float32)
    mean = np.asarray(d["feat_mean"], np.float32)
    scale = np.asarray(d["feat_scale"], np.float32)
    if p.shape[0] != P or mean.shape[0] != IN:
        raise ValueError(f"{path}: model shape does not match this library")
    check(call, getattr(lib(), call)(p.ctypes.data, mean.ctypes.data, scale.ctypes.data))
    return True


def load_epoch(path: str = EPOCH_MODEL_PATH) -> bool:
    """Load the per-epoch width model only; False if the file is absent."""
    return _load_packed(path, "sp_sched_epoch_load")


def load_level(path: str = LEVEL_MODEL_PATH) -> bool:
    """Load the BC per-level direction model only; False if the file is absent."""
    return _load_packed(path, "sp_sched_level_load")


def unload_level() -> None:
    check("sp_sched_level_load", lib().sp_sched_level_load(None, None, None))


def level_trace(dg):
    """The last traced BC run's levels: (inputs[n][IN], pull[n], ns[n])."""
    cap = 1 << 14
    rec = np.empty((cap, 16), np.float32)
    t = np.empty(cap + 1, np.uint64)
    n = ctypes.c_int32()
    check("sp_bc_level_trace", lib().sp_bc_level_trace(dg.handle, rec.ctypes.data, t.ctypes.data, cap,
                                                       ctypes.byref(n)))
    k = min(int(n.value), cap)
    if int(n.value) > cap:
        k -= 1
    ns = (t[1:k + 1].astype(np.int64) - t[:k].astype(np.int64)).astype(np.float64)
    return rec[:k, :IN].copy(), rec[:k, IN].copy(), ns


def bc_training_graphs():
    """(name, graph, sources) for the level model: sizes below the benchmark's R-MAT 20."""
    from . import generators as G

    out = []
    for sc in (14, 16, 18, 19):
        g = G.rmat(sc, 16, seed=sc + 50)
        out.append((f"rmat{sc}u", g, G.pick_sources(g, 64, seed=sc)))
    g = G.rmat(17, 8, seed=9, directed=True)
    out.append(("rmat17d", g, G.pick_sources(g, 64, seed=9)))
    for n, d in ((1 << 16, 8), (1 << 18, 16)):
        g = G.erdos_renyi(n, d, seed=n % 97)
        out.append((f"er{n}_d{d}", g, G.pick_sources(g, 64, seed=3)))
    g = G.grid(512, 512)
    out.append(("grid512", g, G.pick_sources(g, 32, seed=5)))
    g = G.sbm(1 << 17, 64, seed=3)
    out.append(("sbm17", g, G.pick_sources(g, 64, seed=2)))
    return out


def collect_levels(graphs, seeds=(1, 2, 3, 4, 5, 6), log=print):
    """Exploration runs (a seeded random direction per level) with traces: one sample
    per level, target log2 of its device nanoseconds."""
    from .device import DeviceGraph

    import torch

    X, T = [], []
    for name, g, srcs in graphs:
        with DeviceGraph.from_csr(g, with_weights=False) as dg:
            dg.set_stream(torch.cuda.current_stream())
            dg.tune_set("bc.dir", 0)
            dg.bc(srcs)  # warm-up
            dg.tune_set("bc.dir", 2)
            dg.tune_set("bc.trace", 1)
            n0 = sum(x.shape[0] for x in X)
            for sd in seeds:
                dg.tune_set("bc.dir_seed", sd)
                dg.bc(srcs)
                torch.cuda.synchronize()
                x, pull, ns = level_trace(dg)
                ok = ns > 0
                X.append(x[ok])
                T.append(np.log2(ns[ok]).astype(np.float32))
            dg.tune_set("bc.trace", 0)
            dg.tune_set("bc.dir", -1)
        log(f"  {name}: {sum(x.shape[0] for x in X) - n0} levels")
    return np.concatenate(X), np.concatenate(T)


def time_bc(dg, srcs, policy: int, reps: int = 3) -> float:
    """Best-of-reps device time of sp_bc under a direction policy."""
    import torch

    dg.tune_set("bc.dir", policy)
    dg.bc(srcs)
    best = None
    for _ in range(reps):
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(torch.cuda.current_stream())
        dg.bc(srcs)
        b.record(torch.cuda.current_stream())
        torch.cuda.synchronize()
        t = a.elapsed_time(b)
        best = t if best is None else min(best, t)
    dg.tune_set("bc.dir", -1)
    return best


def train_level(out: str = LEVEL_MODEL_PATH, log=print) -> dict:
    """Collect BC exploration traces, fit the level model with the fused training kernel,
    and write it."""
    import torch

    t0 = time.time()
    graphs = bc_training_graphs()
    log(f"collecting BC level traces on {len(graphs)} graphs")
    X, T = collect_levels(graphs, log=log)
    params, mean, scale, loss = fit(X, T, steps=6000)
    d = {"params": params.tolist(), "feat_mean": mean.tolist(), "feat_scale": scale.tolist(),
         "train_loss": loss, "samples": int(X.shape[0]), "target": "log2(device ns) of one forward level",
         "gpu": torch.cuda.get_device_name(0), "collect_and_train_s": round(time.time() - t0, 1)}
    with open(out, "w") as f:
        json.dump(d, f, indent=1)
    log(f"trained on {X.shape[0]} levels: loss {loss:.4f}; wrote {out}")
    return d


def unload_epoch() -> None:
    """Fixed bucket widths again (the per-call model stays)."""
    check("sp_sched_epoch_load", lib().sp_sched_epoch_load(None, None, None))


def epoch_trace(dg):
    """The last traced solve's epochs: (inputs[n][IN], factor[n], advance[n], ns[n]), the
    time of each epoch from its advance to the next (the last epoch's to the end)."""
    cap = 1 << 16
    rec = np.empty((cap, 16), np.float32)
    t = np.empty(cap + 1, np.uint64)
    n = ctypes.c_int32()
    check("sp_sssp_epoch_trace", lib().sp_sssp_epoch_trace(dg.handle, rec.ctypes.data, t.ctypes.data, cap,
                                                           ctypes.byref(n)))
    k = min(int(n.value), cap)
    if int(n.value) > cap:
        k -= 1  # the last record's end lies past the trace
    ns = (t[1:k + 1].astype(np.int64) - t[:k].astype(np.int64)).astype(np.float64)
    return rec[:k, :IN].copy(), rec[:k, IN].copy(), rec[:k, IN + 1].copy(), ns


def epoch_scores(params, mean, scale, inputs):
    """Scores of every width factor for each traced epoch's state (the kernel's argmin
    is the chosen factor): inputs[n][IN] with the candidate columns replaced."""
    rows = []
    for x in inputs:
        for f in EPOCH_FACTORS:
            r = np.array(x, np.float32)
            r[10] = math.log2(f)
            r[11] = r[10] * r[4]
            rows.append(r)
    y = mlp_forward(params, (np.array(rows, np.float32) - mean) * scale)
    return y.reshape(len(inputs), len(EPOCH_FACTORS))


def collect_epochs(graphs, seeds=(1, 2, 3, 4, 5, 6), log=print):
    """Exploration solves (a seeded random width factor per epoch) with traces: one
    sample per epoch, target log2(ns per unit of distance advanced)."""
    from .device import DeviceGraph

    import torch

    X, T, meta = [], [], []
    for name, g, src in graphs:
        with DeviceGraph.from_csr(g) as dg:
            dg.set_stream(torch.cuda.current_stream())
            out = torch.empty(g.V, dtype=torch.int32, device="cuda")
            dg.sssp(src, out=out)  # warm-up; fixes the call's learned delta
            dg.tune_set("sssp.trace", 1)
            dg.tune_set("sssp.epoch", 2)
            for sd in seeds:
                dg.tune_set("sssp.epoch_seed", sd)
                dg.sssp(src, out=out)
                torch.cuda.synchronize()
                x, f, adv, ns = epoch_trace(dg)
                ok = (adv > 0) & (ns > 0)
                X.append(x[ok])
                T.append(np.log2(ns[ok] / adv[ok]).astype(np.float32))
                meta += [(name, sd)] * int(ok.sum())
            dg.tune_set("sssp.epoch", -1)
            dg.tune_set("sssp.trace", 0)
        log(f"  {name}: {sum(1 for m in meta if m[0] == name)} epochs")
    return np.concatenate(X), np.concatenate(T), meta


def time_policy(dg, src, policy: int, reps: int = 3) -> float:
    """Best-of-reps device time of one solve under an epoch policy (0 fixed, 1 learned)."""
    import torch

    dg.tune_set("sssp.epoch", policy)
    out = torch.empty(dg.V, dtype=torch.int32, device="cuda")
    dg.sssp(src, out=out)
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
    dg.tune_set("sssp.epoch", -1)
    return best


def train_epoch(out: str = EPOCH_MODEL_PATH, log=print) -> dict:
    """Collect exploration traces on the training graphs, fit the epoch model with the
    fused training kernel, and write it."""
    import torch

    t0 = time.time()
    load(MODEL_PATH, epoch_path=None)  # the per-call choice fixes each solve's base delta
    graphs = training_graphs()
    log(f"collecting per-epoch traces on {len(graphs)} graphs")
    X, T, meta = collect_epochs(graphs, log=log)
    params, mean, scale, loss = fit(X, T, steps=6000)
    d = {"params": params.tolist(), "feat_mean": mean.tolist(), "feat_scale": scale.tolist(),
         "factors": list(EPOCH_FACTORS), "train_loss": loss, "samples": int(X.shape[0]),
         "target": "log2(device ns per unit of distance advanced) of one epoch",
         "gpu": torch.cuda.get_device_name(0), "collect_and_train_s": round(time.time() - t0, 1)}
    with open(out, "w") as f:
        json.dump(d, f, indent=1)
    log(f"trained on {X.shape[0]} epochs: loss {loss:.4f}; wrote {out}")
    return d


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
    if argv and argv[0] == "train-level":
        torch.cuda.set_device(0)
        train_level(argv[1] if len(argv) > 1 else LEVEL_MODEL_PATH)
        return 0
    if argv and argv[0] == "train-epoch":
        torch.cuda.set_device(0)
        train_epoch(argv[1] if len(argv) > 1 else EPOCH_MODEL_PATH)
        return 0
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
