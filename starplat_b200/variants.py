"""Learned kernel-variant choice for PageRank, TC, BC and Louvain.

Each of these algorithms has a small table of kernel variants in the library
(sp_variant_count): PageRank chooses which of the most-gathered sources allocate their
contrib gathers in L1, the srcList cache policy and the load width; TC chooses the
shared-bitmap kernel's CTA width (up to 65536 vertices) or the hash kernel's probe-list
elements per lane (above); BC chooses the degree above which a level-list entry is cut
into pieces shared by all warps, and the piece size; Louvain chooses, at every level,
the shared-memory table size of its CTA degree bin. Variants change only how work is
split or cached: counts, levels and path counts are the same under every one of them.

A network of the scheduler's shape (csrc/sp_mlp.cu) per algorithm predicts the log run
time of every applicable candidate from 13 inputs the library computes on the device
(sp_variant_features: degree statistics of the graph, or of the level graph, and the
candidate), and the call runs the lowest prediction. Training data are this method's
own timings: ``collect`` forces every candidate (knob ``<a>.variant`` = k) on a set of
training graphs and times it with CUDA events; for Louvain the per-level device times
come from the level trace (``lv.trace``). The fused training kernel (sp_mlp_train) fits
the network.

    python -m starplat_b200.variants train [pagerank tc bc louvain] [--out-dir DIR]
    python -m starplat_b200.variants refit MODEL.json ...   # again from the stored samples

Training selects the number of Adam steps and a switch margin (a call leaves the
defaults' candidate only when the predicted gain exceeds it) by leave-one-graph-out
regret, and records that regret beside the fixed defaults' on the same held-out graphs.

A trained model is loaded with ``load``; the knob ``<a>.variant`` = -2 keeps the fixed
defaults with a model loaded, and ``<a>.last_variant`` reports the candidate a call ran.
"""
from __future__ import annotations

import ctypes
import json
import math
import os
import statistics
import sys
import time

import numpy as np

from . import _lib
from ._lib import check, lib

_HERE = os.path.dirname(os.path.abspath(__file__))
ALGOS = {"pagerank": _lib.SP_VARIANT_PAGERANK, "tc": _lib.SP_VARIANT_TC, "bc": _lib.SP_VARIANT_BC,
         "louvain": _lib.SP_VARIANT_LOUVAIN}
KNOB = {"pagerank": "pr", "tc": "tc", "bc": "bc", "louvain": "lv"}
# the candidate each algorithm runs without a model (its fixed defaults)
DEFAULT_CANDIDATE = {"pagerank": 10, "tc": None, "bc": 3, "louvain": 4}
IN, P = _lib.SP_MLP_IN, _lib.SP_MLP_PARAMS


def model_path(algo: str) -> str:
    return os.path.join(_HERE, f"sched_variant_{algo}.json")


def count(algo: str) -> int:
    n = ctypes.c_int32()
    check("sp_variant_count", lib().sp_variant_count(ALGOS[algo], ctypes.byref(n)))
    return int(n.value)


def default_candidate(dg, algo: str) -> int:
    """The table entry equal to the fixed defaults on this graph."""
    if algo == "tc":
        return 2 if dg.V <= 65536 else 7
    return DEFAULT_CANDIDATE[algo]


def features(dg, algo: str, nsrc: int = 1):
    """(X[n][IN], applicable[n]) for every candidate of algo's table on dg."""
    n = count(algo)
    X = np.empty((n, IN), np.float32)
    ok = np.zeros(n, bool)
    a = ctypes.c_int32()
    for k in range(n):
        check("sp_variant_features", lib().sp_variant_features(dg.handle, ALGOS[algo], k, int(nsrc),
                                                               X[k].ctypes.data, ctypes.byref(a)))
        ok[k] = bool(a.value)
    return X, ok


def load_params(algo: str, params, mean, scale, margin: float = 0.0) -> None:
    """Load a network for algo; calls leave the defaults' candidate only for a predicted
    gain above `margin` (log units)."""
    p = np.ascontiguousarray(params, np.float32)
    mu = np.ascontiguousarray(mean, np.float32)
    sc = np.ascontiguousarray(scale, np.float32)
    if p.shape[0] != P or mu.shape[0] != IN or sc.shape[0] != IN:
        raise ValueError("variant model shape does not match this library")
    check("sp_sched_variant_load", lib().sp_sched_variant_load(ALGOS[algo], p.ctypes.data, mu.ctypes.data,
                                                               sc.ctypes.data, float(margin)))


def load(algos=None, shipped_only: bool = True) -> list:
    """Load the trained variant models whose files exist (by default only those marked
    shipped: measured no slower than the defaults); returns the algorithms loaded."""
    done = []
    for a in (algos or list(ALGOS)):
        path = model_path(a)
        if not os.path.exists(path):
            continue
        d = json.load(open(path))
        if shipped_only and not d.get("shipped", False):
            continue
        load_params(a, d["params"], d["feat_mean"], d["feat_scale"], d.get("margin", 0.0))
        done.append(a)
    return done


def unload(algos=None) -> None:
    for a in (algos or list(ALGOS)):
        check("sp_sched_variant_load", lib().sp_sched_variant_load(ALGOS[a], None, None, None, 0.0))


def louvain_trace(dg):
    """The last traced Louvain run's levels: (inputs[k][IN], candidate[k], ms[k])."""
    cap = 64
    rec = np.empty((cap, 16), np.float32)
    n = ctypes.c_int32()
    check("sp_louvain_level_trace", lib().sp_louvain_level_trace(dg.handle, rec.ctypes.data, cap,
                                                                 ctypes.byref(n)))
    k = min(int(n.value), cap)
    return rec[:k, :IN].copy(), rec[:k, IN].astype(np.int64), rec[:k, IN + 1].astype(np.float64)


# ----------------------------------------------------------------------------- timing

def _runner(dg, algo: str, args: dict):
    import torch

    if algo == "tc":
        return lambda: dg.tc()
    if algo == "pagerank":
        out = torch.empty(dg.V, dtype=torch.float32, device="cuda")
        return lambda: dg.pagerank(1e-6, 0.85, 100, out=out)
    if algo == "bc":
        src = np.asarray(args["sources"], np.int32)
        out = torch.empty(dg.V, dtype=torch.float32, device="cuda")
        return lambda: dg.bc(src, out=out)
    if algo == "louvain":
        return lambda: dg.louvain()
    raise ValueError(algo)


def time_call(fn, reps: int = 3) -> float:
    """Median device milliseconds of fn() over reps runs after one untimed run."""
    import torch

    fn()
    stream = torch.cuda.current_stream()
    ts = []
    for _ in range(reps):
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        fn()
        b.record(stream)
        torch.cuda.synchronize()
        ts.append(a.elapsed_time(b))
    return statistics.median(ts)


def time_variant(dg, algo: str, mode: int, args: dict | None = None, reps: int = 3) -> float:
    """Device ms of one call with knob <a>.variant = mode (-2 defaults, -1 learned, k)."""
    key = KNOB[algo] + ".variant"
    old = dg.tune_get(key)
    dg.tune_set(key, mode)
    try:
        return time_call(_runner(dg, algo, args or {}), reps)
    finally:
        dg.tune_set(key, old)


# ----------------------------------------------------------------------------- training data

def training_graphs(algo: str):
    """(name, graph, args) per algorithm. None of them is a benchmark configuration
    (PageRank R-MAT 22, TC R-MAT 16, BC R-MAT 20 with 256 sources, Louvain on the
    1M-vertex planted partition)."""
    from . import generators as G

    out = []
    if algo == "pagerank":
        for sc in (14, 16, 18, 20, 21, 23):
            out.append((f"rmat{sc}d", G.rmat(sc, 16, seed=sc, directed=True), {}))
        out.append(("rmat19d_ef8", G.rmat(19, 8, seed=5, directed=True), {}))
        out.append(("rmat18u", G.rmat(18, 16, seed=118), {}))
        out.append(("er18_d16", G.erdos_renyi(1 << 18, 16, seed=3), {}))
        out.append(("er20_d8", G.erdos_renyi(1 << 20, 8, seed=4), {}))
        out.append(("grid1024", G.grid(1024, 1024), {}))
        out.append(("grid2048", G.grid(2048, 2048), {}))
    elif algo == "tc":
        for sc in (12, 13, 14, 15):
            out.append((f"rmat{sc}u", G.rmat(sc, 16, seed=sc + 200), {}))
        out.append(("rmat15u_ef8", G.rmat(15, 8, seed=9), {}))
        out.append(("er16_d16", G.erdos_renyi(1 << 16, 16, seed=6), {}))
        out.append(("er15_d32", G.erdos_renyi(1 << 15, 32, seed=7), {}))
        out.append(("grid256", G.grid(256, 256), {}))
        out.append(("rmat16d", G.rmat(16, 16, seed=16, directed=True), {}))
        for sc in (17, 18, 19):
            out.append((f"rmat{sc}u", G.rmat(sc, 16, seed=sc + 200), {}))
        out.append(("rmat16u_ef12", G.rmat(16, 12, seed=216), {}))
        out.append(("rmat16u_ef20", G.rmat(16, 20, seed=217), {}))
        out.append(("er18_d16", G.erdos_renyi(1 << 18, 16, seed=8), {}))
        out.append(("er19_d8", G.erdos_renyi(1 << 19, 8, seed=10), {}))
        out.append(("grid1024", G.grid(1024, 1024), {}))
        out.append(("rmat18d", G.rmat(18, 16, seed=18, directed=True), {}))
    elif algo == "bc":
        for sc, ns in ((16, 64), (17, 128), (18, 64), (19, 128), (19, 256)):
            g = G.rmat(sc, 16, seed=sc + 300)
            out.append((f"rmat{sc}u_s{ns}", g, {"sources": G.pick_sources(g, ns, seed=sc)}))
        for n, ns in ((512, 64), (1024, 32)):
            g = G.grid(n, n)
            out.append((f"grid{n}_s{ns}", g, {"sources": G.pick_sources(g, ns, seed=n)}))
        g = G.erdos_renyi(1 << 18, 8, seed=11)
        out.append(("er18_d8_s64", g, {"sources": G.pick_sources(g, 64, seed=1)}))
        g = G.erdos_renyi(1 << 17, 32, seed=12)
        out.append(("er17_d32_s64", g, {"sources": G.pick_sources(g, 64, seed=2)}))
        g = G.rmat(18, 16, seed=18, directed=True)
        out.append(("rmat18d_s64", g, {"sources": G.pick_sources(g, 64, seed=3)}))
    elif algo == "louvain":
        for v, nb in ((1 << 16, 64), (1 << 18, 128), (1 << 19, 512)):
            out.append((f"sbm{v}_{nb}", G.sbm(v, nb, seed=nb), {}))
        out.append(("sbm262144_16_d64", G.sbm(1 << 18, 16, avg_degree=64.0, seed=5), {}))
        out.append(("sbm1048576_64", G.sbm(1 << 20, 64, seed=7), {}))
        for sc in (15, 17, 19):
            out.append((f"rmat{sc}u", G.rmat(sc, 16, seed=sc + 400), {}))
        out.append(("er18_d16", G.erdos_renyi(1 << 18, 16, seed=13), {}))
        out.append(("grid512", G.grid(512, 512), {}))
    else:
        raise ValueError(algo)
    return out


def collect(algo: str, graphs, reps: int = 3, log=print):
    """Time every applicable candidate on every graph. Returns X[N][IN], T[N] (log ms)
    and meta [(graph, candidate, ms)]; for Louvain one sample per level and candidate."""
    from .device import DeviceGraph

    import torch

    rows, targets, meta = [], [], []
    key = KNOB[algo] + ".variant"
    for name, g, args in graphs:
        with DeviceGraph.from_csr(g) as dg:
            dg.set_stream(torch.cuda.current_stream())
            nsrc = len(args.get("sources", ())) or 1
            X, ok = features(dg, algo, nsrc)
            cands = [k for k in range(len(ok)) if ok[k]]
            if algo == "louvain":
                dg.tune_set("lv.trace", 1)
                for k in cands:
                    dg.tune_set(key, k)
                    per_level = []
                    for _ in range(reps):
                        dg.louvain()
                        xs, cs, ms = louvain_trace(dg)
                        per_level.append((xs, ms))
                    xs = per_level[0][0]
                    nl = min(len(p[1]) for p in per_level)
                    for lvl in range(nl):
                        m = statistics.median(float(p[1][lvl]) for p in per_level)
                        rows.append(xs[lvl])
                        targets.append(math.log(max(m, 1e-3)))
                        meta.append((f"{name}/L{lvl}", k, m))
                dg.tune_set(key, -1)
                dg.tune_set("lv.trace", 0)
            else:
                for k in cands:
                    m = time_variant(dg, algo, k, args, reps)
                    rows.append(X[k])
                    targets.append(math.log(m))
                    meta.append((name, k, m))
        mine = [x for x in meta if x[0].split("/")[0] == name]
        best = min(mine, key=lambda x: x[2])
        log(f"  {name}: best candidate {best[1]} ({best[2]:.3f} ms) of {len(cands)}")
    return np.array(rows, np.float32), np.array(targets, np.float32), meta


def default_of(algo: str, cands) -> int:
    """The defaults' candidate among the applicable ones of a decision."""
    if algo == "tc":
        return 2 if 2 in cands else 7
    return DEFAULT_CANDIDATE[algo]


def _picks(y, T, meta, algo, margin):
    """Per graph: (time of the picked candidates / time of the best ones, time of the
    defaults / time of the best ones), the times summed over the graph's decisions (one
    per graph, or one per Louvain level) and the picks made with the library's margin
    rule."""
    acc = {}
    units = sorted(set(m[0] for m in meta), key=[m[0] for m in meta].index)
    for u in units:
        idx = [i for i, m in enumerate(meta) if m[0] == u]
        cands = [meta[i][1] for i in idx]
        d = idx[cands.index(default_of(algo, cands))]
        b = idx[int(np.argmin(y[idx]))]
        pick = b if y[d] - y[b] > margin else d
        a = acc.setdefault(u.split("/")[0], [0.0, 0.0, 0.0])
        a[0] += math.exp(T[pick])
        a[1] += math.exp(T[d])
        a[2] += min(math.exp(T[i]) for i in idx)
    return {g: (v[0] / v[2], v[1] / v[2]) for g, v in acc.items()}


MARGINS = (0.0, math.log(1.02), math.log(1.05), math.log(1.10))
STEPS = (300, 1000, 3000)


def _loo(algo, X, T, meta, steps):
    """Leave one graph out: network predictions for every sample of the held-out graph."""
    from .scheduler import fit, mlp_forward

    graph_of = [m[0].split("/")[0] for m in meta]
    y = np.empty(len(meta), np.float64)
    for name in sorted(set(graph_of), key=graph_of.index):
        te = np.array([gname == name for gname in graph_of])
        p, mu, sc, _ = fit(X[~te], T[~te], steps=steps)
        y[te] = mlp_forward(p, (X[te] - mu) * sc)
    return y


def fit_and_select(algo: str, X, T, meta, log=print) -> dict:
    """Choose the training length and the switch margin by leave-one-graph-out regret,
    then fit on every sample."""
    from .scheduler import fit

    best = None
    table = {}
    for steps in STEPS:
        y = _loo(algo, X, T, meta, steps)
        for mg in MARGINS:
            r = _picks(y, T, meta, algo, mg)
            learned = float(np.mean([v[0] for v in r.values()]))
            fixed = float(np.mean([v[1] for v in r.values()]))
            table[f"steps{steps}_margin{math.exp(mg):.2f}"] = {"learned_regret": learned, "fixed_regret": fixed}
            if best is None or learned < best[0] - 1e-9:
                best = (learned, steps, mg, fixed, r)
    learned, steps, mg, fixed, r = best
    params, mean, scale, loss = fit(X, T, steps=steps)
    log(f"{algo}: held-out regret learned {learned:.3f} vs fixed {fixed:.3f} (steps {steps}, margin "
        f"x{math.exp(mg):.2f}), train loss {loss:.4f}")
    return {"params": params.tolist(), "feat_mean": mean.tolist(), "feat_scale": scale.tolist(),
            "margin": mg, "train_steps": steps, "train_loss": loss,
            "leave_one_graph_out": {"learned_regret": learned, "fixed_regret": fixed,
                                    "per_graph": {u: [round(a, 4), round(b, 4)] for u, (a, b) in r.items()},
                                    "selection": table}}


def train(algo: str, out: str | None = None, reps: int = 3, log=print) -> dict:
    """Collect timings, select and fit (fit_and_select), write the model file with its
    samples (not marked shipped: shipping is a measured decision)."""
    import torch

    out = out or model_path(algo)
    t0 = time.time()
    graphs = training_graphs(algo)
    log(f"{algo}: timing {count(algo)} candidates on {len(graphs)} graphs")
    X, T, meta = collect(algo, graphs, reps, log)
    d = {"algo": algo, **fit_and_select(algo, X, T, meta, log), "samples": int(X.shape[0]),
         "X": X.tolist(), "T": T.tolist(), "meta": [[m[0], int(m[1]), round(m[2], 4)] for m in meta],
         "shipped": False, "gpu": torch.cuda.get_device_name(0), "collect_and_train_s": round(time.time() - t0, 1)}
    with open(out, "w") as f:
        json.dump(d, f)
    log(f"{algo}: wrote {out}")
    return d


def refit(path: str, log=print) -> dict:
    """Select and fit again from the samples stored in a model file (GPU training
    kernel); keeps the file's shipped flag."""
    d = json.load(open(path))
    X = np.asarray(d["X"], np.float32)
    T = np.asarray(d["T"], np.float32)
    meta = [tuple(m) for m in d["meta"]]
    d.update(fit_and_select(d["algo"], X, T, meta, log))
    with open(path, "w") as f:
        json.dump(d, f)
    return d


def main(argv=None):
    import torch

    argv = sys.argv[1:] if argv is None else argv
    if argv and argv[0] == "refit":
        torch.cuda.set_device(0)
        for path in argv[1:]:
            refit(path)
        return 0
    if not argv or argv[0] != "train":
        print(__doc__)
        return 1
    out_dir = None
    rest = argv[1:]
    if "--out-dir" in rest:
        i = rest.index("--out-dir")
        out_dir = rest[i + 1]
        rest = rest[:i] + rest[i + 2:]
    torch.cuda.set_device(0)
    for a in (rest or list(ALGOS)):
        train(a, os.path.join(out_dir, os.path.basename(model_path(a))) if out_dir else None)
    return 0


if __name__ == "__main__":
    sys.exit(main())
