"""Benchmark: GTEPS of the static-graph hot path on B200 (one JSON line on rank 0).

Headline (value / e2e / roofline / cpu_baseline): PageRank, pull over the reverse
CSR, on a directed R-MAT graph, scale 22 (4,194,304 vertices), edge factor 16,
a/b/c/d = .57/.19/.19/.05, seed 1, damping 0.85, L1 threshold 1e-6, maxIter 100.
A step is one full PageRank call (all iterations until convergence);
GTEPS = E * iterations / time.

  value         device-resident CSR (uploaded before timing), CUDA events on the stream
  e2e           through the C ABI with HOST buffers: upload from pinned memory +
                PageRank + result D2H, every step
  roofline      the iteration kernel: algorithmic bytes 8E + 16V per launch over its
                average launch time (from two fixed-iteration runs) vs the measured HBM peak
  cpu_baseline  the OpenMP form of the generated code (oracle port), 3 iterations

"algorithms" holds the other workloads of the metric "GTEPS per algorithm", each
timed the same way (device-resident, events), with the plain fixed-schedule GPU
form beside the tuned one, an algorithm-level roofline fraction and a bounded CPU
baseline:
  tc_rmat16        triangle counting, undirected R-MAT 16 ef16 (GTEPS = m / t)
  sssp_rmat23      SSSP, directed R-MAT 23 ef16, weights U[1,100] (E_r / t)
  sssp_grid4096    SSSP, 4096x4096 4-neighbour grid, weights U[1,1000] (E_r / t)
  bc_rmat20        BC, undirected R-MAT 20 ef16, 256 sources (S * E_r / t)
  bc_er1000        BC, 1000 ER graphs (1k-50k vertices, degree 8-32), 16 sources each
  louvain_sbm1m    Louvain, planted partition 1,048,576 vertices, 256 blocks (E * sweeps / t)
  ingest_rmat20    text edge list -> device mirror (sp_graph_load_text), directed R-MAT 20
                   ef16 with weights (M edge lines / s; not a GTEPS figure)
  update_rmat20    one batch of 2^20 edge updates (half deletions) applied to the device
                   mirror of directed R-MAT 20 (M updates / s, host arrays to rebuilt CSR);
                   with batches of 4096 added edges, SSSP resumed from the old distances
                   and PageRank started from the old ranks, each against a cold solve; on
                   undirected R-MAT 20, triangles counted through the batch against a recount
  centrality       per-vertex triangle counts on the TC graph (m / t), and closeness on
                   the BC graph: unweighted over its 256 sources, weighted (U[1,100])
                   over 16 of them (sum of E_r / t)
Inputs are seeded synthetic graphs with the configs' shapes (no dataset is
available offline). Every workload's inputs exceed L2 (126 MB) except the TC
graph (7 MB CSR), which is small by definition of its config.

--impl reference times the reference's CPU path (the OpenMP form of the generated
PageRank, restated in oracle/) alone on the host cores, same metric and config.
Multi-GPU (--gpus N under torchrun): the headline runs N replicas of the whole
PageRank, and value sums the edges all ranks processed over the max time (weak
scaling). Beside it, "pagerank_split" runs the same graph split over the ranks by
vertices (all-gather of contrib blocks and all-reduce of the diff per iteration on
device buffers; strong scaling), the BC, clustering-coefficient and closeness legs
split their sources or anchor parts over the ranks with one all-reduce, and the SSSP
legs add a "split" entry: the single-source solve split over the ranks by vertices.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

PR_SCALE, PR_EF, PR_SEED = 22, 16, 1
BETA, DELTA, MAX_ITER = 1e-6, 0.85, 100
METRIC = "GTEPS per algorithm on 1 B200 (pagerank headline)"
INT_MAX = 2**31 - 1
TUNE = []  # (key, value) schedule knobs from --tune, applied to every device graph
REP = None  # the replica group of a multi-GPU run (set in main)


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


class Clocks:
    """nvidia-smi sampling during a timed region."""

    def __init__(self, index: int):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(index), f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                       "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None
        time.sleep(0.25)

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.3)
        self.p.terminate()
        self.p.wait()
        self.f.flush()
        rows = [r.split(",") for r in open(self.f.name).read().strip().splitlines() if r.strip()]
        os.unlink(self.f.name)

        def num(x):
            try:
                return float(x)
            except ValueError:
                return None

        sm = [num(r[1]) for r in rows if len(r) >= 9 and num(r[1]) is not None]
        mx = [num(r[2]) for r in rows if len(r) >= 9 and num(r[2]) is not None]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            if len(r) < 9:
                continue
            for n, v in zip(names, r[5:9]):
                if v.strip().lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(rows)}


def pr_graph(scale=None):
    from starplat_b200 import generators as G

    t = time.time()
    g = G.rmat(scale or PR_SCALE, PR_EF, seed=PR_SEED, directed=True)
    return g, time.time() - t


def cpu_pagerank(g, iters: int = 3):
    """OpenMP form of the generated PageRank on the host cores, `iters` iterations."""
    from oracle import oracle as O

    nt = O.num_threads()
    t = time.perf_counter()
    _, it = O.pagerank_omp(g.indexofNodes, g.rev_indexofNodes, g.srcList, 0.0, DELTA, iters, nthreads=nt)
    dt = time.perf_counter() - t
    return {"value": g.E * it / dt / 1e9, "unit": "GTEPS", "cores": nt, "kind": "port",
            "sample": f"{it} iterations of the OpenMP-form PageRank over the full graph ({dt:.2f} s)"}


def pr_config(g, world):
    """The headline's config, the same keys and values in both arms."""
    return {"workload": f"pagerank rmat{PR_SCALE} ef{PR_EF} directed seed{PR_SEED}", "V": g.V, "E": g.E,
            "beta": BETA, "delta": DELTA, "max_iter": MAX_ITER,
            "l2": "inputs larger than L2 (srcList %.2f GB streamed per iteration)" % (4 * g.E / 1e9),
            "parallelism": "replicas" if world > 1 else "single"}


def run_reference(args, rank):
    if rank != 0:
        return
    g, _ = pr_graph()
    for _ in range(args.warmup):
        cpu_pagerank(g, 1)
    vals = [cpu_pagerank(g, 3) for _ in range(args.steps)]
    v = statistics.median([x["value"] for x in vals])
    line = {"metric": METRIC, "value": v, "unit": "GTEPS", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic", "impl": "reference",
            "config": pr_config(g, args.gpus),
            "cpu_baseline": {**vals[-1], "value": v,
                             "sample": vals[-1]["sample"] + "; sampled: 3 of the run's iterations per step"},
            "e2e": {"value": v, "unit": "GTEPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------------------- timing helpers

def timed(fn, steps, warmup, stream):
    """Run fn() warmup times, then time `steps` runs with CUDA events on `stream`.
    Returns (ms per step, list of fn results)."""
    import torch

    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    a.record(stream)
    res = [fn() for _ in range(steps)]
    b.record(stream)
    torch.cuda.synchronize()
    return a.elapsed_time(b) / steps, res


def tuned(dg):
    for k, v in TUNE:
        try:
            dg.tune_set(k, v)
        except Exception:
            pass
    return dg


def learned_vs_fixed(dg, algo, run, stream, reps=3):
    """The algorithm's kernel-variant choice: fixed defaults (knob -2) against the trained
    network (-1), each timed over `reps` calls after one warm-up. A model not marked
    shipped is loaded for this comparison only."""
    from starplat_b200 import variants

    path = variants.model_path(algo)
    if not os.path.exists(path):
        return {"model": "none"}
    d = json.load(open(path))
    key = variants.KNOB[algo] + ".variant"
    variants.load([algo], shipped_only=False)
    try:
        dg.tune_set(key, -2)
        ms_f, _ = timed(run, reps, 1, stream)
        dg.tune_set(key, -1)
        ms_l, _ = timed(run, reps, 1, stream)
        cand = dg.tune_get(variants.KNOB[algo] + ".last_variant")
    finally:
        dg.tune_set(key, -1)
        if not d.get("shipped", False):
            variants.unload([algo])
    lo = d.get("leave_one_graph_out", {})
    return {"fixed_ms": ms_f, "learned_ms": ms_l, "learned_over_fixed": ms_f / ms_l, "learned_candidate": cand,
            "shipped": bool(d.get("shipped", False)), "decision": d.get("ship_decision"),
            "held_out_regret": {"learned": lo.get("learned_regret"), "fixed": lo.get("fixed_regret")}}


def bc_error(got, ref):
    """BC against the FP64 oracle: per-vertex bar |got - ref| <= 1e-5 |ref| + 1e-9 max(1, max ref).
    Returns the largest ratio of error to bar (<= 1 passes) and the largest relative
    error over vertices with BC >= 1."""
    got = np.asarray(got, np.float64)
    ref = np.asarray(ref, np.float64)
    err = np.abs(got - ref)
    bar = 1e-5 * np.abs(ref) + 1e-9 * max(1.0, float(ref.max(initial=0.0)))
    big = np.abs(ref) >= 1.0
    rel = float((err[big] / np.abs(ref[big])).max(initial=0.0))
    return float((err / bar).max(initial=0.0)), rel


def roof(alg_bytes, ms, hbm):
    gbs = alg_bytes / (ms / 1e3) / 1e9
    return {"achieved_gbs": round(gbs, 1), "frac": round(gbs / hbm, 4), "alg_bytes": int(alg_bytes)}


def component_edges(g):
    """Connected components of an undirected CSR: (label per vertex, edge entries per component)."""
    from scipy.sparse import csr_matrix
    from scipy.sparse.csgraph import connected_components

    A = csr_matrix((np.ones(g.E, np.int8), g.edgeList, g.indexofNodes), shape=(g.V, g.V))
    _, lab = connected_components(A, directed=False)
    ce = np.bincount(lab, weights=np.diff(g.indexofNodes))
    return lab, ce


# ----------------------------------------------------------------------------- other algorithms

def bench_tc(steps, warmup, stream, hbm, cpu):
    from starplat_b200 import _lib
    from starplat_b200 import generators as G
    from starplat_b200.device import DeviceGraph

    g = G.rmat(16, 16, seed=1)
    m = g.E // 2
    deg = np.diff(g.indexofNodes).astype(np.int64)
    u = np.repeat(np.arange(g.V), deg)
    v = g.edgeList.astype(np.int64)
    keep = (deg[u] < deg[v]) | ((deg[u] == deg[v]) & (u < v))
    dplus = np.bincount(u[keep], minlength=g.V)
    eplus = int(keep.sum())
    alg = 4 * int((dplus[u[keep]] + dplus[v[keep]]).sum()) + 4 * (g.V + 1) + 4 * eplus
    out = {"workload": "tc rmat16 ef16 undirected seed1", "V": g.V, "m": m, "E_plus": eplus}
    with DeviceGraph.from_csr(g, with_weights=False) as dg:
        dg.set_stream(stream)
        tuned(dg)
        if REP is not None and REP.world > 1:
            # anchor parts over the GPUs, one all-reduce of the int64 count (strong scaling)
            from starplat_b200.distributed import tc_on_gpus

            REP.barrier()
            ms, res = timed(lambda: tc_on_gpus(dg, REP), steps, warmup, stream)
            ms = REP.max(ms)
            out["parallelism"] = f"anchor parts over {REP.world} GPUs, one all-reduce of the count"
        else:
            ms, res = timed(lambda: dg.tc(), steps, warmup, stream)
        msp, resp = timed(lambda: dg.tc(_lib.SP_TC_PLAIN), max(1, steps // 2), 1, stream)
        if REP is None or REP.world == 1:
            out["learned_vs_fixed"] = learned_vs_fixed(dg, "tc", lambda: dg.tc(), stream)
    out.update({"triangles": res[0], "value": m / (ms / 1e3) / 1e9, "unit": "GTEPS", "ms": ms,
                "plain": {"value": m / (msp / 1e3) / 1e9, "ms": msp, "triangles": resp[0]},
                "roofline": roof(alg, ms, hbm)})
    if cpu:
        from oracle import oracle as O

        # work model of the OpenMP form: every (u, w) pair builds and scans N(u)
        k = 64
        low = v < u
        hi_cnt = np.bincount(u[v > u], minlength=g.V)
        sdeg = np.bincount(u[low], weights=deg[v[low]] + 1, minlength=g.V)
        work = sdeg * hi_cnt
        sample = work[np.arange(g.V) % k == 7].sum()
        nt = O.num_threads()
        kind = "reference" if O.ref_lib() is not None else "port"
        fn = O.ref_tc if kind == "reference" else O.tc_omp
        t = time.perf_counter()
        tc_s = fn(g.indexofNodes, g.edgeList, nthreads=nt, vfirst=7, vstride=k)
        dt = time.perf_counter() - t
        est = dt * work.sum() / max(1.0, sample)
        out["cpu_baseline"] = {"value": m / est / 1e9, "unit": "GTEPS", "cores": nt, "kind": kind,
                               "sample": f"OpenMP Compute_TC loop with graph::check_if_nbr over every {k}th vertex "
                                         f"({dt:.2f} s, {tc_s} triangles), scaled by the pair-scan work model "
                                         f"to a full run of {est:.1f} s"}
    return out


def bench_sssp(name, g, src, steps, warmup, stream, hbm, cpu, cpu_mode):
    import torch

    from starplat_b200 import _lib
    from starplat_b200.device import DeviceGraph

    from starplat_b200 import scheduler as S

    out = {"workload": name, "V": g.V, "E": g.E, "source": int(src)}
    with DeviceGraph.from_csr(g) as dg:
        dg.set_stream(stream)
        tuned(dg)
        dist = torch.empty(g.V, dtype=torch.int32, device="cuda")
        # fixed heuristic schedule (no model) against the learned one (model loaded):
        # warm both, then alternate single timed runs and take each one's median
        S.unload()  # also keeps the first sssp call from loading the shipped model
        timed(lambda: dg.sssp(src, out=dist), 1, max(1, warmup), stream)
        fixed = {"delta": dg.tune_get("sssp.last_delta"), "ctas_per_sm": dg.tune_get("sssp.last_ctas"),
                 "local": dg.tune_get("sssp.last_local")}
        d_fixed = dist.cpu().numpy()
        learned = S.load()
        timed(lambda: dg.sssp(src, out=dist), 1, max(1, warmup), stream)
        t_fixed, t_learned = [], []
        for _ in range(max(3, steps)):
            # the fixed heuristic through the knobs, so the loaded model (and its cached
            # choice for this graph) stays in place between the learned runs
            dg.tune_set("sssp.delta", fixed["delta"])
            dg.tune_set("sssp.ctas_per_sm", fixed["ctas_per_sm"])
            msf, resf = timed(lambda: dg.sssp(src, out=dist), 1, 0, stream)
            t_fixed.append(msf)
            dg.tune_set("sssp.delta", 0)
            dg.tune_set("sssp.ctas_per_sm", 0)
            ms1, res = timed(lambda: dg.sssp(src, out=dist), 1, 0, stream)
            t_learned.append(ms1)
            relaxed = dg.tune_get("sssp.last_relaxed")
        tuned(dg)
        msf, ms = statistics.median(t_fixed), statistics.median(t_learned)
        fixed.update({"ms": msf, "rounds": resf[0][1]})
        d = dist.cpu().numpy()
        reached = d < INT_MAX
        er = int(np.diff(g.indexofNodes)[reached].sum())
        nr = int(reached.sum())
        sched = {"learned": learned, "delta": dg.tune_get("sssp.last_delta"),
                 "ctas_per_sm": dg.tune_get("sssp.last_ctas"), "local": dg.tune_get("sssp.last_local")}
        msp, resp = timed(lambda: dg.sssp(src, out=dist, variant=_lib.SP_SSSP_PLAIN), 1, 0, stream)
        same = bool(np.array_equal(dist.cpu().numpy(), d) and np.array_equal(d_fixed, d))
        if REP is not None and REP.world > 1:
            # the same solve split over the GPUs by vertices (strong scaling): an all-to-all
            # of (vertex, distance) pairs per round, MIN reductions per bucket
            from starplat_b200.distributed import sssp_on_gpus

            dsplit = torch.empty(g.V, dtype=torch.int32, device="cuda")
            sssp_on_gpus(dg, REP, src, out=dsplit)
            REP.barrier()
            mss, ress = timed(lambda: sssp_on_gpus(dg, REP, src, out=dsplit), max(1, min(steps, 3)), 0, stream)
            mss = REP.max(mss)
            out["split"] = {"value": er / (mss / 1e3) / 1e9, "unit": "GTEPS", "ms": mss, "rounds": ress[-1][1],
                            "scaling": "strong", "same_distances": bool(np.array_equal(dsplit.cpu().numpy(), d)),
                            "parallelism": f"1-D vertex partition over {REP.world} GPUs (v mod {REP.world})"}
    fixed["value"] = er / (msf / 1e3) / 1e9
    out.update({"value": er / (ms / 1e3) / 1e9, "unit": "GTEPS", "ms": ms, "E_r": er, "reached": nr,
                "rounds": res[0][1], "relaxed_per_edge": round(relaxed / max(1, er), 3), "schedule": sched,
                "fixed_schedule": fixed,
                "plain": {"value": er / (msp / 1e3) / 1e9, "ms": msp, "rounds": resp[0][1]},
                "same_distances_all_forms": same,
                "roofline": roof(12 * er + 12 * g.V, ms, hbm)})
    if cpu:
        from oracle import oracle as O

        nt = O.num_threads()
        t = time.perf_counter()
        if cpu_mode == "omp":
            ref, rounds = O.sssp_omp(g.indexofNodes, g.edgeList, g.edgeLen, src, nthreads=nt)
            dt = time.perf_counter() - t
            out["cpu_baseline"] = {"value": er / dt / 1e9, "unit": "GTEPS", "cores": nt, "kind": "port",
                                   "sample": f"OpenMP fixed-point Compute_SSSP to convergence ({rounds} rounds, "
                                             f"{dt:.2f} s), full run"}
            oracle = "the OpenMP fixed-point Compute_SSSP (correct CAS atomicMin), full graph"
        else:
            ref = O.sssp(g.indexofNodes, g.edgeList, g.edgeLen, src)
            dt = time.perf_counter() - t
            out["cpu_baseline"] = {"value": er / dt / 1e9, "unit": "GTEPS", "cores": 1, "kind": "port",
                                   "sample": f"sequential Dijkstra ({dt:.2f} s), full run; the OpenMP fixed-point "
                                             "form needs thousands of full-vertex sweeps on this high-diameter grid"}
            oracle = "sequential Dijkstra, full graph"
        out["parity"] = {"dist_equal_oracle": bool(np.array_equal(d, ref)),
                         "mismatches": int((d != ref).sum()), "oracle": oracle, "tolerance": "bit-exact"}
    return out


def bench_bc(steps, warmup, stream, hbm, cpu, nsrc=256):
    from starplat_b200 import _lib
    from starplat_b200 import generators as G
    from starplat_b200.device import DeviceGraph

    g = G.rmat(20, 16, seed=1)
    srcs = G.pick_sources(g, 256, seed=20)[:nsrc]
    lab, ce = component_edges(g)
    er = ce[lab[srcs]]
    sum_er = int(er.sum())
    alg = int(16 * er.sum() + 32 * g.V * len(srcs))
    out = {"workload": f"bc rmat20 ef16 undirected seed1, {len(srcs)} sources", "V": g.V, "E": g.E,
           "sources": len(srcs),
           "sum_E_r": sum_er}
    with DeviceGraph.from_csr(g, with_weights=False) as dg:
        dg.set_stream(stream)
        tuned(dg)
        if REP is not None and REP.world > 1:
            # the sources split over the GPUs, one all-reduce of BC[V] (strong scaling)
            from starplat_b200.distributed import bc_on_gpus

            import torch

            bc_dev = torch.empty(g.V, dtype=torch.float32, device="cuda")  # summed in place by NCCL
            REP.barrier()
            ms, _ = timed(lambda: bc_on_gpus(dg, srcs, REP, out=bc_dev), steps, warmup, stream)
            ms = REP.max(ms)
            out["parallelism"] = f"sources split over {REP.world} GPUs, one all-reduce of BC[V]"
        else:
            ms, res = timed(lambda: dg.bc(srcs), steps, warmup, stream)
            bc_gpu = res[-1]
            # forward direction per level: the default (push at every level, or the level
            # model's choice when one is loaded) against the on-device frontier rule
            dflt = dg.tune_get("bc.dir")
            dg.tune_set("bc.dir", 1)
            ms_rule, _ = timed(lambda: dg.bc(srcs), 3, 1, stream)
            dg.tune_set("bc.dir", dflt)
            out["direction"] = {"default": {"bc.dir": dflt, "ms": ms},
                                "device_rule": {"bc.dir": 1, "ms": ms_rule},
                                "note": "bc.dir -1 = the library default (push at every level, or the level "
                                        "model when a model file is loaded); 1 = per-level push/pull rule on "
                                        "the device"}
            out["learned_vs_fixed"] = learned_vs_fixed(dg, "bc", lambda: dg.bc(srcs), stream)
        few = srcs[:8]
        msp, _ = timed(lambda: dg.bc(few, variant=_lib.SP_BC_PLAIN), 1, 0, stream)
    out.update({"value": sum_er / (ms / 1e3) / 1e9, "unit": "GTEPS", "ms": ms,
                "plain": {"value": float(er[:8].sum()) / (msp / 1e3) / 1e9, "ms_8_sources": msp,
                          "sample": "8 sources, one at a time"},
                "roofline": roof(alg, ms, hbm)})
    if cpu:
        from oracle import oracle as O

        nt = O.num_threads()
        t = time.perf_counter()
        O.bc_omp(g.indexofNodes, g.edgeList, srcs[:4], nthreads=nt)
        dt = time.perf_counter() - t
        out["cpu_baseline"] = {"value": float(er[:4].sum()) / dt / 1e9, "unit": "GTEPS", "cores": nt, "kind": "port",
                               "sample": f"OpenMP-form Compute_BC over 4 of the 256 sources ({dt:.2f} s), "
                                         "sampled: 4 of 256 sources"}
        if REP is None or REP.world == 1:
            t = time.perf_counter()
            ref = O.bc(g.indexofNodes, g.edgeList, srcs, nthreads=nt)
            excess, rel = bc_error(bc_gpu, ref)
            out["parity"] = {"oracle": f"FP64 Brandes with exact path counts over all {len(srcs)} sources "
                                       f"({time.perf_counter() - t:.1f} s on {nt} threads)",
                             "max_error_over_bar": excess, "max_rel_err_bc_ge_1": rel,
                             "tolerance": "per vertex |bc - ref| <= 1e-5 |ref| + 1e-9 max(1, max ref)",
                             "pass": excess <= 1.0}
    return out


def bench_bc_er(steps, warmup, stream, hbm, cpu, ngraphs=1000):
    from starplat_b200 import generators as G
    from starplat_b200.device import DeviceGraph

    t0 = time.time()
    gs = G.er_batch(1000, 1000, 50000, 8, 32, seed=11)[:ngraphs]
    voff = np.zeros(len(gs) + 1, np.int64)
    eoff = np.zeros(len(gs) + 1, np.int64)
    for k, g in enumerate(gs):
        voff[k + 1] = voff[k] + g.V
        eoff[k + 1] = eoff[k] + g.E
    V, E = int(voff[-1]), int(eoff[-1])
    off = np.empty(V + 1, np.int32)
    adj = np.empty(E, np.int32)
    srcs, soff, er_tot, er_k = [], [0], 0, []
    for k, g in enumerate(gs):
        off[voff[k]:voff[k + 1]] = g.indexofNodes[:-1] + eoff[k]
        adj[eoff[k]:eoff[k + 1]] = g.edgeList + voff[k]
        s = G.pick_sources(g, 16, seed=k)
        lab, ce = component_edges(g)
        er_k.append(int(ce[lab[s]].sum()))
        er_tot += er_k[-1]
        srcs.append(s + voff[k])
        soff.append(soff[-1] + len(s))
    off[V] = E
    srcs = np.concatenate(srcs).astype(np.int32)
    soff = np.array(soff, np.int32)
    voff32 = voff.astype(np.int32)
    gen_s = time.time() - t0
    alg = int(16 * er_tot + 32 * sum(g.V * 16 for g in gs))
    out = {"workload": f"bc {len(gs)} ER graphs, n log-uniform in [1e3, 5e4], degree U[8,32], 16 sources each, seed11",
           "V": V, "E": E, "sources": int(srcs.shape[0]), "sum_E_r": er_tot, "graph_gen_s": round(gen_s, 1)}
    with DeviceGraph(off, adj, None, off, adj) as dg:
        dg.set_stream(stream)
        ms, res = timed(lambda: dg.bc_graphs(voff32, soff, srcs), steps, warmup, stream)
        bc_all = res[-1]
    out.update({"value": er_tot / (ms / 1e3) / 1e9, "unit": "GTEPS", "ms": ms, "roofline": roof(alg, ms, hbm)})
    # plain form: one graph per call, one source at a time, on every 50th graph
    from starplat_b200 import _lib

    ms_plain, er_plain = 0.0, 0
    for k in range(0, len(gs), 50):
        with DeviceGraph.from_csr(gs[k], with_weights=False) as dgk:
            dgk.set_stream(stream)
            s_k = (srcs[soff[k]:soff[k + 1]] - voff32[k]).astype(np.int32)
            msk, _ = timed(lambda: dgk.bc(s_k, variant=_lib.SP_BC_PLAIN), 1, 1, stream)
        ms_plain += msk
        er_plain += er_k[k]
    out["plain"] = {"value": er_plain / (ms_plain / 1e3) / 1e9, "ms_sample": ms_plain,
                    "sample": "every 50th graph (20 of 1000), all 16 sources, one graph per call, "
                              "one source at a time"}
    if cpu:
        from oracle import oracle as O

        nt = O.num_threads()
        t = time.perf_counter()
        er_s = 0
        for k in range(0, len(gs), 50):
            g = gs[k]
            O.bc_omp(g.indexofNodes, g.edgeList, srcs[soff[k]:soff[k + 1]] - voff32[k], nthreads=nt)
            er_s += er_k[k]
        dt = time.perf_counter() - t
        out["cpu_baseline"] = {"value": er_s / dt / 1e9, "unit": "GTEPS", "cores": nt, "kind": "port",
                               "sample": f"OpenMP-form Compute_BC on 20 of the 1000 graphs, all 16 sources ({dt:.2f} s), "
                                         "sampled: every 50th graph"}
        worst, worst_rel = 0.0, 0.0
        for k in range(0, len(gs), 50):
            g = gs[k]
            ref = O.bc(g.indexofNodes, g.edgeList, srcs[soff[k]:soff[k + 1]] - voff32[k], nthreads=nt)
            e, r = bc_error(bc_all[voff32[k]:voff32[k + 1]], ref)
            worst, worst_rel = max(worst, e), max(worst_rel, r)
        out["parity"] = {"oracle": "FP64 Brandes with exact path counts on every 50th graph (20 of 1000), "
                                   "all 16 sources, against the same graphs' slices of the batched result",
                         "max_error_over_bar": worst, "max_rel_err_bc_ge_1": worst_rel,
                         "tolerance": "per vertex |bc - ref| <= 1e-5 |ref| + 1e-9 max(1, max ref)",
                         "pass": worst <= 1.0}
    return out


def bench_louvain(steps, warmup, stream, hbm, cpu):
    from starplat_b200 import generators as G
    from starplat_b200.device import DeviceGraph

    g = G.sbm(1 << 20, 256, exponent=2.0, avg_degree=32, p_in=0.8, seed=1)
    out = {"workload": "louvain sbm 1048576 vertices, 256 blocks (power-law sizes, exponent 2), degree 32, "
                       "80% intra, unit weights, seed1", "V": g.V, "E": g.E}
    res = {}
    with DeviceGraph.from_csr(g, with_weights=False) as dg:
        dg.set_stream(stream)

        def run():
            q, _, lv = dg.louvain(None, 1e-4)
            res["q"], res["levels"], res["sweeps"] = q, lv, dg.last_louvain_sweeps
            return q

        ms, _ = timed(run, steps, warmup, stream)
        out["variant"] = {"last_level_candidate": dg.tune_get("lv.last_variant"),
                          "note": "-1 = the fixed CTA-bin table; the shipped per-level model loads on first use"}
        out["learned_vs_fixed"] = learned_vs_fixed(dg, "louvain", lambda: dg.louvain(None, 1e-4), stream)

        def run_plain():
            from starplat_b200 import _lib

            q, _, _ = dg.louvain(None, 1e-4, variant=_lib.SP_LV_PLAIN)
            res["pq"], res["psweeps"] = q, dg.last_louvain_sweeps

        msp, _ = timed(run_plain, 1, 0, stream)
    sweeps = res["sweeps"]
    out.update({"value": g.E * sweeps / (ms / 1e3) / 1e9, "unit": "GTEPS", "ms": ms, "modularity": res["q"],
                "levels": res["levels"], "sweeps": sweeps,
                "plain": {"value": g.E * res["psweeps"] / (msp / 1e3) / 1e9, "ms": msp, "modularity": res["pq"],
                          "sweeps": res["psweeps"],
                          "sample": "one full run, one thread per vertex, O(deg^2) neighbour rescans"},
                "roofline": roof((12 * g.E + 16 * g.V) * sweeps, ms, hbm)})
    if cpu:
        from oracle import oracle as O

        t = time.perf_counter()
        q, _, lv, sw = O.louvain(g.indexofNodes, g.edgeList, None, 1e-4, with_sweeps=True)
        dt = time.perf_counter() - t
        out["cpu_baseline"] = {"value": g.E * sw / dt / 1e9, "unit": "GTEPS", "cores": 1, "kind": "port",
                               "modularity": q, "sample": f"sequential restatement of the DSL, full run "
                                                          f"({sw} sweeps, {lv} levels, {dt:.2f} s)"}
        out["modularity_minus_cpu"] = res["q"] - q
    fx = os.path.join(ROOT, "tests", "golden", "reference_gpu", "louvain.json")
    if os.path.exists(fx):
        ref = json.load(open(fx)).get("sbm1m")
        if ref:
            out["parity"] = {"oracle": "modularity (FP64) of the partition of the reference's own CUDA Louvain "
                                       "(communitydetection_sequential_allocation.cu) on this graph, run on a B200 "
                                       "and committed as a fixture",
                             "reference_q": ref["reference_q"], "q_minus_reference": res["q"] - ref["reference_q"],
                             "tolerance": "q >= reference_q - 1e-3; where both stop in the same optimum, also "
                                          "q <= reference_q + 1e-3",
                             "same_optimum": abs(res["q"] - ref["reference_q"]) <= 1e-3,
                             "reference_communities": ref.get("reference_communities"),
                             "note": "Louvain is order dependent; the two may stop in different optima",
                             "pass": res["q"] >= ref["reference_q"] - 1e-3}
    return out


def bench_ingest(steps, warmup, cpu):
    """Text edge list -> device mirror through sp_graph_load_text, wall time of the call
    (file read from the page cache, host tokenising, copy, device sort / merge / both
    CSRs / check). The CPU figure is the reference's own graph::parseGraph (compiled
    from graph.hpp) on an R-MAT 16 file of the same shape, when that build is present."""
    import shutil
    import tempfile

    import torch

    from starplat_b200 import generators as G
    from starplat_b200.device import DeviceGraph

    d = tempfile.mkdtemp(prefix="sp_ingest_")
    try:
        g = G.rmat(20, 16, seed=20, directed=True)
        w = G.hash_weights(g, 20, 1, 100, False)
        path = os.path.join(d, "rmat20.txt")
        nbytes = G.write_edgelist(g, path, w)
        times, E = [], 0
        for i in range(warmup + steps):
            t = time.perf_counter()
            dg = DeviceGraph.load_text(path)
            torch.cuda.synchronize()
            dt = time.perf_counter() - t
            E = dg.E
            dg.free()
            if i >= warmup:
                times.append(dt)
        ms = 1e3 * statistics.median(times)
        out = {"workload": "text edge list of directed R-MAT 20 ef16 (seed 20), weights U[1,100], "
                           "one 'src dst weight' line per edge", "lines": int(g.E), "bytes": int(nbytes),
               "V": int(g.V), "E": int(E), "value": g.E / (ms / 1e3) / 1e6, "unit": "M edge lines/s", "ms": ms,
               "text_gb_per_s": nbytes / (ms / 1e3) / 1e9}
        if cpu:
            from oracle import oracle as O

            if O.ref_lib() is not None:
                g16 = G.rmat(16, 16, seed=20, directed=True)
                p16 = os.path.join(d, "rmat16.txt")
                G.write_edgelist(g16, p16, G.hash_weights(g16, 20, 1, 100, False))
                t = time.perf_counter()
                O.ref_parse_graph(p16)
                dt = time.perf_counter() - t
                out["cpu_baseline"] = {"value": g16.E / dt / 1e6, "unit": "M edge lines/s",
                                       "cores": O.num_threads(), "kind": "reference",
                                       "sample": f"graph::parseGraph on the R-MAT 16 file ({g16.E} lines, {dt:.2f} s; "
                                                 "its line reading is sequential, its sorts use OpenMP)"}
        return out
    finally:
        shutil.rmtree(d, ignore_errors=True)


EXTRAS = ("tc_rmat16", "sssp_rmat23", "sssp_grid4096", "bc_rmat20", "bc_er1000", "louvain_sbm1m", "ingest_rmat20",
          "centrality", "update_rmat20")


def bench_centrality(steps, warmup, stream, hbm, cpu):
    """Algorithms on the same kernels: per-vertex triangle counts (staticClusteringCoeff)
    on the TC graph, and closeness (Compute_CC_Unweighted over BC's graph and sources,
    Compute_CC weighted over 16 of them)."""
    from starplat_b200 import _lib
    from starplat_b200 import generators as G
    from starplat_b200.device import DeviceGraph

    out = {}
    g = G.rmat(16, 16, seed=1)
    m = g.E // 2
    with DeviceGraph.from_csr(g, with_weights=False) as dg:
        dg.set_stream(stream)
        tuned(dg)
        lcc_sharded = REP is not None and REP.world > 1
        if lcc_sharded:
            # anchor parts over the GPUs, one all-reduce of the int32 counts (strong scaling)
            from starplat_b200.distributed import clustering_coeff_on_gpus

            import torch

            cf_dev = torch.empty(g.V, dtype=torch.int32, device="cuda")
            REP.barrier()
            ms, _ = timed(lambda: clustering_coeff_on_gpus(dg, REP, out=cf_dev), steps, warmup, stream)
            res = [cf_dev.cpu().numpy()]
            ms = REP.max(ms)
        else:
            ms, res = timed(lambda: dg.clustering_coeff(), steps, warmup, stream)
        msp, _ = timed(lambda: dg.clustering_coeff(variant=_lib.SP_TC_PLAIN), 1, 1, stream)
        cf = res[0]
    lcc = {"workload": "clustering_coeff rmat16 ef16 undirected seed1", "value": m / (ms / 1e3) / 1e9,
           "unit": "GTEPS", "ms": ms, "triangle_incidences": int(cf.astype(np.int64).sum()),
           "plain": {"value": m / (msp / 1e3) / 1e9, "ms": msp}}
    if lcc_sharded:
        lcc["parallelism"] = f"anchor parts over {REP.world} GPUs, one all-reduce of cf[V]"
    if cpu:
        from oracle import oracle as O

        nt = O.num_threads()
        t = time.perf_counter()
        ref = O.lcc(g.indexofNodes, g.edgeList, nthreads=nt)
        dt = time.perf_counter() - t
        lcc["same_as_oracle"] = bool(np.array_equal(ref, cf))
        lcc["cpu_baseline"] = {"value": m / dt / 1e9, "unit": "GTEPS", "cores": nt, "kind": "port",
                               "sample": f"OpenMP clustering_coeff loop, binary-search form, full graph ({dt:.2f} s)"}
    out["clustering_coeff_rmat16"] = lcc

    g = G.rmat(20, 16, seed=1)
    g.edgeLen = G.hash_weights(g, 20, 1, 100, True)
    srcs = np.sort(G.pick_sources(g, 256, seed=20)).astype(np.int32)
    lab, ce = component_edges(g)
    er = ce[lab[srcs]].astype(np.int64)
    w16 = srcs[:16]
    sharded = REP is not None and REP.world > 1
    with DeviceGraph.from_csr(g) as dg:
        dg.set_stream(stream)
        tuned(dg)
        if sharded:
            # the sources split over the GPUs, one all-reduce of CC[V] (strong scaling)
            from starplat_b200.distributed import closeness_on_gpus

            import torch

            cu_dev = torch.empty(g.V, dtype=torch.float32, device="cuda")
            cw_dev = torch.empty(g.V, dtype=torch.float32, device="cuda")
            REP.barrier()
            msu, _ = timed(lambda: closeness_on_gpus(dg, srcs, REP, weighted=False, out=cu_dev), max(1, steps // 2),
                           1, stream)
            msw, _ = timed(lambda: closeness_on_gpus(dg, w16, REP, out=cw_dev), max(1, steps // 2), 1, stream)
            resu, resw = [cu_dev.cpu().numpy()], [cw_dev.cpu().numpy()]
            msu, msw = REP.max(msu), REP.max(msw)
        else:
            msu, resu = timed(lambda: dg.closeness_unweighted(srcs), max(1, steps // 2), 1, stream)
            msw, resw = timed(lambda: dg.closeness(w16), max(1, steps // 2), 1, stream)
    cu = {"workload": "closeness unweighted rmat20 ef16 undirected seed1, 256 sources",
          "value": int(er.sum()) / (msu / 1e3) / 1e9, "unit": "GTEPS", "ms": msu}
    cw = {"workload": "closeness weighted rmat20 ef16 undirected seed1, w U[1,100], 16 sources",
          "value": int(er[:16].sum()) / (msw / 1e3) / 1e9, "unit": "GTEPS", "ms": msw}
    if sharded:
        cu["parallelism"] = cw["parallelism"] = f"sources split over {REP.world} GPUs, one all-reduce of CC[V]"
    if cpu:
        from oracle import oracle as O

        t = time.perf_counter()
        refw = O.closeness(g.indexofNodes, g.edgeList, g.edgeLen, w16[:4])
        dt = time.perf_counter() - t
        cw["same_as_oracle_on_sample"] = bool(np.array_equal(refw[w16[:4]], resw[0][w16[:4]]))
        cw["cpu_baseline"] = {"value": int(er[:4].sum()) / dt / 1e9, "unit": "GTEPS", "cores": 1, "kind": "port",
                              "sample": f"sequential Dijkstra from 4 of the 16 sources ({dt:.2f} s)"}
        t = time.perf_counter()
        refu = O.closeness_unweighted(g.indexofNodes, g.edgeList, srcs[:8])
        dt = time.perf_counter() - t
        cu["same_as_oracle_on_sample"] = bool(np.array_equal(refu[srcs[:8]], resu[0][srcs[:8]]))
        cu["cpu_baseline"] = {"value": int(er[:8].sum()) / dt / 1e9, "unit": "GTEPS", "cores": 1, "kind": "port",
                              "sample": f"sequential BFS from 8 of the 256 sources ({dt:.2f} s)"}
    out["closeness_unweighted_rmat20"] = cu
    out["closeness_rmat20"] = cw
    return out


def bench_update(steps, warmup, stream, cpu, nupd=1 << 20):
    """One batch of nupd edge updates (sp_graph_update) on directed R-MAT 20 ef16 with
    weights: half deletions of existing edges, half additions of random edges. Timed
    from host arrays to the rebuilt device CSR (M updates / s)."""
    from starplat_b200 import generators as G
    from starplat_b200.device import DeviceGraph

    g = G.rmat(20, 16, seed=7, directed=True)
    g.edgeLen = G.hash_weights(g, 7, 1, 100, False)
    rng = np.random.default_rng(20)
    src_all = np.repeat(np.arange(g.V, dtype=np.int32), np.diff(g.indexofNodes))
    pick = rng.choice(g.E, nupd // 2, replace=False)
    ds, dd = src_all[pick], g.edgeList[pick]
    as_, ad = rng.integers(0, g.V, (2, nupd - nupd // 2)).astype(np.int32)
    types = "d" * (nupd // 2) + "a" * (nupd - nupd // 2)
    src = np.concatenate([ds, as_]).astype(np.int32)
    dst = np.concatenate([dd, ad]).astype(np.int32)
    w = rng.integers(1, 100, nupd).astype(np.int32)
    times = []
    for k in range(warmup + steps):
        with DeviceGraph.from_csr(g, with_reverse=False) as dg:
            dg.set_stream(stream)
            torch_sync()
            t = time.perf_counter()
            dg.update(types, src, dst, w)
            torch_sync()
            if k >= warmup:
                times.append(time.perf_counter() - t)
            e_after = dg.E
    ms = 1e3 * statistics.median(times)
    out = {"workload": f"update rmat20 ef16 directed seed7, {nupd} updates (half deletions of existing edges)",
           "value": nupd / (ms / 1e3) / 1e6, "unit": "M updates/s", "ms": ms, "E_before": g.E, "E_after": e_after}
    # DynSSSP batches of 4096 added edges: resume from the old distances (sp_sssp_dynamic)
    # against the same update followed by a full solve; both rebuild the CSR
    import torch

    source = int(G.pick_sources(g, 1, seed=20)[0])
    nb = 4096
    res_t, full_t, same = [], [], True
    with DeviceGraph.from_csr(g, with_reverse=False) as da, DeviceGraph.from_csr(g, with_reverse=False) as db:
        da.set_stream(stream)
        db.set_stream(stream)
        dist = torch.empty(g.V, dtype=torch.int32, device="cuda")
        dfull = torch.empty(g.V, dtype=torch.int32, device="cuda")
        da.sssp(source, out=dist)
        for k in range(warmup + steps):
            bs = rng.integers(0, g.V, nb).astype(np.int32)
            bd = rng.integers(0, g.V, nb).astype(np.int32)
            bw = rng.integers(1, 100, nb).astype(np.int32)
            torch_sync()
            t = time.perf_counter()
            resumed = da.sssp_dynamic("a" * nb, bs, bd, bw, source, dist)
            torch_sync()
            t1 = time.perf_counter()
            db.update("a" * nb, bs, bd, bw)
            db.sssp(source, out=dfull)
            torch_sync()
            t2 = time.perf_counter()
            if k >= warmup:
                res_t.append(t1 - t)
                full_t.append(t2 - t1)
            same = same and resumed and bool(torch.equal(dist, dfull))
    out["sssp_dynamic"] = {"workload": f"{nb} added edges per batch, source {source}",
                           "resume_ms": 1e3 * statistics.median(res_t),
                           "update_and_full_solve_ms": 1e3 * statistics.median(full_t),
                           "same_distances": same}
    # DynSSSP batches of deletions of edges the graph holds (64 or 4096 per batch): the
    # decremental pass through parents (or a new solve when it would reset > V / 4)
    # against the same update followed by a full solve
    src_of = np.repeat(np.arange(g.V, dtype=np.int32), np.diff(g.indexofNodes))
    out["sssp_dynamic_deletions"] = {}
    gd = G.grid(1024, 1024)  # high diameter: a full solve takes hundreds of rounds
    gd.edgeLen = G.hash_weights(gd, 1024, 1, 1000, True)
    gd_src = np.repeat(np.arange(gd.V, dtype=np.int32), np.diff(gd.indexofNodes))
    for key, gg, gsrc, sv, nd in (("rmat20_64", g, src_of, source, 64), ("rmat20_4096", g, src_of, source, 4096),
                                  ("grid1024_64", gd, gd_src, 3 * gd.V // 7, 64)):
        rep_t, full_t, same, paths, marked = [], [], True, [], []
        with DeviceGraph.from_csr(gg, with_reverse=False) as da, DeviceGraph.from_csr(gg, with_reverse=False) as db:
            da.set_stream(stream)
            db.set_stream(stream)
            dist = torch.empty(gg.V, dtype=torch.int32, device="cuda")
            dfull = torch.empty(gg.V, dtype=torch.int32, device="cuda")
            _, first_rounds = da.sssp(sv, out=dist)
            da.tune_set("sssp.repair", 1)  # time the repair itself; the default picks by rounds
            for k in range(warmup + steps):
                pick = rng.choice(gg.E, nd, replace=False)  # edges of the original graph (some already gone)
                bs, bd = gsrc[pick], gg.edgeList[pick].astype(np.int32)
                torch_sync()
                t = time.perf_counter()
                da.sssp_dynamic("d" * nd, bs, bd, None, sv, dist)
                torch_sync()
                t1 = time.perf_counter()
                paths.append(da.tune_get("sssp.last_incremental"))
                marked.append(da.tune_get("sssp.last_marked"))
                db.update("d" * nd, bs, bd)
                db.sssp(sv, out=dfull)
                torch_sync()
                t2 = time.perf_counter()
                if k >= warmup:
                    rep_t.append(t1 - t)
                    full_t.append(t2 - t1)
                same = same and bool(torch.equal(dist, dfull))
        out["sssp_dynamic_deletions"][key] = {
            "workload": f"{nd} deleted edges per batch, source {sv}", "ms": 1e3 * statistics.median(rep_t),
            "update_and_full_solve_ms": 1e3 * statistics.median(full_t), "batches_repaired": paths.count(2),
            "vertices_reset_median": statistics.median(marked), "V": gg.V, "first_solve_rounds": first_rounds,
            "default_policy": "repair" if first_rounds >= 32 else "solve again",
            "batches_solved_again": paths.count(0), "same_distances": same}
    # DynPR batches of 4096 added edges: PageRank from the previous ranks
    # (sp_pagerank_dynamic) against the same update followed by PageRank from 1/V
    warm_t, cold_t, warm_it, cold_it, l1 = [], [], [], [], 0.0
    with DeviceGraph.from_csr(g, with_reverse=False) as da, DeviceGraph.from_csr(g, with_reverse=False) as db:
        da.set_stream(stream)
        db.set_stream(stream)
        ranks = torch.empty(g.V, dtype=torch.float32, device="cuda")
        cold = torch.empty(g.V, dtype=torch.float32, device="cuda")
        da.pagerank(out=ranks)
        for k in range(warmup + steps):
            bs, bd = rng.integers(0, g.V, (2, nb)).astype(np.int32)
            torch_sync()
            t = time.perf_counter()
            _, itw, _ = da.pagerank_dynamic("a" * nb, bs, bd, None, ranks)
            torch_sync()
            t1 = time.perf_counter()
            db.update("a" * nb, bs, bd)
            _, itc, _ = db.pagerank(out=cold)
            torch_sync()
            t2 = time.perf_counter()
            if k >= warmup:
                warm_t.append(t1 - t)
                cold_t.append(t2 - t1)
                warm_it.append(itw)
                cold_it.append(itc)
            l1 = max(l1, float((ranks.double() - cold.double()).abs().sum()))
    # DynTC batches of 2048 undirected updates given in both directions (half deletions of
    # edges of the original graph, half random additions) on undirected R-MAT 20:
    # triangles through the batch only (sp_tc_dynamic) against the same update and a recount
    gu = G.rmat(20, 16, seed=1)
    src_u = np.repeat(np.arange(gu.V, dtype=np.int32), np.diff(gu.indexofNodes))
    inc_t, upd_t, rec_t, same_tc = [], [], [], True
    with DeviceGraph.from_csr(gu, with_weights=False) as da, DeviceGraph.from_csr(gu, with_weights=False) as db:
        da.set_stream(stream)
        db.set_stream(stream)
        count = da.tc()
        for k in range(warmup + steps):
            pick = rng.choice(gu.E, nb // 4, replace=False)
            xs, xd = src_u[pick], gu.edgeList[pick]
            ys, yd = rng.integers(0, gu.V, (2, nb // 4)).astype(np.int32)
            bs = np.concatenate([xs, xd, ys, yd]).astype(np.int32)
            bd = np.concatenate([xd, xs, yd, ys]).astype(np.int32)
            bt = "d" * (nb // 2) + "a" * (nb // 2)
            torch_sync()
            t = time.perf_counter()
            count, inc = da.tc_dynamic(bt, bs, bd, None, count)
            torch_sync()
            t1 = time.perf_counter()
            db.update(bt, bs, bd)
            torch_sync()
            t2 = time.perf_counter()
            full = db.tc()
            torch_sync()
            t3 = time.perf_counter()
            if k >= warmup:
                inc_t.append(t1 - t)
                upd_t.append(t2 - t1)
                rec_t.append(t3 - t2)
            same_tc = same_tc and inc and count == full
    out["tc_dynamic"] = {"workload": f"tc rmat20 ef16 undirected seed1, {nb // 2} undirected updates per batch",
                         "incremental_ms": 1e3 * statistics.median(inc_t),
                         "update_ms": 1e3 * statistics.median(upd_t),
                         "recount_ms": 1e3 * statistics.median(rec_t),
                         "triangles": count, "same_count": same_tc}
    out["pagerank_dynamic"] = {"workload": f"{nb} added edges per batch, beta 1e-6",
                               "warm_ms": 1e3 * statistics.median(warm_t),
                               "update_and_cold_ms": 1e3 * statistics.median(cold_t),
                               "warm_iterations": statistics.median(warm_it),
                               "cold_iterations": statistics.median(cold_it),
                               "max_l1_warm_vs_cold": l1}
    if cpu:
        # the same batch on the host: edge keys, deletions by search, additions merged
        t = time.perf_counter()
        keys = (src_all.astype(np.int64) << 32) | g.edgeList.astype(np.int64)
        dk = np.unique((ds.astype(np.int64) << 32) | dd.astype(np.int64))
        keep = np.ones(g.E, bool)
        pos = np.searchsorted(keys, dk)
        hit = pos < g.E
        hit[hit] = keys[pos[hit]] == dk[hit]
        keep[pos[hit]] = False
        allk = np.concatenate([keys[keep], (as_.astype(np.int64) << 32) | ad.astype(np.int64)])
        allw = np.concatenate([g.edgeLen[keep], w[nupd // 2:]]).astype(np.int64)
        uk, inv = np.unique(allk, return_inverse=True)
        uw = np.zeros(uk.shape[0], np.int64)
        np.add.at(uw, inv, allw)
        dt = time.perf_counter() - t
        out["same_edge_count_as_host"] = bool(uk.shape[0] == e_after)
        out["cpu_baseline"] = {"value": nupd / dt / 1e6, "unit": "M updates/s", "cores": 1, "kind": "port",
                               "sample": f"numpy sort-and-merge of the same batch ({dt:.2f} s)"}
    return out


def torch_sync():
    import torch

    torch.cuda.synchronize()


def run_extras(want, args, stream, hbm, cpu_ok):
    from starplat_b200 import generators as G

    extras = {}
    ks, kw = max(1, min(args.steps, 5)), 2

    def guarded(name, fn):
        try:
            extras[name] = fn()
        except Exception as e:  # report, keep the headline line
            extras[name] = {"error": f"{type(e).__name__}: {e}"}

    if "tc_rmat16" in want:
        guarded("tc_rmat16", lambda: bench_tc(ks, kw, stream, hbm, cpu_ok))
    if "sssp_rmat23" in want:
        def _s1():
            gs = G.rmat(23, 16, seed=1, directed=True)
            gs.edgeLen = G.hash_weights(gs, 23, 1, 100, False)
            src = int(G.pick_sources(gs, 1, seed=23)[0])
            return bench_sssp("sssp rmat23 ef16 directed seed1, w U[1,100]", gs, src, ks, kw, stream, hbm,
                              cpu_ok, "omp")
        guarded("sssp_rmat23", _s1)
    if "sssp_grid4096" in want:
        def _s2():
            gg = G.grid(4096, 4096)
            gg.edgeLen = G.hash_weights(gg, 4096, 1, 1000, True)
            src = int(np.random.default_rng(4096).integers(0, gg.V))
            return bench_sssp("sssp grid 4096x4096 4-neighbour, w U[1,1000] symmetric", gg, src, max(1, ks // 2),
                              1, stream, hbm, cpu_ok, "dijkstra")
        guarded("sssp_grid4096", _s2)
    if "bc_rmat20" in want:
        guarded("bc_rmat20", lambda: bench_bc(max(1, ks // 2), 1, stream, hbm, cpu_ok, args.sources))
    if "bc_er1000" in want:
        guarded("bc_er1000", lambda: bench_bc_er(max(1, ks // 2), 1, stream, hbm, cpu_ok, args.graphs))
    if "louvain_sbm1m" in want:
        guarded("louvain_sbm1m", lambda: bench_louvain(max(1, ks // 2), 1, stream, hbm, cpu_ok))
    if "ingest_rmat20" in want:
        guarded("ingest_rmat20", lambda: bench_ingest(max(1, ks // 2), 1, cpu_ok))
    if "centrality" in want:
        guarded("centrality", lambda: bench_centrality(ks, kw, stream, hbm, cpu_ok))
    if "update_rmat20" in want:
        guarded("update_rmat20", lambda: bench_update(ks, kw, stream, cpu_ok))
    return extras


# ----------------------------------------------------------------------------- main

def main():
    global PR_SCALE, REP
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-parity", action="store_true", help="skip the checks against the oracle")
    ap.add_argument("--quick", action="store_true",
                    help="PageRank device-resident timing only (no other legs): for profiler runs")
    ap.add_argument("--only", default="", help="comma list of extra workloads (default: all)")
    ap.add_argument("--no-extras", action="store_true", help="headline PageRank only")
    ap.add_argument("--scale", type=int, default=PR_SCALE, help="R-MAT scale of the PageRank graph")
    ap.add_argument("--tune", action="append", default=[], help="schedule knob key=value (sp_tune_set)")
    ap.add_argument("--graphs", type=int, default=1000,
                    help="ER graphs of the bc_er1000 workload (1000 = the config; fewer for profiler runs)")
    ap.add_argument("--sources", type=int, default=256,
                    help="BC sources of the bc_rmat20 workload (256 = the config; fewer for profiler runs)")
    ap.add_argument("--algo-only", default="", help="run only these extra workloads (comma list), no headline: "
                                                     "for profiler runs")
    args = ap.parse_args()
    PR_SCALE = args.scale
    args.warmup = max(3, args.warmup)

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank)

    import torch

    from starplat_b200.replicas import Replicas

    torch.cuda.set_device(local)
    rep = Replicas("nccl" if world > 1 else None)
    REP = rep
    barrier, max_over_ranks = rep.barrier, rep.max

    from starplat_b200 import _lib
    from starplat_b200.device import DeviceGraph

    if args.algo_only:
        for kv in args.tune:
            k, v = kv.split("=")
            TUNE.append((k, int(v)))
        res = run_extras(set(args.algo_only.split(",")), args, torch.cuda.current_stream(), peaks()[0], False)
        if rank == 0:
            print(json.dumps({"algo_only": True, "algorithms": res}), flush=True)
        rep.close()
        return

    g, gen_s = pr_graph()
    V, E = g.V, g.E
    stream = torch.cuda.current_stream()
    dg = DeviceGraph.from_csr(g, with_weights=False)
    dg.set_stream(stream)
    for kv in args.tune:
        k, v = kv.split("=")
        TUNE.append((k, int(v)))
    tuned(dg)
    out = torch.empty(V, dtype=torch.float32, device="cuda")

    for _ in range(args.warmup):
        _, iters, _ = dg.pagerank(BETA, DELTA, MAX_ITER, out=out)

    # ---- device-resident timing
    barrier()
    torch.cuda.synchronize()
    clk = Clocks(local)
    l0 = _lib.launch_count()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    it_total = 0
    for _ in range(args.steps):
        _, iters, _ = dg.pagerank(BETA, DELTA, MAX_ITER, out=out)
        it_total += iters
    ev1.record(stream)
    torch.cuda.synchronize()
    barrier()
    clocks = clk.stop()
    launches = _lib.launch_count() - l0
    ms = max_over_ranks(ev0.elapsed_time(ev1))
    value = rep.sum(E * it_total) / (ms / 1e3) / 1e9  # every rank's edges over the slowest rank's time
    if args.quick:
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": value, "unit": "GTEPS", "quick": True, "V": V, "E": E,
                              "iterations": it_total // args.steps, "ms_per_step": ms / args.steps}), flush=True)
        dg.free()
        rep.close()
        return

    hbm, hbm_kind = peaks()

    # ---- parity of the timed result: L1 against FP64 PageRank at the same iteration count
    parity = None
    if rank == 0 and not args.no_parity:
        from oracle import oracle as O

        t = time.perf_counter()
        exact, _, _ = O.pagerank(g.indexofNodes, g.rev_indexofNodes, g.srcList, 0.0, DELTA, iters,
                                 nthreads=O.num_threads())
        l1 = float(np.abs(out.cpu().numpy().astype(np.float64) - exact).sum())
        parity = {"pagerank_l1_vs_fp64": l1, "tolerance": 1e-6, "pass": l1 < 1e-6, "iterations": iters,
                  "oracle": f"FP64 Jacobi PageRank, the same {iters} iterations ({time.perf_counter() - t:.1f} s)"}

    # ---- kernel roofline: average iteration-kernel time from two fixed-iteration runs
    def timed_fixed(n, reps=3):
        best = None
        for _ in range(reps):
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            dg.pagerank(0.0, DELTA, n, out=out)
            b.record(stream)
            torch.cuda.synchronize()
            t = a.elapsed_time(b)
            best = t if best is None else min(best, t)
        return best

    n1, n2 = 10, 60
    t1, t2 = timed_fixed(n1), timed_fixed(n2)
    per_launch_ms = (t2 - t1) / (n2 - n1)
    alg_bytes = 8 * E + 16 * V
    achieved = alg_bytes / (per_launch_ms / 1e3) / 1e9
    roofline = {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                "traffic": None, "peak_kind": hbm_kind, "kernel": "sp::pr::k_phase<1>",
                "alg_bytes_per_launch": alg_bytes, "avg_launch_ms": per_launch_ms}
    tf = os.path.join(ROOT, "profiles", "pagerank_rmat22_traffic.json")
    if os.path.exists(tf):
        try:
            roofline["traffic"] = json.load(open(tf)).get("traffic_bytes_per_launch")
        except Exception:
            pass

    # kernel-variant choice of the iteration: fixed defaults against the trained network
    pr_variants = None
    if rank == 0 and world == 1:
        pr_variants = learned_vs_fixed(dg, "pagerank", lambda: dg.pagerank(BETA, DELTA, MAX_ITER, out=out), stream)

    # plain (generated-code form) PageRank for comparison
    msp, resp = timed(lambda: dg.pagerank(BETA, DELTA, MAX_ITER, out=out, variant=_lib.SP_PR_PLAIN), 1, 1, stream)
    pr_plain = {"value": E * resp[0][1] / (msp / 1e3) / 1e9, "ms_per_step": msp, "iterations": resp[0][1]}

    # ---- end to end through the C ABI with host buffers (pinned), every step
    # what the drop-in header uploads: the forward CSR (PageRank builds its relabelled
    # reverse rows on the device)
    pin = {k: torch.from_numpy(getattr(g, k)).pin_memory() for k in ("indexofNodes", "edgeList")}
    host_out = torch.empty(V, dtype=torch.float32).pin_memory()
    h2d = sum(t.numel() * 4 for t in pin.values())
    d2h = V * 4

    def e2e_step():
        with DeviceGraph(pin["indexofNodes"].numpy(), pin["edgeList"].numpy()) as hg:
            _, n, _ = hg.pagerank(BETA, DELTA, MAX_ITER, out=host_out.numpy())
        return n

    e2e_step()
    barrier()
    torch.cuda.synchronize()
    e_steps = max(1, min(args.steps, 5))
    t0 = time.perf_counter()
    e_it = 0
    for _ in range(e_steps):
        e_it += e2e_step()
    torch.cuda.synchronize()
    e_s = max_over_ranks(time.perf_counter() - t0)
    e2e = {"value": rep.sum(E * e_it) / e_s / 1e9, "unit": "GTEPS", "h2d_bytes_per_step": h2d,
           "d2h_bytes_per_step": d2h, "ms_per_step": 1e3 * e_s / e_steps}

    # ---- N > 1: the same graph split over the ranks by vertices (strong scaling), one
    # all-gather of the contrib blocks and one all-reduce of the diff per iteration
    split = None
    if world > 1:
        from starplat_b200.distributed import pagerank_on_gpus

        split_out = torch.empty(V, dtype=torch.float32, device="cuda")
        for _ in range(2):
            pagerank_on_gpus(dg, rep, BETA, DELTA, MAX_ITER, out=split_out)
        barrier()
        torch.cuda.synchronize()
        s0 = torch.cuda.Event(enable_timing=True)
        s1 = torch.cuda.Event(enable_timing=True)
        s0.record(stream)
        sp_steps = max(1, min(args.steps, 5))
        sp_it = 0
        for _ in range(sp_steps):
            _, it_s, _ = pagerank_on_gpus(dg, rep, BETA, DELTA, MAX_ITER, out=split_out)
            sp_it += it_s
        s1.record(stream)
        torch.cuda.synchronize()
        sp_ms = max_over_ranks(s0.elapsed_time(s1)) / sp_steps
        split = {"workload": f"pagerank rmat{PR_SCALE} split over {world} GPUs by vertices",
                 "value": E * (sp_it / sp_steps) / (sp_ms / 1e3) / 1e9, "unit": "GTEPS", "ms_per_step": sp_ms,
                 "iterations": sp_it // sp_steps, "scaling": "strong",
                 "parallelism": f"1-D vertex partition over {world} GPUs: NCCL all-gather of contrib blocks and "
                                "all-reduce of the diff per iteration, stop test on the device"}
        if rank == 0 and not args.no_parity:
            from oracle import oracle as O

            exact, _, _ = O.pagerank(g.indexofNodes, g.rev_indexofNodes, g.srcList, 0.0, DELTA, it_s,
                                     nthreads=O.num_threads())
            split["parity"] = {"pagerank_l1_vs_fp64": float(np.abs(split_out.cpu().numpy().astype(np.float64)
                                                                   - exact).sum()), "tolerance": 1e-6}

    cpu_ok = rank == 0 and world == 1 and not args.no_cpu_baseline
    cpu = cpu_pagerank(g, 3) if cpu_ok else None
    if cpu:
        cpu["sample"] += "; sampled: 3 of the run's iterations"
    cfg = pr_config(g, world)
    dg.free()
    del g

    # ---- the other algorithms of the metric
    extras = {}
    if not args.no_extras:
        want = set(filter(None, args.only.split(","))) or set(EXTRAS)
        extras = run_extras(want, args, stream, hbm, cpu_ok)

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "GTEPS", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": cfg, "iterations": it_total // args.steps, "graph_gen_s": round(gen_s, 2),
                "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches, "clocks": clocks,
                "parity": parity, "plain": pr_plain, "learned_vs_fixed": pr_variants, "algorithms": extras}
        if split:
            line["pagerank_split"] = split
        print(json.dumps(line), flush=True)
    rep.close()


if __name__ == "__main__":
    main()
