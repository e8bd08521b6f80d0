"""Benchmark: GTEPS of the static-graph hot path on B200.

Headline workload (one JSON line on rank 0): PageRank, pull over the reverse CSR,
on a directed R-MAT graph, scale 22 (4,194,304 vertices), edge factor 16,
a/b/c/d = .57/.19/.19/.05, seed 1, damping 0.85, L1 threshold 1e-6, maxIter 100.
A step is one full PageRank call (all iterations until convergence); GTEPS =
E * iterations / time.

  value       device-resident CSR (uploaded before timing), events on the stream
  e2e         through the C ABI with HOST buffers: upload (pinned H2D) + PageRank +
              result D2H, every step
  roofline    the iteration kernel: algorithmic bytes 8E + 16V per launch over its
              average launch time (from two fixed-iteration runs), vs measured HBM peak
  cpu_baseline  the OpenMP form of the generated code (oracle port), bounded sample

--impl reference times that OpenMP form alone on the host cores (the reference's
CPU path; its generated sources cannot be produced here).
Multi-GPU: PageRank on one graph is replicated per GPU ("replicas only"); value
sums the edges all ranks processed over the max time.
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


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


class Clocks:
    """nvidia-smi sampling during the timed region."""

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

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.3)
        self.p.terminate()
        self.p.wait()
        self.f.flush()
        rows = [r.split(",") for r in open(self.f.name).read().strip().splitlines() if r.strip()]
        os.unlink(self.f.name)
        sm = [float(r[1]) for r in rows if len(r) >= 9 and r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if len(r) >= 9 and r[2].strip().replace(".", "").isdigit()]
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


def make_graph():
    from starplat_b200 import generators as G

    t = time.time()
    g = G.rmat(PR_SCALE, PR_EF, seed=PR_SEED, directed=True)
    return g, time.time() - t


def cpu_baseline(g, iters: int = 3):
    """OpenMP form of the generated PageRank on the host cores, `iters` iterations."""
    from oracle import oracle as O

    nt = O.num_threads()
    t = time.perf_counter()
    _, it = O.pagerank_omp(g.indexofNodes, g.rev_indexofNodes, g.srcList, 0.0, DELTA, iters, nthreads=nt)
    dt = time.perf_counter() - t
    return {"value": g.E * it / dt / 1e9, "unit": "GTEPS", "cores": nt, "kind": "port",
            "sample": f"{it} iterations of the OpenMP-form PageRank over the full graph ({dt:.2f} s)"}


def run_reference(args, rank, world):
    if rank != 0:
        return
    g, _ = make_graph()
    for _ in range(args.warmup):
        cpu_baseline(g, 1)
    vals = []
    for _ in range(args.steps):
        vals.append(cpu_baseline(g, 3))
    v = statistics.median([x["value"] for x in vals])
    line = {"metric": METRIC, "value": v, "unit": "GTEPS", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic", "impl": "reference",
            "config": {"workload": f"pagerank rmat{PR_SCALE} ef{PR_EF} directed seed{PR_SEED}", "V": g.V, "E": g.E,
                       "beta": BETA, "delta": DELTA, "max_iter": MAX_ITER},
            "cpu_baseline": {**vals[-1], "value": v},
            "e2e": {"value": v, "unit": "GTEPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    global PR_SCALE
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--quick", action="store_true",
                    help="device-resident timing only (no roofline/e2e/CPU legs): for profiler runs")
    ap.add_argument("--scale", type=int, default=PR_SCALE, help="R-MAT scale (profiling on smaller cases)")
    ap.add_argument("--tune", action="append", default=[], help="schedule knob key=value (sp_tune_set)")
    args = ap.parse_args()
    PR_SCALE = args.scale

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank, world)

    import torch

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))

    def barrier():
        if dist is not None:
            dist.barrier()

    from starplat_b200 import _lib
    from starplat_b200.device import DeviceGraph

    g, gen_s = make_graph()
    V, E = g.V, g.E
    stream = torch.cuda.current_stream()
    dg = DeviceGraph.from_csr(g, with_weights=False)
    dg.set_stream(stream)
    for kv in args.tune:
        k, v = kv.split("=")
        dg.tune_set(k, int(v))
    out = torch.empty(V, dtype=torch.float32, device="cuda")

    for _ in range(max(3, args.warmup)):
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
    ms = ev0.elapsed_time(ev1)
    if dist is not None:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    value = world * E * it_total / (ms / 1e3) / 1e9
    if args.quick:
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": value, "unit": "GTEPS", "quick": True, "V": V, "E": E,
                              "iterations": it_total // args.steps, "ms_per_step": ms / args.steps}), flush=True)
        dg.free()
        if dist is not None:
            dist.destroy_process_group()
        return

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
    hbm, hbm_kind = peaks()
    achieved = alg_bytes / (per_launch_ms / 1e3) / 1e9
    roofline = {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                "traffic": None, "peak_kind": hbm_kind, "kernel": "sp::pr::k_iter",
                "alg_bytes_per_launch": alg_bytes, "avg_launch_ms": per_launch_ms}
    tf = os.path.join(ROOT, "profiles", "pagerank_traffic.json")
    if os.path.exists(tf):
        try:
            roofline["traffic"] = json.load(open(tf)).get("traffic_bytes_per_launch")
        except Exception:
            pass

    # ---- end to end through the C ABI with host buffers (pinned), every step
    pin = {k: torch.from_numpy(getattr(g, k)).pin_memory()
           for k in ("indexofNodes", "edgeList", "rev_indexofNodes", "srcList")}
    host_out = torch.empty(V, dtype=torch.float32).pin_memory()
    h2d = sum(t.numel() * 4 for t in pin.values())
    d2h = V * 4

    def e2e_step():
        with DeviceGraph(pin["indexofNodes"].numpy(), pin["edgeList"].numpy(), None,
                         pin["rev_indexofNodes"].numpy(), pin["srcList"].numpy()) as hg:
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
    e_s = time.perf_counter() - t0
    if dist is not None:
        t = torch.tensor([e_s], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e_s = float(t.item())
    e2e = {"value": world * E * e_it / e_s / 1e9, "unit": "GTEPS", "h2d_bytes_per_step": h2d,
           "d2h_bytes_per_step": d2h, "ms_per_step": 1e3 * e_s / e_steps}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(g, 3)

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "GTEPS", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": f"pagerank rmat{PR_SCALE} ef{PR_EF} directed seed{PR_SEED}", "V": V, "E": E,
                           "beta": BETA, "delta": DELTA, "max_iter": MAX_ITER, "iterations": it_total // args.steps,
                           "l2": "inputs larger than L2 (srcList %.2f GB streamed per iteration)" % (4 * E / 1e9),
                           "parallelism": "replicas" if world > 1 else "single", "graph_gen_s": round(gen_s, 2)},
                "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches, "clocks": clocks}
        print(json.dumps(line), flush=True)
    dg.free()
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
