"""Autotuner for the schedule knobs (sp_tune_set) of one graph.

Each algorithm's kernels take thresholds that change only how work is split:
  tc        tc.cta_warps: a bitmap per warp (0) or per CTA of 2 / 4 / 8 warps
  pagerank  pr.order: vertex order by out-degree (0) or in-degree class first (1);
            pr.src_hint: L1 policy of the srcList loads; pr.hot: sources of the
            L1-resident hot phase (0 = one phase); pr.l1_hot: sources whose gathers
            allocate in L1
  sssp      sssp.hub_deg / sssp.hub_chunk: queued vertices above hub_deg out-edges are
            relaxed in hub_chunk-edge pieces shared by all warps; sssp.local: warp
            cascade budget per round (0 = off)
  bc        bc.hub_deg / bc.hub_chunk: the same for level-list entries; bc.dir: push
            only (0) or the pull rule (1) per forward level
tune() times every candidate on the caller's graph with CUDA events on the graph's
stream (median of `reps` runs after one untimed run), keeps the fastest, leaves it set
on the graph and returns the table. Counts, distances, levels and path counts are the
same under every candidate; PageRank sums change grouping (FP32 rounding), which the
PageRank tests bound.
"""
from __future__ import annotations

import itertools
import statistics
from typing import Callable, Dict, List, Sequence, Tuple

import numpy as np

KNOBS: Dict[str, Dict[str, Sequence[int]]] = {
    "tc": {"tc.cta_warps": (0, 2, 4, 8)},
    "pagerank": {"pr.order": (0, 1), "pr.src_hint": (0, 2), "pr.hot": (0, 4096), "pr.l1_hot": (0, 32768, 131072)},
    "sssp": {"sssp.hub_deg": (64, 128, 512, 2048), "sssp.hub_chunk": (32, 64, 256), "sssp.local": (0, 16, 64)},
    "bc": {"bc.hub_deg": (32, 64, 256, 4096), "bc.hub_chunk": (64, 128, 256), "bc.dir": (0, 1)},
}


def _runner(dg, algo: str, args: dict) -> Callable[[], object]:
    if algo == "tc":
        return lambda: dg.tc()
    if algo == "pagerank":
        out = args.get("out")
        return lambda: dg.pagerank(args.get("beta", 1e-6), args.get("delta", 0.85), args.get("max_iter", 100),
                                   out=out)
    if algo == "sssp":
        src, weight, out = args.get("src", 0), args.get("weight"), args.get("out")
        return lambda: dg.sssp(src, weight=weight, out=out)
    if algo == "bc":
        sources = np.asarray(args["sources"], np.int32)
        return lambda: dg.bc(sources)
    raise ValueError(f"no knobs to tune for {algo!r} (choose from {sorted(KNOBS)})")


def _time(fn, reps: int, stream) -> float:
    import torch

    fn()  # untimed: plan building, graph capture
    times = []
    for _ in range(reps):
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        fn()
        b.record(stream)
        torch.cuda.synchronize()
        times.append(a.elapsed_time(b))
    return statistics.median(times)


def tune(dg, algo: str, reps: int = 3, space: Dict[str, Sequence[int]] | None = None,
         **args) -> List[Tuple[Dict[str, int], float]]:
    """Time every combination of `algo`'s knob candidates on `dg` and keep the fastest
    set on it. Returns [(setting, median ms)], fastest first. The graph's stream must
    be torch's current stream (DeviceGraph.set_stream) for the event timing."""
    if algo not in KNOBS:
        raise ValueError(f"no knobs to tune for {algo!r} (choose from {sorted(KNOBS)})")
    import torch

    space = dict(space or KNOBS[algo])
    run = _runner(dg, algo, args)
    stream = torch.cuda.current_stream()
    keys = list(space)
    table = []
    for values in itertools.product(*(space[k] for k in keys)):
        setting = dict(zip(keys, values))
        for k, v in setting.items():
            dg.tune_set(k, v)
        table.append((setting, _time(run, reps, stream)))
    table.sort(key=lambda t: t[1])
    for k, v in table[0][0].items():
        dg.tune_set(k, v)
    return table
