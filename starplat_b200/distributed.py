"""Brandes BC over the GPUs of one node: the sources are split among the ranks, each
rank runs its slice on its own GPU (sp_bc, all batches in one launch), and one
all-reduce adds the per-vertex dependency sums. BC is a sum over sources
(bc_dslV2: BC[v] += delta_s[v] for every source s), so the split is exact up to FP32
rounding of the partial sums. The process group comes from replicas.Replicas (NCCL on
GPUs, gloo on the host).
"""
from __future__ import annotations

from typing import Callable, Optional

import numpy as np

from .replicas import Replicas


def split_sources(sources, world: int, rank: int) -> np.ndarray:
    """Rank `rank`'s contiguous slice of `sources` (sizes differ by at most one)."""
    s = np.asarray(sources, np.int32)
    n = s.shape[0]
    lo = n * rank // world
    hi = n * (rank + 1) // world
    return s[lo:hi]


def bc_sharded(V: int, sources, rep: Replicas, compute: Callable[[np.ndarray], np.ndarray]) -> np.ndarray:
    """BC[V] over all `sources`: this rank computes its slice with `compute` (slice ->
    float32[V]; DeviceGraph.bc on a GPU), then the partial vectors are summed over the
    ranks. Every rank returns the full result."""
    mine = split_sources(sources, rep.world, rep.rank)
    part = compute(mine) if mine.shape[0] else np.zeros(V, np.float32)
    return rep.all_reduce_sum(np.ascontiguousarray(part, np.float32))


def bc_on_gpus(dg, sources, rep: Optional[Replicas] = None) -> np.ndarray:
    """bc_sharded with this rank's DeviceGraph doing its slice."""
    rep = rep or Replicas()
    return bc_sharded(dg.V, sources, rep, lambda s: dg.bc(s))
