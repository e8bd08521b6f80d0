"""Multi-source algorithms over the GPUs of one node: the sources are split among the
ranks, each rank runs its slice on its own GPU, and one all-reduce adds the per-vertex
vectors.
  * Brandes BC (sp_bc, all batches in one launch): BC is a sum over sources
    (bc_dslV2: BC[v] += delta_s[v] for every source s), so the split is exact up to
    FP32 rounding of the partial sums.
  * Closeness (sp_closeness / sp_closeness_unweighted): CC is nonzero only at the
    sources and each source's entry comes from one rank, so the sum of the slices is
    the whole, bit for bit.
Triangle counting and the clustering coefficient split anchors instead: rank r counts
the triangles of part r of the anchor order (sp_tc_part / sp_clustering_coeff_part), and
one all-reduce adds an int64 count or an int32[V] vector, exactly.
PageRank splits vertices (pagerank_on_gpus): rank r owns the rows of part r, and every
iteration ends with an all-gather of the parts' contrib blocks and an all-reduce of the
L1 diff, both on device buffers; the stop test runs on the device.
Single-source SSSP splits vertices too (sssp_on_gpus): rank r owns v % world == r, and
every delta-stepping round ends with an all-to-all of (vertex, distance) messages for
the other ranks' vertices and a sum of the frontier sizes.
The process group comes from replicas.Replicas (NCCL on GPUs, gloo on the host).
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


def sum_over_sources(V: int, sources, rep: Replicas, compute: Callable, out=None):
    """A float32[V] that is a sum over `sources`: this rank computes its slice, then the
    partial vectors are summed over the ranks, and every rank returns the full result.
    Without `out`, compute(slice) returns a float32[V] array and the result is numpy.
    With `out` (a float32[V] torch tensor on the backend's device: this rank's GPU under
    NCCL), compute(slice, out) writes the slice's vector into it and the sum is taken in
    place, so the vector never leaves the device; `out` is returned."""
    mine = split_sources(sources, rep.world, rep.rank)
    if out is not None:
        if mine.shape[0]:
            compute(mine, out)
        else:
            out.zero_()
        return rep.all_reduce_sum(out)
    part = compute(mine) if mine.shape[0] else np.zeros(V, np.float32)
    return rep.all_reduce_sum(np.ascontiguousarray(part, np.float32))


def bc_sharded(V: int, sources, rep: Replicas, compute: Callable, out=None):
    """BC[V] over all `sources` (compute: DeviceGraph.bc on a GPU; see sum_over_sources
    for `out`)."""
    return sum_over_sources(V, sources, rep, compute, out)


def closeness_on_gpus(dg, sources, rep: Optional[Replicas] = None, weighted: bool = True, weight=None, out=None):
    """Compute_CC (weighted, the graph's edgeLen or `weight`) or Compute_CC_Unweighted
    over `sources`, split over the ranks; every rank returns CC[V] (in `out`, a device
    tensor under NCCL, when given)."""
    rep = rep or Replicas()
    if weighted:
        if out is not None:
            return sum_over_sources(dg.V, sources, rep, lambda s, o: dg.closeness(s, weight=weight, out=o), out)
        return sum_over_sources(dg.V, sources, rep, lambda s: dg.closeness(s, weight=weight))
    if out is not None:
        return sum_over_sources(dg.V, sources, rep, lambda s, o: dg.closeness_unweighted(s, out=o), out)
    return sum_over_sources(dg.V, sources, rep, lambda s: dg.closeness_unweighted(s))


def bc_on_gpus(dg, sources, rep: Optional[Replicas] = None, out=None):
    """bc_sharded with this rank's DeviceGraph doing its slice; with `out` (a float32[V]
    tensor on this rank's GPU) the slice's BC is written there by the kernel and summed
    over the ranks in place by NCCL."""
    rep = rep or Replicas()
    if out is not None:
        return bc_sharded(dg.V, sources, rep, lambda s, o: dg.bc(s, out=o), out)
    return bc_sharded(dg.V, sources, rep, lambda s: dg.bc(s))


def tc_sharded(rep: Replicas, compute: Callable[[int, int], int]) -> int:
    """Compute_TC over the ranks: compute(part, nparts) counts this rank's part (an exact
    int64), and the parts are summed."""
    mine = np.array([compute(rep.rank, rep.world)], np.int64)
    return int(rep.all_reduce_sum(mine)[0])


def lcc_sharded(V: int, rep: Replicas, compute: Callable, out=None):
    """staticClusteringCoeff over the ranks: compute(part, nparts) gives this rank's
    int32[V] counts, and the vectors are summed (int32, exact). With `out` (an int32[V]
    tensor on the backend's device) compute(part, nparts, out) writes into it and the
    sum is taken in place."""
    if out is not None:
        compute(rep.rank, rep.world, out)
        return rep.all_reduce_sum(out)
    mine = np.ascontiguousarray(compute(rep.rank, rep.world), np.int32)
    assert mine.shape == (V,)
    return rep.all_reduce_sum(mine)


def tc_on_gpus(dg, rep: Optional[Replicas] = None) -> int:
    """tc_sharded with this rank's DeviceGraph (the whole graph on every GPU)."""
    rep = rep or Replicas()
    return tc_sharded(rep, dg.tc_part)


def clustering_coeff_on_gpus(dg, rep: Optional[Replicas] = None, out=None):
    """lcc_sharded with this rank's DeviceGraph (the counts stay on the GPU in `out`)."""
    rep = rep or Replicas()
    if out is not None:
        return lcc_sharded(dg.V, rep, lambda r, n, o: dg.clustering_coeff_part(r, n, out=o), out)
    return lcc_sharded(dg.V, rep, lambda r, n: dg.clustering_coeff_part(r, n))


def pagerank_on_gpus(dg, rep: Optional[Replicas] = None, beta: float = 1e-6, delta: float = 0.85,
                     max_iter: int = 100, out=None, check_every: int = 8):
    """ComputePageRank split over the ranks by vertices (sp_pagerank_part_*): every rank
    holds the whole graph and computes the rows of its part; per iteration, one NCCL
    all-gather of the parts' contrib blocks (S floats each) and one all-reduce of the
    diff, in stream order with the kernels, so nothing crosses to the host. The stop
    test runs on the device; the host reads the state once every `check_every`
    iterations. Replaces the host-staged exchange of the reference's multi-GPU code
    (backend_multigpu/dsl_cpp_generator.cpp:604-678). Returns (pageRank[V] float32 in
    the caller's vertex order, iterations, final diff); `out` (host or device) receives
    the ranks when given."""
    import torch

    from .device import DeviceGraph

    rep = rep or Replicas()
    dev = rep.device()
    if isinstance(dg, DeviceGraph):
        if dev.type != "cuda":
            raise ValueError("pagerank_on_gpus: the part buffers must be device tensors (NCCL or one GPU)")
        dg.set_stream(torch.cuda.current_stream())  # the collectives' stream order
    n, r = rep.world, rep.rank
    S = -(-dg.V // n)
    con = [torch.empty(n * S, dtype=torch.float32, device=dev) for _ in range(2)]
    diff = torch.zeros(1, dtype=torch.float64, device=dev)
    if dg.pagerank_part_begin(r, n, beta, delta, max_iter, con[0], con[1], diff) != S:
        raise RuntimeError("pagerank_on_gpus: slice size mismatch")
    k = 0
    while True:
        for _ in range(check_every):
            dg.pagerank_part_iterate(k)
            nxt = con[(k + 1) & 1]
            rep.all_gather_into(nxt, nxt[r * S:(r + 1) * S])
            rep.all_reduce_sum(diff)
            dg.pagerank_part_decide()
            k += 1
        it, done, d = dg.pagerank_part_state()
        if done:
            break
        if k > max(1, max_iter) + check_every:
            raise RuntimeError("pagerank_on_gpus: the stop test never fired")
    part = torch.empty(S, dtype=torch.float32, device=dev)
    dg.pagerank_part_ranks(part)
    full = torch.empty(n * S, dtype=torch.float32, device=dev)
    rep.all_gather_into(full, part)
    if out is None:
        out = np.empty(dg.V, np.float32)
    dg.pagerank_part_finish(full, out)
    return out, it, d


INT_MAX = 2**31 - 1


def sssp_on_gpus(dg, rep: Optional[Replicas] = None, src: int = 0, weight=None, delta: int = 0, out=None):
    """Compute_SSSP split over the ranks by vertices (sp_sssp_part_*): every rank holds
    the whole graph and owns the vertices v with v % world == rank. A delta-stepping
    round relaxes each rank's frontier; candidates for other ranks' vertices travel as
    (vertex, distance) pairs, at most one per vertex per round, in one all-to-all (its
    counts first); the frontier sizes are summed to decide whether the bucket goes on.
    An empty bucket everywhere moves all ranks to the bucket of the smallest far
    distance (a minimum over the ranks), and INT_MAX there ends the solve. This is the
    1-D partition with a per-bucket frontier exchange that replaces the host-staged
    copies of the reference's multi-GPU code (backend_multigpu/dsl_cpp_generator.cpp:
    604-678). Returns (dist int32[V], rounds); `out` (host or device) receives dist."""
    import torch

    from .device import DeviceGraph

    rep = rep or Replicas()
    dev = rep.device()
    if isinstance(dg, DeviceGraph):
        if dev.type != "cuda":
            raise ValueError("sssp_on_gpus: the message buffers must be device tensors (NCCL or one GPU)")
        dg.set_stream(torch.cuda.current_stream())  # the collectives' stream order
    n, r = rep.world, rep.rank
    cap = dg.sssp_part_begin(r, n, src, weight, delta)
    send = torch.empty((n * cap, 2), dtype=torch.int32, device=dev)
    recv = torch.empty((n * cap, 2), dtype=torch.int32, device=dev)
    scount = torch.zeros(n, dtype=torch.int32, device=dev)
    rcount = torch.zeros(n, dtype=torch.int32, device=dev)
    frontier = torch.zeros(1, dtype=torch.int32, device=dev)
    far = torch.zeros(1, dtype=torch.int32, device=dev)
    rounds = 0
    while True:
        while True:  # the rounds of one bucket
            dg.sssp_part_relax(send, scount)
            rep.all_to_all(rcount, scount, [1] * n, [1] * n)
            sc, rc = scount.tolist(), rcount.tolist()
            ns, nr = sum(sc), sum(rc)
            rep.all_to_all(recv[:nr], send[:ns], rc, sc)
            dg.sssp_part_apply(recv, nr, frontier)
            rep.all_reduce_sum(frontier)
            rounds += 1
            if int(frontier.item()) == 0:
                break
        dg.sssp_part_far_min(far)
        rep.all_reduce_min(far)
        if int(far.item()) == INT_MAX:
            break
        dg.sssp_part_advance(far, frontier)
        rep.all_reduce_sum(frontier)
    full = torch.empty(dg.V, dtype=torch.int32, device=dev)
    dg.sssp_part_dist(full)
    rep.all_reduce_min(full)
    if out is None:
        out = full.cpu().numpy()
    elif isinstance(out, np.ndarray):
        out[:] = full.cpu().numpy()
    else:
        out.copy_(full)
    return out, rounds
