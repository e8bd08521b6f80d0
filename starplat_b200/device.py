"""Device mirror of a CSR graph and the algorithm entry points.

``DeviceGraph`` owns an ``sp_graph_h`` from the C ABI: the forward CSR (and the
reverse CSR / weights when given) uploaded once and reused by every algorithm
call, replacing the per-call host-to-device copy of StarPlat's generated CUDA
code (backend_cuda/dsl_cpp_generator.cpp:4104-4297).

Arrays passed in may be numpy arrays (host) or CUDA tensors (device); outputs
are written to caller-provided arrays of either kind.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional

import numpy as np

from . import _lib
from ._lib import check, lib
from .graph import CSRGraph


def _ptr(a) -> Optional[int]:
    """Data pointer of a numpy array or a torch tensor (None for None)."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        if not a.flags["C_CONTIGUOUS"]:
            raise ValueError("array must be C-contiguous")
        return a.ctypes.data
    if hasattr(a, "data_ptr"):
        if not a.is_contiguous():
            raise ValueError("tensor must be contiguous")
        return a.data_ptr()
    raise TypeError(f"unsupported array type {type(a)}")


def _is_device(a) -> bool:
    return hasattr(a, "is_cuda") and bool(a.is_cuda)


CUDA_STREAM_LEGACY = 1  # cudaStreamLegacy: the legacy default stream, as a stream handle

_SCHED_TRIED = False


def _ensure_scheduler():
    """Load the trained scheduling model once per process, if it ships with the package."""
    global _SCHED_TRIED
    if not _SCHED_TRIED:
        _SCHED_TRIED = True
        from . import scheduler

        scheduler.load()


class DeviceGraph:
    """A graph resident in GPU memory (the C ABI's sp_graph_h)."""

    def __init__(self, indexofNodes, edgeList, edgeLen=None, rev_indexofNodes=None, srcList=None):
        dev = _is_device(indexofNodes)
        arrs = [indexofNodes, edgeList, edgeLen, rev_indexofNodes, srcList]
        for a in arrs:
            if a is not None and _is_device(a) != dev:
                raise ValueError("mix of host and device arrays")
            if a is not None:
                dt = a.dtype
                if str(dt) not in ("int32", "torch.int32"):
                    raise TypeError(f"CSR arrays must be int32, got {dt}")
        V = int(indexofNodes.shape[0]) - 1
        E = int(edgeList.shape[0])
        h = ctypes.c_void_p()
        flags = _lib.SP_GRAPH_DEVICE_PTRS if dev else 0
        check("sp_graph_create", lib().sp_graph_create(V, E, *[_ptr(a) for a in arrs], flags, ctypes.byref(h)))
        self._h = h
        self.V = V
        self.E = E
        self._keep = arrs if dev else None

    @classmethod
    def load_text(cls, path: str, nthreads: int = 0) -> "DeviceGraph":
        """Read a text edge list (the reference's graph::parseGraph format) straight into
        GPU memory: tokenised on the host, sorted, merged and turned into both CSRs on the
        device."""
        h = ctypes.c_void_p()
        check("sp_graph_load_text", lib().sp_graph_load_text(os.fsencode(path), int(nthreads), ctypes.byref(h)))
        self = cls.__new__(cls)
        self._h = h
        self._keep = None
        V = ctypes.c_int32()
        E = ctypes.c_int64()
        check("sp_graph_info", lib().sp_graph_info(h, ctypes.byref(V), ctypes.byref(E), None))
        self.V, self.E = int(V.value), int(E.value)
        return self

    @staticmethod
    def _batch(types, src, dst, weight):
        t = np.ascontiguousarray(np.frombuffer(types.encode() if isinstance(types, str) else bytes(types), np.uint8))
        s = np.ascontiguousarray(src, np.int32)
        d = np.ascontiguousarray(dst, np.int32)
        n = t.shape[0]
        if s.shape[0] != n or d.shape[0] != n:
            raise ValueError("types, src and dst must have one entry per update")
        w = None if weight is None else np.ascontiguousarray(weight, np.int32)
        if w is not None and w.shape[0] != n:
            raise ValueError("weight must have one entry per update")
        ptrs = [a.ctypes.data if n else None for a in (t, s, d)]
        return n, ptrs + [None if w is None or n == 0 else w.ctypes.data], (t, s, d, w)

    def _refresh_size(self):
        V = ctypes.c_int32()
        E = ctypes.c_int64()
        check("sp_graph_info", lib().sp_graph_info(self.handle, ctypes.byref(V), ctypes.byref(E), None))
        self.V, self.E = int(V.value), int(E.value)

    def update(self, types, src, dst, weight=None) -> None:
        """One batch of edge updates (graph::updateCSRDel then updateCSRAdd): types is a
        str or bytes of 'a' / 'd' per update, src and dst int32 ids, weight int32 or None
        (1). Deletions apply first; an added edge that exists gets its weights summed."""
        n, ptrs, _keep = self._batch(types, src, dst, weight)
        check("sp_graph_update", lib().sp_graph_update(self.handle, n, *ptrs))
        self._refresh_size()

    def sssp_dynamic(self, types, src, dst, weight, source: int, dist):
        """DynSSSP's Batch block: apply the updates, then bring dist (the distances from
        source before the batch, int32[V], host or device) up to date on the new graph.
        A batch that only adds new edges resumes from dist; a batch with deletions on a
        graph with all weights >= 1 repairs the subtrees that lost their parent edge and
        resumes; other batches with deletions, and additions to edges the graph already
        holds (their weight grows, so distances can rise), solve again. Returns True when
        the call resumed or repaired (incremental) and False when it solved again;
        tune_get("sssp.last_incremental") tells 1 (resumed) from 2 (repaired)."""
        _ensure_scheduler()
        n, ptrs, _keep = self._batch(types, src, dst, weight)
        check("sp_sssp_dynamic", lib().sp_sssp_dynamic(self.handle, n, *ptrs, int(source), _ptr(dist)))
        self._refresh_size()
        return bool(self.tune_get("sssp.last_incremental"))

    def tc_dynamic(self, types, src, dst, weight, count: int):
        """DynTC's Batch block: apply the updates, then bring `count` (the graph's
        triangle count before the batch) up to date. Returns (new count, True when only
        the triangles through the batch's edges were counted)."""
        n, ptrs, _keep = self._batch(types, src, dst, weight)
        c = ctypes.c_int64(int(count))
        check("sp_tc_dynamic", lib().sp_tc_dynamic(self.handle, n, *ptrs, ctypes.byref(c)))
        self._refresh_size()
        return int(c.value), bool(self.tune_get("tc.last_incremental"))

    def clustering_coeff_dynamic(self, types, src, dst, weight, cf):
        """DynCF's Batch block: apply the updates, then bring cf (int32[V], host or device:
        the per-vertex triangle counts before the batch) up to date in place. Returns
        True when only the triangles through the batch's edges were counted."""
        if str(cf.dtype) not in ("int32", "torch.int32") or len(cf) != self.V:
            raise ValueError("cf must be int32 with one entry per vertex")
        n, ptrs, _keep = self._batch(types, src, dst, weight)
        check("sp_clustering_coeff_dynamic", lib().sp_clustering_coeff_dynamic(self.handle, n, *ptrs, _ptr(cf)))
        self._refresh_size()
        return bool(self.tune_get("tc.last_incremental"))

    def degree_dynamic(self, types, src, dst, weight=None, out=None):
        """DynDegree's Batch block: apply the updates, then the out-degrees: int32[V]."""
        if out is None:
            out = np.empty(self.V, np.int32)
        n, ptrs, _keep = self._batch(types, src, dst, weight)
        check("sp_degree_dynamic", lib().sp_degree_dynamic(self.handle, n, *ptrs, _ptr(out)))
        self._refresh_size()
        return out

    def bc_dynamic(self, types, src, dst, weight, sources, out=None):
        """DynBC's Batch block: apply the updates, then BC over `sources` on the new graph
        (float32[V])."""
        if out is None:
            out = np.empty(self.V, np.float32)
        if isinstance(sources, (list, tuple, np.ndarray)):
            sources = np.ascontiguousarray(sources, np.int32)
        ns = int(sources.shape[0])
        n, ptrs, _keep = self._batch(types, src, dst, weight)
        check("sp_bc_dynamic", lib().sp_bc_dynamic(self.handle, n, *ptrs, _ptr(sources) if ns else None, ns,
                                                   _ptr(out)))
        self._refresh_size()
        return out

    def pagerank_dynamic(self, types, src, dst, weight, pagerank, beta: float = 1e-6, delta: float = 0.85,
                         max_iter: int = 100):
        """DynPR's Batch block: apply the updates (none if types is empty), then run
        PageRank on the new graph from `pagerank` (float32[V], host or device: the ranks
        before the batch) instead of 1/V. The new ranks overwrite `pagerank`; returns
        (pagerank, iterations, final L1 diff)."""
        if str(pagerank.dtype) not in ("float32", "torch.float32") or len(pagerank) != self.V:
            raise ValueError("pagerank must be float32 with one entry per vertex")
        n, ptrs, _keep = self._batch(types, src, dst, weight)
        it = ctypes.c_int32()
        diff = ctypes.c_double()
        check("sp_pagerank_dynamic", lib().sp_pagerank_dynamic(self.handle, n, *ptrs, beta, delta, max_iter,
                                                               _ptr(pagerank), ctypes.byref(it), ctypes.byref(diff)))
        self._refresh_size()
        return pagerank, int(it.value), float(diff.value)

    def export(self) -> dict:
        """The mirror's CSR as host arrays named like graph.hpp's fields."""
        V, E = self.V, self.E
        out = {"indexofNodes": np.empty(V + 1, np.int32), "edgeList": np.empty(E, np.int32),
               "edgeLen": np.empty(E, np.int32), "rev_indexofNodes": np.empty(V + 1, np.int32),
               "srcList": np.empty(E, np.int32), "edgeMap": np.empty(E, np.int32)}
        names = ("indexofNodes", "edgeList", "edgeLen", "rev_indexofNodes", "srcList", "edgeMap")
        try:
            check("sp_graph_export", lib().sp_graph_export(self.handle, *[_ptr(out[k]) for k in names]))
        except _lib.SPError:  # a graph created without weights has no edgeLen
            del out["edgeLen"]
            check("sp_graph_export", lib().sp_graph_export(self.handle, *[_ptr(out.get(k)) for k in names]))
        return out

    @classmethod
    def from_csr(cls, g: CSRGraph, with_reverse: bool = True, with_weights: bool = True) -> "DeviceGraph":
        return cls(g.indexofNodes, g.edgeList, g.edgeLen if with_weights else None,
                   g.rev_indexofNodes if with_reverse else None, g.srcList if with_reverse else None)

    @property
    def handle(self):
        if self._h is None:
            raise RuntimeError("graph already freed")
        return self._h

    def free(self) -> None:
        if getattr(self, "_h", None) is not None:
            lib().sp_graph_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.free()

    def set_stream(self, stream) -> None:
        """Run later work on this CUDA stream (torch.cuda.Stream or raw cudaStream_t int).

        Torch's default stream has the handle 0, which the C ABI reads as "the library's
        own stream"; it is passed as cudaStreamLegacy instead, so that the library's
        kernels and torch's (and NCCL's) work on that stream stay in stream order."""
        raw = getattr(stream, "cuda_stream", stream)
        if hasattr(stream, "cuda_stream") and raw == 0:
            raw = CUDA_STREAM_LEGACY
        check("sp_graph_set_stream", lib().sp_graph_set_stream(self.handle, raw))

    def tune_set(self, key: str, value: int) -> None:
        check("sp_tune_set", lib().sp_tune_set(self.handle, key.encode(), int(value)))

    def tune_get(self, key: str) -> int:
        v = ctypes.c_int64()
        check("sp_tune_get", lib().sp_tune_get(self.handle, key.encode(), ctypes.byref(v)))
        return int(v.value)

    def info(self):
        V = ctypes.c_int32()
        E = ctypes.c_int64()
        s = ctypes.c_int32()
        check("sp_graph_info", lib().sp_graph_info(self.handle, ctypes.byref(V), ctypes.byref(E), ctypes.byref(s)))
        return V.value, E.value, bool(s.value)

    # ---------------------------------------------------------------- algorithms
    def tc(self, variant: int = _lib.SP_TC_TUNED) -> int:
        out = ctypes.c_int64()
        check("sp_tc", lib().sp_tc(self.handle, ctypes.byref(out), variant))
        return int(out.value)

    def tc_part(self, part: int, nparts: int) -> int:
        """Triangles anchored in part `part` of `nparts` of the anchor order; the parts sum
        to tc()."""
        out = ctypes.c_int64()
        check("sp_tc_part", lib().sp_tc_part(self.handle, int(part), int(nparts), ctypes.byref(out)))
        return int(out.value)

    def pagerank(self, beta: float = 1e-6, delta: float = 0.85, max_iter: int = 100, out=None,
                 variant: int = _lib.SP_PR_TUNED):
        if out is None:
            out = np.empty(self.V, np.float32)
        it = ctypes.c_int32()
        diff = ctypes.c_double()
        check("sp_pagerank", lib().sp_pagerank(self.handle, beta, delta, max_iter, _ptr(out), ctypes.byref(it),
                                               ctypes.byref(diff), variant))
        return out, int(it.value), float(diff.value)

    def sssp(self, src: int, weight=None, out=None, delta: int = 0, variant: int = _lib.SP_SSSP_DELTA):
        """Exact int32 distances from src (INT_MAX = unreachable). weight: int32[E] in
        forward-CSR order, host or device; None uses the graph's edgeLen. delta <= 0
        lets the learned scheduler pick the schedule (fixed heuristic without a model)."""
        _ensure_scheduler()
        if out is None:
            out = np.empty(self.V, np.int32)
        if weight is not None and str(weight.dtype) not in ("int32", "torch.int32"):
            raise TypeError("weights must be int32")
        rounds = ctypes.c_int32()
        check("sp_sssp", lib().sp_sssp(self.handle, _ptr(weight), int(src), _ptr(out), int(delta), variant,
                                       ctypes.byref(rounds)))
        return out, int(rounds.value)

    # ---- PageRank split over ranks by vertices (sp_pagerank_part_*; driven by
    # distributed.pagerank_on_gpus)
    def pagerank_part_begin(self, part: int, nparts: int, beta: float, delta: float, max_iter: int, con0, con1,
                            diff) -> int:
        """Starts this rank's part; con0 / con1 (nparts * S float32) and diff (one float64)
        are device tensors the caller's collectives work on. Returns S."""
        S = ctypes.c_int32()
        check("sp_pagerank_part_begin", lib().sp_pagerank_part_begin(
            self.handle, int(part), int(nparts), float(beta), float(delta), int(max_iter), _ptr(con0), _ptr(con1),
            _ptr(diff), ctypes.byref(S)))
        return int(S.value)

    def pagerank_part_iterate(self, k: int) -> None:
        check("sp_pagerank_part_iterate", lib().sp_pagerank_part_iterate(self.handle, int(k)))

    def pagerank_part_decide(self) -> None:
        check("sp_pagerank_part_decide", lib().sp_pagerank_part_decide(self.handle))

    def pagerank_part_state(self):
        """(iterations, done, summed diff); synchronises the stream."""
        it, done, diff = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_double()
        check("sp_pagerank_part_state", lib().sp_pagerank_part_state(self.handle, ctypes.byref(it), ctypes.byref(done),
                                                                     ctypes.byref(diff)))
        return int(it.value), bool(done.value), float(diff.value)

    def pagerank_part_ranks(self, slice_out) -> None:
        check("sp_pagerank_part_ranks", lib().sp_pagerank_part_ranks(self.handle, _ptr(slice_out)))

    def pagerank_part_finish(self, ranks, out) -> None:
        check("sp_pagerank_part_finish", lib().sp_pagerank_part_finish(self.handle, _ptr(ranks), _ptr(out)))

    # ---- single-source SSSP split over ranks by vertices (sp_sssp_part_*; driven by
    # distributed.sssp_on_gpus)
    def sssp_part_begin(self, part: int, nparts: int, src: int, weight=None, delta: int = 0) -> int:
        """Starts this rank's part of a split solve from src; returns cap (the send and
        receive buffers hold nparts * cap int32 pairs)."""
        _ensure_scheduler()  # delta <= 0: the width sp_sssp would choose
        if weight is not None and str(weight.dtype) not in ("int32", "torch.int32"):
            raise TypeError("weights must be int32")
        cap = ctypes.c_int32()
        check("sp_sssp_part_begin", lib().sp_sssp_part_begin(self.handle, int(part), int(nparts), _ptr(weight),
                                                             int(src), int(delta), ctypes.byref(cap)))
        return int(cap.value)

    def sssp_part_relax(self, send, send_counts) -> None:
        check("sp_sssp_part_relax", lib().sp_sssp_part_relax(self.handle, _ptr(send), _ptr(send_counts)))

    def sssp_part_apply(self, msgs, n: int, frontier) -> None:
        check("sp_sssp_part_apply", lib().sp_sssp_part_apply(self.handle, _ptr(msgs) if n else None, int(n),
                                                             _ptr(frontier)))

    def sssp_part_far_min(self, far_min) -> None:
        check("sp_sssp_part_far_min", lib().sp_sssp_part_far_min(self.handle, _ptr(far_min)))

    def sssp_part_advance(self, far_min, frontier) -> None:
        check("sp_sssp_part_advance", lib().sp_sssp_part_advance(self.handle, _ptr(far_min), _ptr(frontier)))

    def sssp_part_dist(self, dist) -> None:
        check("sp_sssp_part_dist", lib().sp_sssp_part_dist(self.handle, _ptr(dist)))

    def sssp_batch(self, sources, weight=None, out=None):
        """Distances from every source (int32, host or device) in batched cooperative
        launches, one CTA group per source: int32[nsrc][V], row k from sources[k]
        (host array, or `out` of that size on the host or the device)."""
        _ensure_scheduler()
        if isinstance(sources, (list, tuple)):
            sources = np.asarray(sources, np.int32)
        n = int(sources.shape[0])
        if out is None:
            out = np.empty((n, self.V), np.int32)
        if weight is not None and str(weight.dtype) not in ("int32", "torch.int32"):
            raise TypeError("weights must be int32")
        check("sp_sssp_batch", lib().sp_sssp_batch(self.handle, _ptr(weight), _ptr(sources), n, _ptr(out)))
        return out

    def bc(self, sources, out=None, variant: int = _lib.SP_BC_BATCHED):
        """Brandes BC over distinct `sources` (int32, host or device); float32[V]."""
        _ensure_scheduler()  # the level model, when shipped, picks each level's direction
        if out is None:
            out = np.empty(self.V, np.float32)
        if isinstance(sources, (list, tuple)):
            sources = np.asarray(sources, np.int32)
        n = int(sources.shape[0])
        check("sp_bc", lib().sp_bc(self.handle, _ptr(sources) if n else None, n, _ptr(out), variant))
        return out

    def bc_graphs(self, vertex_offset, source_offset, sources, out=None):
        """BC of many independent graphs stored as one disjoint union (see sp_bc_graphs)."""
        if out is None:
            out = np.empty(self.V, np.float32)
        G = int(vertex_offset.shape[0]) - 1
        check("sp_bc_graphs", lib().sp_bc_graphs(self.handle, G, _ptr(vertex_offset), _ptr(source_offset),
                                                 _ptr(sources), _ptr(out)))
        return out

    def bfs_sigma(self, sources):
        """BFS levels and shortest-path counts from up to 64 sources: (level[k][V], sigma[k][V])."""
        sources = np.ascontiguousarray(sources, np.int32)
        k = sources.shape[0]
        lvl = np.empty((k, self.V), np.int32)
        sig = np.empty((k, self.V), np.float64)
        check("sp_bfs_sigma", lib().sp_bfs_sigma(self.handle, _ptr(sources), k, _ptr(lvl), _ptr(sig)))
        return lvl, sig

    def clustering_coeff(self, out=None, variant: int = _lib.SP_TC_TUNED):
        """Per-vertex triangle counts of the Compute_TC loop (staticClusteringCoeff): int32[V]."""
        if out is None:
            out = np.empty(self.V, np.int32)
        check("sp_clustering_coeff", lib().sp_clustering_coeff(self.handle, _ptr(out), variant))
        return out

    def clustering_coeff_part(self, part: int, nparts: int, out=None):
        """Per-vertex counts of the triangles in part `part` of `nparts`; the parts' vectors
        sum to clustering_coeff()."""
        if out is None:
            out = np.empty(self.V, np.int32)
        check("sp_clustering_coeff_part",
              lib().sp_clustering_coeff_part(self.handle, int(part), int(nparts), _ptr(out)))
        return out

    def degree(self, out=None):
        """Out-degree of every vertex (Degree): int32[V]."""
        if out is None:
            out = np.empty(self.V, np.int32)
        check("sp_degree_centrality", lib().sp_degree_centrality(self.handle, _ptr(out)))
        return out

    def closeness(self, sources, weight=None, out=None):
        """Compute_CC: CC[src] = 1 / (sum of finite weighted distances from src), 0
        elsewhere; float32[V]. weight: int32[E] or None for the graph's edgeLen."""
        _ensure_scheduler()
        if out is None:
            out = np.empty(self.V, np.float32)
        if weight is not None and str(weight.dtype) not in ("int32", "torch.int32"):
            raise TypeError("weights must be int32")
        if isinstance(sources, (list, tuple)):
            sources = np.asarray(sources, np.int32)
        n = int(sources.shape[0])
        check("sp_closeness", lib().sp_closeness(self.handle, _ptr(weight), _ptr(sources) if n else None, n,
                                                 _ptr(out)))
        return out

    def closeness_unweighted(self, sources, out=None):
        """Compute_CC_Unweighted: CC[src] = 1 / (sum of BFS levels from src), 0 elsewhere."""
        if out is None:
            out = np.empty(self.V, np.float32)
        if isinstance(sources, (list, tuple)):
            sources = np.asarray(sources, np.int32)
        n = int(sources.shape[0])
        check("sp_closeness_unweighted", lib().sp_closeness_unweighted(self.handle, _ptr(sources) if n else None,
                                                                       n, _ptr(out)))
        return out

    def louvain(self, weight=None, threshold: float = 1e-4, community=None, variant: int = _lib.SP_LV_TUNED):
        """Louvain; returns (modularity, community[V] int32, levels). The shipped variant
        model, loaded on first use, picks each level's CTA-bin table size."""
        _ensure_scheduler()
        if community is None:
            community = np.empty(self.V, np.int32)
        if weight is not None and str(weight.dtype) not in ("float32", "torch.float32"):
            raise TypeError("Louvain weights must be float32")
        q = ctypes.c_double()
        lv = ctypes.c_int32()
        sw = ctypes.c_int32()
        check("sp_louvain", lib().sp_louvain(self.handle, _ptr(weight), threshold, _ptr(community), ctypes.byref(q),
                                             ctypes.byref(lv), ctypes.byref(sw), variant))
        self.last_louvain_sweeps = int(sw.value)
        return float(q.value), community, int(lv.value)
