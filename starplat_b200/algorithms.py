"""The generated StarPlat entry points, same names and argument meaning.

Each takes a ``CSRGraph`` (the host container in the layout of graph.hpp) plus
the property arrays, exactly like the C++ functions the StarPlat generator
emits (signature emitter backend_omp/dsl_cpp_generator.cpp:3098-3151). The device
mirror is uploaded on first use and cached on the graph object, as the C++
wrappers in include/starplat_b200.hpp cache it per `graph*`.
"""
from __future__ import annotations

import numpy as np

from .device import DeviceGraph
from .graph import CSRGraph


def device_graph(g: CSRGraph) -> DeviceGraph:
    dg = getattr(g, "_device_mirror", None)
    if dg is None:
        dg = DeviceGraph.from_csr(g)
        g._device_mirror = dg
    return dg


def invalidate(g: CSRGraph) -> None:
    """Drop the cached device mirror (call after mutating the host CSR)."""
    dg = getattr(g, "_device_mirror", None)
    if dg is not None:
        dg.free()
        g._device_mirror = None


def Compute_TC(g: CSRGraph) -> int:
    """staticDSLCodes/triangle_counting_dsl: returns the int64 triangle count."""
    return device_graph(g).tc()


def ComputePageRank(g: CSRGraph, beta: float, delta: float, maxIter: int, pageRank: np.ndarray) -> None:
    """staticDSLCodes/PageRankDSLV3: writes float pageRank[num_nodes()]."""
    device_graph(g).pagerank(beta, delta, maxIter, out=pageRank)


Compute_PR = ComputePageRank  # the V2 DSL's name, same parameters


def Compute_SSSP(g: CSRGraph, dist: np.ndarray, weight: np.ndarray, src: int) -> None:
    """staticDSLCodes/sssp_dslV3: fills int dist[num_nodes()] (INT_MAX = unreachable);
    weight is int[E] in forward-CSR order, as the reference drivers build it."""
    device_graph(g).sssp(src, weight=weight, out=dist)


def Compute_BC(g: CSRGraph, BC: np.ndarray, sourceSet) -> None:
    """staticDSLCodes/bc_dslV2: fills float BC[num_nodes()] over the sources in
    sourceSet (any iterable of distinct vertex ids, like the reference's std::set<int>)."""
    src = np.array(sorted(set(int(s) for s in sourceSet)), np.int32)
    device_graph(g).bc(src, out=BC)


def staticClusteringCoeff(g: CSRGraph, cf: np.ndarray) -> None:
    """staticDSLCodes/clustering_coeff: fills int cf[num_nodes()] with the number of
    triangles of the Compute_TC loop through each vertex."""
    device_graph(g).clustering_coeff(out=cf)


def Degree(g: CSRGraph, deg: np.ndarray) -> None:
    """staticDSLCodes/degree_centrality: fills int deg[num_nodes()] with out-degrees."""
    device_graph(g).degree(out=deg)


def Compute_CC(g: CSRGraph, CC: np.ndarray, sourceSet) -> None:
    """staticDSLCodes/CC: fills float CC[num_nodes()]: 1 / (sum of finite shortest-path
    distances over the graph's edgeLen) at each source, 0 elsewhere."""
    src = np.array(sorted(set(int(s) for s in sourceSet)), np.int32)
    if src.shape[0] == 0:
        CC[:] = 0
        return
    device_graph(g).closeness(src, out=CC)


def Compute_CC_Unweighted(g: CSRGraph, CC: np.ndarray, sourceSet) -> None:
    """staticDSLCodes/closeness_centrality_unwt: fills float CC[num_nodes()]: 1 / (sum
    of BFS levels) at each source, 0 elsewhere."""
    src = np.array(sorted(set(int(s) for s in sourceSet)), np.int32)
    if src.shape[0] == 0:
        CC[:] = 0
        return
    device_graph(g).closeness_unweighted(src, out=CC)


def Compute_CD(g: CSRGraph, weight=None) -> float:
    """staticDSLCodes/community_detection: returns the modularity of the Louvain
    partition; weight is int[E] (or float[E]) in forward-CSR order, None = unit."""
    w = None if weight is None else np.ascontiguousarray(weight, np.float32)
    q, _, _ = device_graph(g).louvain(w, 1e-4)
    return q


# ---- the dynamic programs (dynamicDSLCodes): the static pass, then one Batch block per
# batchSize updates. updateBatch is a sequence of update records (type 'a' / 'd',
# source, destination, weight), as graph.hpp's `update` struct. Each program works on a
# private device copy of g that it frees on return: the host CSRGraph and the mirror that
# the static entry points cache on it keep the graph as it was before the batches.

def _batches(updateBatch, batchSize: int):
    """updates<g>.currentBatch(): consecutive slices of batchSize records, as arrays."""
    if batchSize <= 0:
        raise ValueError("batchSize must be positive")
    ups = list(updateBatch)
    for k in range(0, len(ups), batchSize):
        chunk = ups[k:k + batchSize]
        yield ("".join(u[0] for u in chunk), np.array([u[1] for u in chunk], np.int32),
               np.array([u[2] for u in chunk], np.int32), np.array([u[3] for u in chunk], np.int32))


def DynTC(g: CSRGraph, updateBatch, batchSize: int) -> int:
    """dynamicBatchTCV2 DynTC: the triangle count after every batch (the last is returned)."""
    with DeviceGraph.from_csr(g) as dg:
        count = dg.tc()
        for t, s, d, w in _batches(updateBatch, batchSize):
            count, _ = dg.tc_dynamic(t, s, d, w, count)
        return count


def DynPR(g: CSRGraph, beta: float, delta: float, maxIter: int, pageRank: np.ndarray, updateBatch,
          batchSize: int) -> None:
    """dynamicBatchPR DynPR: pageRank[V] of the graph after the last batch, each batch
    started from the ranks before it."""
    with DeviceGraph.from_csr(g) as dg:
        dg.pagerank(beta, delta, maxIter, out=pageRank)
        for t, s, d, w in _batches(updateBatch, batchSize):
            dg.pagerank_dynamic(t, s, d, w, pageRank, beta, delta, maxIter)


def DynSSSP(g: CSRGraph, dist: np.ndarray, parent, weight, updateBatch, batchSize: int, src: int) -> None:
    """dynamicBatchSSSP DynSSSP: dist[V] from src after the last batch, over the graph's
    edgeLen as the batches change it. parent is not computed (pass None), and weight must
    be None: the device copy's edgeLen is the propEdge the batches update."""
    if parent is not None or weight is not None:
        raise ValueError("DynSSSP: parent is not computed and weight must be None (edgeLen is used)")
    with DeviceGraph.from_csr(g) as dg:
        dg.sssp(int(src), out=dist)
        for t, s, d, w in _batches(updateBatch, batchSize):
            dg.sssp_dynamic(t, s, d, w, int(src), dist)


def DynCF(g: CSRGraph, updateBatch, cf: np.ndarray, batchSize: int) -> None:
    """dynamicBatchClustering DynCF: cf[V] after the last batch."""
    with DeviceGraph.from_csr(g) as dg:
        dg.clustering_coeff(out=cf)
        for t, s, d, w in _batches(updateBatch, batchSize):
            dg.clustering_coeff_dynamic(t, s, d, w, cf)


def DynDegree(g: CSRGraph, updateBatch, deg: np.ndarray, batchSize: int) -> None:
    """dynamicBatchDeg DynDegree: deg[V] (out-degrees) after the last batch."""
    with DeviceGraph.from_csr(g) as dg:
        dg.degree(out=deg)
        for t, s, d, w in _batches(updateBatch, batchSize):
            dg.degree_dynamic(t, s, d, w, out=deg)


def DynBC(g: CSRGraph, BC: np.ndarray, seeds, updateBatch, batchSize: int) -> None:
    """dynamicDecBC / dynamicBatchIncNorm / dynamicBatchDecNorm DynBC: BC[V] over seeds
    after the last batch."""
    with DeviceGraph.from_csr(g) as dg:
        src = np.array(sorted(seeds), np.int32)
        dg.bc(src, out=BC)
        for t, s, d, w in _batches(updateBatch, batchSize):
            dg.bc_dynamic(t, s, d, w, src, out=BC)
