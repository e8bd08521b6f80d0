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
