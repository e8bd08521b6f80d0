"""ORACLE — test infrastructure only.

ctypes front end over ``oracle/libsporacle.so`` (the CPU restatement in
sp_oracle.cpp) and, when it was built in a reference checkout,
``oracle/_ref/libspref.so`` (the reference's own graph.hpp CSR container and
check_if_nbr, via ref_harness.cpp). Only tests, ``__graft_entry__.smoke()`` and
the CPU-baseline leg of ``bench.py`` import this module; the product path never
does.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")

_OR = None
_REF = None


def lib():
    global _OR
    if _OR is None:
        path = os.path.join(_HERE, "libsporacle.so")
        if not os.path.exists(path):
            raise RuntimeError(f"{path} missing: build it with `make -C oracle`")
        L = ctypes.CDLL(path)
        L.or_tc.restype = ctypes.c_int64
        L.or_tc.argtypes = [ctypes.c_int32, i32p, i32p, ctypes.c_int]
        L.or_lcc.restype = None
        L.or_lcc.argtypes = [ctypes.c_int32, i32p, i32p, i32p, ctypes.c_int]
        L.or_tc_omp.restype = ctypes.c_int64
        L.or_tc_omp.argtypes = [ctypes.c_int32, i32p, i32p, ctypes.c_int, ctypes.c_int32, ctypes.c_int32]
        L.or_pagerank.restype = ctypes.c_int32
        L.or_pagerank.argtypes = [ctypes.c_int32, i32p, i32p, i32p, ctypes.c_double, ctypes.c_double,
                                  ctypes.c_int32, ctypes.c_int32, f64p, ctypes.POINTER(ctypes.c_double),
                                  ctypes.c_int]
        L.or_pagerank_omp.restype = ctypes.c_int32
        L.or_pagerank_omp.argtypes = [ctypes.c_int32, i32p, i32p, i32p, ctypes.c_float, ctypes.c_float,
                                      ctypes.c_int32, f32p, ctypes.c_int]
        L.or_sssp.restype = ctypes.c_int32
        L.or_sssp.argtypes = [ctypes.c_int32, i32p, i32p, i32p, ctypes.c_int32, i32p]
        L.or_sssp_bf.restype = ctypes.c_int32
        L.or_sssp_bf.argtypes = [ctypes.c_int32, i32p, i32p, i32p, ctypes.c_int32, i32p]
        L.or_sssp_omp.restype = ctypes.c_int32
        L.or_sssp_omp.argtypes = [ctypes.c_int32, i32p, i32p, i32p, ctypes.c_int32, i32p, ctypes.c_int32,
                                  ctypes.c_int]
        L.or_bfs_sigma.restype = ctypes.c_int32
        L.or_bfs_sigma.argtypes = [ctypes.c_int32, i32p, i32p, ctypes.c_int32, i32p, f64p]
        L.or_bc.restype = None
        L.or_bc.argtypes = [ctypes.c_int32, i32p, i32p, i32p, ctypes.c_int32, f64p, ctypes.c_int]
        L.or_bc_omp.restype = None
        L.or_bc_omp.argtypes = [ctypes.c_int32, i32p, i32p, i32p, ctypes.c_int32, f32p, ctypes.c_int]
        L.or_louvain.restype = ctypes.c_double
        L.or_louvain.argtypes = [ctypes.c_int32, i32p, i32p, ctypes.c_void_p, ctypes.c_double, i32p,
                                 ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int32)]
        L.or_modularity.restype = ctypes.c_double
        L.or_modularity.argtypes = [ctypes.c_int32, i32p, i32p, ctypes.c_void_p, i32p]
        L.or_num_threads.restype = ctypes.c_int32
        _OR = L
    return _OR


def ref_lib() -> Optional[ctypes.CDLL]:
    """The reference-compiled harness, or None when it was not built."""
    global _REF
    if _REF is None:
        path = os.path.join(_HERE, "_ref", "libspref.so")
        if not os.path.exists(path):
            return None
        L = ctypes.CDLL(path)
        L.ref_parse_graph.restype = ctypes.c_void_p
        L.ref_parse_graph.argtypes = [ctypes.c_char_p]
        L.ref_graph_sizes.restype = None
        L.ref_graph_sizes.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int32)]
        L.ref_graph_copy.restype = None
        L.ref_graph_copy.argtypes = [ctypes.c_void_p, i32p, i32p, i32p, i32p, i32p, i32p]
        L.ref_lcc.restype = None
        L.ref_lcc.argtypes = [ctypes.c_int32, i32p, i32p, i32p]
        L.ref_tc.restype = ctypes.c_int64
        L.ref_tc.argtypes = [ctypes.c_int32, i32p, i32p, ctypes.c_int, ctypes.c_int32, ctypes.c_int32]
        _REF = L
    return _REF


def _c(a, dt=np.int32):
    return np.ascontiguousarray(a, dtype=dt)


def tc(off, adj, nthreads: int = 0) -> int:
    return int(lib().or_tc(len(off) - 1, _c(off), _c(adj), nthreads))


def tc_omp(off, adj, nthreads: int = 0, vfirst: int = 0, vstride: int = 1) -> int:
    return int(lib().or_tc_omp(len(off) - 1, _c(off), _c(adj), nthreads, vfirst, vstride))


def lcc(off, adj, nthreads: int = 0) -> np.ndarray:
    """staticClusteringCoeff (staticDSLCodes/clustering_coeff:1-14): per-vertex counts
    of the triangles the Compute_TC loop finds (int32)."""
    V = len(off) - 1
    cf = np.empty(V, np.int32)
    lib().or_lcc(V, _c(off), _c(adj), cf, nthreads)
    return cf


def degree(off) -> np.ndarray:
    """Degree (staticDSLCodes/degree_centrality:1-6): count_outNbrs(v), the out-degree."""
    return np.diff(np.asarray(off, np.int64)).astype(np.int32)


def closeness(off, adj, w, srcs) -> np.ndarray:
    """Compute_CC (staticDSLCodes/CC:1-26): CC[src] = 1.0 / (sum of the finite
    shortest-path distances from src) for every source, 0 elsewhere. The sum is kept
    in 64 bits (the DSL's int overflows past 2^31-1); 1.0 / sum is a double division
    stored as float, as the generated C++ does."""
    V = len(off) - 1
    cc = np.zeros(V, np.float32)
    for s in np.asarray(srcs, np.int64):
        d = sssp(off, adj, w, int(s)).astype(np.int64)
        tot = int(d[d != np.iinfo(np.int32).max].sum())
        cc[s] = np.float32(1.0 / tot) if tot != 0 else np.float32(np.inf)
    return cc


def closeness_unweighted(off, adj, srcs) -> np.ndarray:
    """Compute_CC_Unweighted (staticDSLCodes/closeness_centrality_unwt:1-20): dist starts
    at 0 everywhere and the BFS body sets w.dist = v.dist + 1 for each next-level w (the
    generator's bfsDist guard, backend_omp/dsl_cpp_generator.cpp:1461-1468), so dist is
    the BFS level of reached vertices and 0 elsewhere; CC[src] = 1.0 / sum of dist."""
    V = len(off) - 1
    cc = np.zeros(V, np.float32)
    for s in np.asarray(srcs, np.int64):
        lvl, _, _ = bfs_sigma(off, adj, int(s))
        tot = int(lvl[lvl > 0].astype(np.int64).sum())
        cc[s] = np.float32(1.0 / tot) if tot != 0 else np.float32(np.inf)
    return cc


def pagerank(off, roff, radj, beta=1e-6, delta=0.85, max_iter=100, fixed_iters=0, nthreads=0):
    V = len(off) - 1
    out = np.empty(V, np.float64)
    diff = ctypes.c_double(0)
    it = lib().or_pagerank(V, _c(off), _c(roff), _c(radj), beta, delta, max_iter, fixed_iters, out,
                           ctypes.byref(diff), nthreads)
    return out, int(it), float(diff.value)


def pagerank_omp(off, roff, radj, beta=1e-6, delta=0.85, max_iter=100, nthreads=0):
    V = len(off) - 1
    out = np.empty(V, np.float32)
    it = lib().or_pagerank_omp(V, _c(off), _c(roff), _c(radj), beta, delta, max_iter, out, nthreads)
    return out, int(it)


def sssp(off, adj, w, src: int) -> np.ndarray:
    V = len(off) - 1
    dist = np.empty(V, np.int32)
    rc = lib().or_sssp(V, _c(off), _c(adj), _c(w), src, dist)
    if rc == -2:
        rc = lib().or_sssp_bf(V, _c(off), _c(adj), _c(w), src, dist)
    if rc != 0:
        raise ValueError(f"oracle sssp failed ({rc})")
    return dist


def sssp_omp(off, adj, w, src: int, max_rounds: int = 0, nthreads: int = 0):
    V = len(off) - 1
    dist = np.empty(V, np.int32)
    rounds = lib().or_sssp_omp(V, _c(off), _c(adj), _c(w), src, dist, max_rounds, nthreads)
    return dist, int(rounds)


def bfs_sigma(off, adj, src: int):
    V = len(off) - 1
    lvl = np.empty(V, np.int32)
    sig = np.empty(V, np.float64)
    n = lib().or_bfs_sigma(V, _c(off), _c(adj), src, lvl, sig)
    return lvl, sig, int(n)


def bc(off, adj, srcs, nthreads: int = 0) -> np.ndarray:
    V = len(off) - 1
    out = np.empty(V, np.float64)
    s = _c(srcs)
    lib().or_bc(V, _c(off), _c(adj), s, s.shape[0], out, nthreads)
    return out


def bc_omp(off, adj, srcs, nthreads: int = 0) -> np.ndarray:
    V = len(off) - 1
    out = np.empty(V, np.float32)
    s = _c(srcs)
    lib().or_bc_omp(V, _c(off), _c(adj), s, s.shape[0], out, nthreads)
    return out


def louvain(off, adj, w=None, threshold: float = 1e-4, with_sweeps: bool = False):
    V = len(off) - 1
    comm = np.empty(V, np.int32)
    levels = ctypes.c_int32(0)
    sweeps = ctypes.c_int32(0)
    wp = None
    if w is not None:
        w = _c(w, np.float32)
        wp = w.ctypes.data
    q = lib().or_louvain(V, _c(off), _c(adj), wp, threshold, comm, ctypes.byref(levels), ctypes.byref(sweeps))
    if with_sweeps:
        return float(q), comm, int(levels.value), int(sweeps.value)
    return float(q), comm, int(levels.value)


def modularity(off, adj, comm, w=None) -> float:
    V = len(off) - 1
    wp = None
    if w is not None:
        w = _c(w, np.float32)
        wp = w.ctypes.data
    return float(lib().or_modularity(V, _c(off), _c(adj), wp, _c(comm)))


def num_threads() -> int:
    return int(lib().or_num_threads())


# ---- reference-compiled harness ------------------------------------------------

def ref_lcc(off, adj) -> Optional[np.ndarray]:
    """staticClusteringCoeff's generated loop over the reference's own check_if_nbr
    (None when the reference harness was not built)."""
    L = ref_lib()
    if L is None:
        return None
    V = len(off) - 1
    cf = np.empty(V, np.int32)
    L.ref_lcc(V, _c(off), _c(adj), cf)
    return cf


def ref_tc(off, adj, nthreads: int = 0, vfirst: int = 0, vstride: int = 1) -> int:
    L = ref_lib()
    if L is None:
        raise RuntimeError("oracle/_ref/libspref.so not built (needs the reference checkout)")
    return int(L.ref_tc(len(off) - 1, _c(off), _c(adj), nthreads, vfirst, vstride))


def ref_parse_graph(path: str):
    """Reference graph::parseGraph on a text edge list -> dict of CSR arrays."""
    L = ref_lib()
    if L is None:
        raise RuntimeError("oracle/_ref/libspref.so not built (needs the reference checkout)")
    h = L.ref_parse_graph(path.encode())
    V = ctypes.c_int32(0)
    E = ctypes.c_int32(0)
    L.ref_graph_sizes(h, ctypes.byref(V), ctypes.byref(E))
    V, E = V.value, E.value
    arrs = [np.empty(V + 1, np.int32), np.empty(max(E, 1), np.int32), np.empty(max(E, 1), np.int32),
            np.empty(V + 1, np.int32), np.empty(max(E, 1), np.int32), np.empty(max(E, 1), np.int32)]
    L.ref_graph_copy(h, *arrs)
    names = ["indexofNodes", "edgeList", "edgeLen", "rev_indexofNodes", "srcList", "edgeMap"]
    return {k: (a if k in ("indexofNodes", "rev_indexofNodes") else a[:E]) for k, a in zip(names, arrs)}


# ----------------------------------------------------------------------------- text edge lists

_WS = " \t\r\v\f"


def _read_int(line: str, i: int):
    """std::stringstream >> int32 at line[i:]: optional sign, digits up to the first other
    character. Returns (value, next index, status): status 0 ok, 1 no digits, 2 out of
    range (value saturated)."""
    j = i
    neg = False
    if j < len(line) and line[j] in "+-":
        neg = line[j] == "-"
        j += 1
    k = j
    while k < len(line) and "0" <= line[k] <= "9":
        k += 1
    if k == j:
        return 0, k, 1
    x = int(line[j:k])
    x = -x if neg else x
    if x > 2**31 - 1 or x < -2**31:
        return (-2**31 if neg else 2**31 - 1), k, 2
    return x, k, 0


def parse_edgelist(path: str):
    """graph::parseGraph (graph.hpp:464-512, :720-865) restated for small files: skip lines
    that are empty or do not start with a digit; "src dst weight" read as stringstream
    reads int32; V = largest id + 1; duplicate pairs summed (int32 wrap); self-loops kept;
    rows sorted; edgeMap[i] = forward index of reverse entry i. A line without a weight
    gets 1 (the reference leaves it uninitialised); an id that is missing, malformed,
    negative or out of range raises ValueError."""
    pairs = {}
    max_id = 0
    with open(path, "rb") as f:
        data = f.read().decode("latin-1")
    for ln, line in enumerate(data.split("\n"), 1):
        if not line or not ("0" <= line[0] <= "9"):
            continue
        s, i, st = _read_int(line, 0)
        if st:
            raise ValueError(f"line {ln}: source out of range")
        while i < len(line) and line[i] in _WS:
            i += 1
        d, i, st = _read_int(line, i)
        if st or d < 0:
            raise ValueError(f"line {ln}: bad destination")
        while i < len(line) and line[i] in _WS:
            i += 1
        w = 1
        if i < len(line):
            w, i, st = _read_int(line, i)
            if st == 1:
                w = 0
        if s == 2**31 - 1 or d == 2**31 - 1:
            raise ValueError(f"line {ln}: id too large")
        key = (s, d)
        pairs[key] = ((pairs.get(key, 0) + w + 2**31) % 2**32) - 2**31
        max_id = max(max_id, s, d)
    V = max_id + 1
    keys = sorted(pairs)
    E = len(keys)
    src = np.array([k[0] for k in keys], np.int64).reshape(-1)
    dst = np.array([k[1] for k in keys], np.int32).reshape(-1)
    w = np.array([pairs[k] for k in keys], np.int32).reshape(-1)
    off = np.zeros(V + 1, np.int32)
    np.add.at(off, src + 1, 1)
    off = np.cumsum(off).astype(np.int32)
    order = np.lexsort((src, dst))  # by dst, then src
    rev_src = src[order].astype(np.int32)
    roff = np.zeros(V + 1, np.int32)
    np.add.at(roff, dst.astype(np.int64) + 1, 1)
    roff = np.cumsum(roff).astype(np.int32)
    return {"indexofNodes": off, "edgeList": dst, "edgeLen": w, "rev_indexofNodes": roff, "srcList": rev_src,
            "edgeMap": order.astype(np.int32)}
