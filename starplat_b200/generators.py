"""Seeded synthetic graphs (R-MAT, 2-D grid, Erdos-Renyi, planted partition).

Thin ctypes front end over ``libspgen.so`` (csrc/spgen.cpp, host C++/OpenMP).
Each random draw is a pure function of (seed, index), so a graph is identical on
any machine and thread count. These stand in for the SNAP graphs the reference
mentions (not available offline), with the shapes of the benchmark configs.
"""
from __future__ import annotations

import ctypes
import math
import os

from typing import Optional

import numpy as np

from .graph import CSRGraph

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")


def _lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "libspgen.so")
        if not os.path.exists(path):
            raise RuntimeError(f"{path} is missing: run `python -c 'import __graft_entry__ as g; g.build()'`")
        L = ctypes.CDLL(path)
        L.spg_rmat_edges.restype = ctypes.c_int64
        L.spg_rmat_edges.argtypes = [ctypes.c_int, ctypes.c_int64, ctypes.c_double, ctypes.c_double,
                                     ctypes.c_double, ctypes.c_uint64, i32p, i32p]
        L.spg_er_edges.restype = ctypes.c_int64
        L.spg_er_edges.argtypes = [ctypes.c_int32, ctypes.c_int64, ctypes.c_uint64, i32p, i32p]
        L.spg_sbm_blocks.restype = ctypes.c_int32
        L.spg_sbm_blocks.argtypes = [ctypes.c_int32, ctypes.c_int32, ctypes.c_double, ctypes.c_int32,
                                     ctypes.c_uint64, i32p]
        L.spg_sbm_edges.restype = ctypes.c_int64
        L.spg_sbm_edges.argtypes = [ctypes.c_int32, ctypes.c_int32, i32p, ctypes.c_int64, ctypes.c_double,
                                    ctypes.c_uint64, i32p, i32p]
        L.spg_csr_from_edges.restype = ctypes.c_int64
        L.spg_csr_from_edges.argtypes = [ctypes.c_int32, ctypes.c_int64, i32p, i32p, ctypes.c_int, ctypes.c_int,
                                         i32p, i32p, ctypes.c_int64]
        L.spg_transpose.restype = None
        L.spg_transpose.argtypes = [ctypes.c_int32, ctypes.c_int64, i32p, i32p, i32p, i32p, ctypes.c_void_p]
        L.spg_weights_hash.restype = None
        L.spg_weights_hash.argtypes = [ctypes.c_int32, ctypes.c_int64, i32p, i32p, ctypes.c_uint64,
                                       ctypes.c_int32, ctypes.c_int32, ctypes.c_int, i32p]
        L.spg_grid.restype = ctypes.c_int64
        L.spg_grid.argtypes = [ctypes.c_int32, ctypes.c_int32, i32p, i32p]
        L.spg_num_threads.restype = ctypes.c_int32
        L.spg_write_edgelist.restype = ctypes.c_int64
        L.spg_write_edgelist.argtypes = [ctypes.c_char_p, ctypes.c_int32, i32p, i32p, ctypes.c_void_p]
        _LIB = L
    return _LIB


def csr_from_edges(V: int, src: np.ndarray, dst: np.ndarray, *, symmetrize: bool, drop_self: bool = True):
    src = np.ascontiguousarray(src, np.int32)
    dst = np.ascontiguousarray(dst, np.int32)
    M = src.shape[0]
    cap = 2 * M if symmetrize else M
    off = np.empty(V + 1, np.int32)
    adj = np.empty(max(cap, 1), np.int32)
    E = _lib().spg_csr_from_edges(V, M, src, dst, int(symmetrize), int(drop_self), off, adj, cap)
    if E < 0:
        raise ValueError("edge count does not fit int32 CSR offsets")
    return off, np.ascontiguousarray(adj[:E])


def transpose(off: np.ndarray, adj: np.ndarray, with_map: bool = False):
    off = np.ascontiguousarray(off, np.int32)
    adj = np.ascontiguousarray(adj, np.int32)
    V = off.shape[0] - 1
    E = int(off[-1])
    roff = np.empty(V + 1, np.int32)
    radj = np.empty(max(E, 1), np.int32)
    emap = np.empty(max(E, 1), np.int32) if with_map else None
    _lib().spg_transpose(V, E, off, adj, roff, radj, emap.ctypes.data if with_map else None)
    radj = radj[:E]
    if with_map:
        return roff, radj, emap[:E]
    return roff, radj


def hash_weights(g: CSRGraph, seed: int, wmin: int, wmax: int, symmetric: bool) -> np.ndarray:
    w = np.empty(max(g.E, 1), np.int32)
    _lib().spg_weights_hash(g.V, g.E, g.indexofNodes, g.edgeList, seed & 0xFFFFFFFFFFFFFFFF, wmin, wmax,
                            int(symmetric), w)
    return w[: g.E]


def rmat(scale: int, edge_factor: int = 16, a: float = 0.57, b: float = 0.19, c: float = 0.19,
         seed: int = 1, directed: bool = False) -> CSRGraph:
    """R-MAT graph on 2^scale vertices from edge_factor * 2^scale generated pairs.

    Undirected: symmetrised; directed: as generated. Self-loops and duplicates are
    removed, adjacency sorted, vertex ids as generated (no permutation).
    """
    V = 1 << scale
    M = edge_factor * V
    src = np.empty(M, np.int32)
    dst = np.empty(M, np.int32)
    _lib().spg_rmat_edges(scale, M, a, b, c, seed & 0xFFFFFFFFFFFFFFFF, src, dst)
    off, adj = csr_from_edges(V, src, dst, symmetrize=not directed, drop_self=True)
    del src, dst
    g = CSRGraph(off, adj, name=f"rmat{scale}{'d' if directed else 'u'}_ef{edge_factor}_s{seed}",
                 meta=dict(kind="rmat", scale=scale, edge_factor=edge_factor, a=a, b=b, c=c, seed=seed,
                           directed=directed))
    if not directed:
        g.rev_indexofNodes, g.srcList = off, adj
    else:
        g.ensure_reverse()
    return g


def grid(rows: int, cols: int) -> CSRGraph:
    """rows x cols 4-neighbour grid with edges in both directions."""
    V = rows * cols
    deg_total = 2 * ((rows - 1) * cols + rows * (cols - 1))
    off = np.empty(V + 1, np.int32)
    adj = np.empty(max(deg_total, 1), np.int32)
    E = _lib().spg_grid(rows, cols, off, adj)
    g = CSRGraph(off, adj[:E], name=f"grid{rows}x{cols}", meta=dict(kind="grid", rows=rows, cols=cols))
    g.rev_indexofNodes, g.srcList = g.indexofNodes, g.edgeList
    return g


def erdos_renyi(n: int, avg_degree: float, seed: int) -> CSRGraph:
    """Undirected G(n, m) with m = round(n * avg_degree / 2) uniform pairs (symmetrised, deduplicated)."""
    m = int(round(n * avg_degree / 2))
    src = np.empty(m, np.int32)
    dst = np.empty(m, np.int32)
    _lib().spg_er_edges(n, m, seed & 0xFFFFFFFFFFFFFFFF, src, dst)
    off, adj = csr_from_edges(n, src, dst, symmetrize=True, drop_self=True)
    g = CSRGraph(off, adj, name=f"er{n}_d{avg_degree:g}_s{seed}",
                 meta=dict(kind="er", n=n, avg_degree=avg_degree, seed=seed))
    g.rev_indexofNodes, g.srcList = off, adj
    return g


def sbm(V: int, nblocks: int, exponent: float = 2.0, avg_degree: float = 32.0, p_in: float = 0.8,
        seed: int = 1, min_size: int = 2) -> CSRGraph:
    """Undirected planted partition: power-law block sizes, every vertex of
    expected degree avg_degree, a fraction p_in of the edges inside blocks."""
    bs = np.empty(nblocks + 1, np.int32)
    if _lib().spg_sbm_blocks(V, nblocks, exponent, min_size, seed & 0xFFFFFFFFFFFFFFFF, bs) != 0:
        raise ValueError("invalid SBM block parameters")
    m = int(round(V * avg_degree / 2))
    src = np.empty(m, np.int32)
    dst = np.empty(m, np.int32)
    _lib().spg_sbm_edges(V, nblocks, bs, m, p_in, seed & 0xFFFFFFFFFFFFFFFF, src, dst)
    off, adj = csr_from_edges(V, src, dst, symmetrize=True, drop_self=True)
    g = CSRGraph(off, adj, name=f"sbm{V}_b{nblocks}_s{seed}",
                 meta=dict(kind="sbm", V=V, nblocks=nblocks, exponent=exponent, avg_degree=avg_degree,
                           p_in=p_in, seed=seed, block_start=bs))
    g.rev_indexofNodes, g.srcList = off, adj
    return g


def er_batch(count: int, n_min: int, n_max: int, deg_min: float, deg_max: float, seed: int):
    """`count` independent ER graphs, n log-uniform in [n_min, n_max], average
    degree uniform in [deg_min, deg_max] (seeded)."""
    rng = np.random.default_rng(seed)
    ns = np.exp(rng.uniform(math.log(n_min), math.log(n_max), size=count)).round().astype(np.int64)
    ds = rng.uniform(deg_min, deg_max, size=count)
    seeds = rng.integers(1, 2**62, size=count)
    return [erdos_renyi(int(n), float(d), int(s)) for n, d, s in zip(ns, ds, seeds)]


def pick_sources(g: CSRGraph, count: int, seed: int, min_out_degree: int = 1) -> np.ndarray:
    """`count` distinct seeded source vertices among those with out-degree >= min_out_degree."""
    cand = np.nonzero(g.out_degree() >= min_out_degree)[0].astype(np.int32)
    rng = np.random.default_rng(seed)
    count = min(count, cand.shape[0])
    return np.sort(rng.choice(cand, size=count, replace=False)).astype(np.int32)


def num_threads() -> int:
    return int(_lib().spg_num_threads())


def write_edgelist(g: CSRGraph, path: str, weights: Optional[np.ndarray] = None) -> int:
    """Writes g as a text edge list ("src dst weight" per line, CSR order), the format
    graph::parseGraph reads; weight 1 where no weights are given. Returns the bytes."""
    w = None if weights is None else np.ascontiguousarray(weights, np.int32)
    n = _lib().spg_write_edgelist(os.fsencode(path), g.V, g.indexofNodes, g.edgeList,
                                  None if w is None else w.ctypes.data)
    if n < 0:
        raise OSError(f"cannot write {path}")
    return int(n)
