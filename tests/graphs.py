"""Seeded small graphs shared by the CPU and GPU tests (sizes the oracle
finishes in well under a second)."""
from __future__ import annotations

import numpy as np

from starplat_b200 import generators as G
from starplat_b200.graph import CSRGraph


def from_pairs(V, pairs, symmetrize=False, name="g"):
    pairs = np.asarray(pairs, np.int32).reshape(-1, 2)
    return CSRGraph.from_edges(V, pairs[:, 0], pairs[:, 1], symmetrize=symmetrize, name=name)


def star(n_leaves: int, directed_in: bool = True) -> CSRGraph:
    """Hub 0; with directed_in every leaf points at the hub (in-degree n_leaves)."""
    leaves = np.arange(1, n_leaves + 1, dtype=np.int32)
    hub = np.zeros_like(leaves)
    if directed_in:
        return from_pairs(n_leaves + 1, np.stack([leaves, hub], 1), name=f"star_in{n_leaves}")
    return from_pairs(n_leaves + 1, np.stack([hub, leaves], 1), symmetrize=True, name=f"star{n_leaves}")


def clique(n: int) -> CSRGraph:
    i, j = np.triu_indices(n, 1)
    return from_pairs(n, np.stack([i, j], 1), symmetrize=True, name=f"K{n}")


def path(n: int) -> CSRGraph:
    a = np.arange(n - 1, dtype=np.int32)
    return from_pairs(n, np.stack([a, a + 1], 1), symmetrize=True, name=f"P{n}")


def empty(n: int) -> CSRGraph:
    return from_pairs(n, np.zeros((0, 2), np.int32), name=f"empty{n}")


def undirected_zoo():
    return [
        G.rmat(10, 8, seed=11),
        G.rmat(12, 16, seed=5),
        G.erdos_renyi(3000, 12, seed=7),
        G.grid(20, 30),
        clique(24),
        star(3000, directed_in=False),
        path(50),
        empty(7),
    ]


def directed_zoo():
    return [
        G.rmat(11, 8, seed=3, directed=True),
        G.rmat(12, 16, seed=9, directed=True),
        star(5000, directed_in=True),   # in-degree 5000 > one 2048-edge chunk
        from_pairs(6, [[0, 1], [1, 2], [2, 0], [0, 2], [3, 4], [4, 3], [5, 0]], name="small_dir"),
    ]
