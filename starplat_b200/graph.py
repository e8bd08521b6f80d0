"""Host-side CSR graph in the layout of StarPlat's `graph` container.

Field names follow graphcode/graph.hpp:44-57 of the reference:
``indexofNodes`` / ``edgeList`` (forward CSR, adjacency sorted by destination),
``rev_indexofNodes`` / ``srcList`` (reverse CSR, sources sorted) and
``edgeLen`` (int32 edge weights in forward-CSR order). Arrays are int32 numpy
arrays; ``num_nodes()`` is the vertex count V (graph.hpp:139-142 returns max id
+ 1, which is V for every graph built here).
"""
from __future__ import annotations

import hashlib
from dataclasses import dataclass, field
from typing import Optional

import numpy as np


@dataclass
class CSRGraph:
    indexofNodes: np.ndarray
    edgeList: np.ndarray
    rev_indexofNodes: Optional[np.ndarray] = None
    srcList: Optional[np.ndarray] = None
    edgeLen: Optional[np.ndarray] = None
    name: str = "graph"
    meta: dict = field(default_factory=dict)

    def num_nodes(self) -> int:
        return int(self.indexofNodes.shape[0] - 1)

    def num_edges(self) -> int:
        return int(self.indexofNodes[-1])

    @property
    def V(self) -> int:
        return self.num_nodes()

    @property
    def E(self) -> int:
        return self.num_edges()

    def out_degree(self) -> np.ndarray:
        return np.diff(self.indexofNodes)

    def ensure_reverse(self) -> "CSRGraph":
        """Build the reverse CSR (graph.hpp:781-833) if it is missing."""
        if self.rev_indexofNodes is None or self.srcList is None:
            from . import generators

            self.rev_indexofNodes, self.srcList = generators.transpose(self.indexofNodes, self.edgeList)
        return self

    def is_symmetric(self) -> bool:
        self.ensure_reverse()
        return bool(
            np.array_equal(self.indexofNodes, self.rev_indexofNodes) and np.array_equal(self.edgeList, self.srcList)
        )

    def digest(self) -> str:
        """SHA-256 of the forward CSR (and weights), recorded with golden results."""
        h = hashlib.sha256()
        h.update(np.ascontiguousarray(self.indexofNodes, dtype=np.int32).tobytes())
        h.update(np.ascontiguousarray(self.edgeList, dtype=np.int32).tobytes())
        if self.edgeLen is not None:
            h.update(np.ascontiguousarray(self.edgeLen, dtype=np.int32).tobytes())
        return h.hexdigest()

    @staticmethod
    def from_edges(V: int, src, dst, *, symmetrize: bool = False, drop_self: bool = True,
                   name: str = "graph") -> "CSRGraph":
        from . import generators

        off, adj = generators.csr_from_edges(V, np.asarray(src, np.int32), np.asarray(dst, np.int32),
                                             symmetrize=symmetrize, drop_self=drop_self)
        g = CSRGraph(off, adj, name=name)
        g.ensure_reverse()
        return g
