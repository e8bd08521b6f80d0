"""ORACLE — test infrastructure only.

Pure-Python restatements, for small graphs, of the batch bodies of two of StarPlat's
dynamic DSL programs, as the DSL text states them:

* DynTC (dynamicDSLCodes/dynamicBatchTCV2): Decremental (:84-140) on the graph before
  the batch, with the deleted edges marked (OnDelete, :155-167), then updateCSRDel /
  updateCSRAdd (:172-174), then Incremental (:24-81) on the new graph with the added
  edges marked (OnAdd, :179-192). Each body walks, for every update (v1, v2), the
  neighbours v3 of v1 (v3 != v1, v2 and v1 != v2) that are also neighbours of v2,
  classes each triangle by how many of its edges (v1, v3), (v2, v3) are marked, and
  moves the count by count1/2 + count2/4 + count3/6.
* DynCF (dynamicDSLCodes/dynamicBatchClustering): Decremental (:16-28) and Incremental
  (:30-42) add -1 / +1 to cf of v1, v2 and every v3 in N(v1) with (v2, v3) an edge.

The tests use them to check where the DSL's arithmetic agrees with an exact recount (the
batches the library's incremental paths are exact on by construction) and to record
where it does not. The product never imports this module.
"""
from __future__ import annotations

from typing import List, Set, Tuple

Edge = Tuple[int, int]
Update = Tuple[str, int, int]


def _nbrs(edges: Set[Edge], V: int) -> List[List[int]]:
    n: List[List[int]] = [[] for _ in range(V)]
    for a, b in sorted(edges):
        n[a].append(b)
    return n


def apply_batch(edges: Set[Edge], batch: List[Update]) -> Set[Edge]:
    """updateCSRDel then updateCSRAdd on an edge set (no parallel edges)."""
    out = set(edges)
    for t, a, b in batch:
        if t == "d":
            out.discard((a, b))
    for t, a, b in batch:
        if t == "a":
            out.add((a, b))
    return out


def _tc_body(edges: Set[Edge], V: int, updates: List[Edge], marked: Set[Edge]) -> int:
    n = _nbrs(edges, V)
    c1 = c2 = c3 = 0
    for v1, v2 in updates:
        if v1 == v2:
            continue
        for v3 in n[v1]:
            if v3 == v2 or v3 == v1:
                continue
            new_edge = 1 + ((v1, v3) in marked)
            if (v2, v3) in edges:
                new_edge += (v2, v3) in marked
                if new_edge == 1:
                    c1 += 1
                elif new_edge == 2:
                    c2 += 1
                else:
                    c3 += 1
    return c1 // 2 + c2 // 4 + c3 // 6


def dyn_tc_dsl(V: int, edges: Set[Edge], count: int, batch: List[Update]) -> Tuple[int, Set[Edge]]:
    """DynTC's Batch block: (new count, new edge set)."""
    dels = [(a, b) for t, a, b in batch if t == "d"]
    adds = [(a, b) for t, a, b in batch if t == "a"]
    marked_del = {(a, b) for a, b in dels if (a, b) in edges}  # OnDelete marks existing edges
    count -= _tc_body(edges, V, dels, marked_del)
    new = apply_batch(edges, batch)
    marked_add = {(a, b) for a, b in adds if (a, b) in new}
    count += _tc_body(new, V, adds, marked_add)
    return count, new


def dyn_cf_dsl(V: int, edges: Set[Edge], cf: List[int], batch: List[Update]) -> Tuple[List[int], Set[Edge]]:
    """DynCF's Batch block: (new cf, new edge set)."""
    cf = list(cf)

    def body(es: Set[Edge], ups: List[Edge], sign: int) -> None:
        n = _nbrs(es, V)
        for v1, v2 in ups:
            for v3 in n[v1]:
                if (v2, v3) in es:
                    cf[v1] += sign
                    cf[v2] += sign
                    cf[v3] += sign

    body(edges, [(a, b) for t, a, b in batch if t == "d"], -1)
    new = apply_batch(edges, batch)
    body(new, [(a, b) for t, a, b in batch if t == "a"], +1)
    return cf, new


def csr(V: int, edges: Set[Edge]):
    """Sorted CSR arrays (numpy int32) of an edge set."""
    import numpy as np

    keys = sorted(edges)
    off = np.searchsorted(np.array([a for a, _ in keys], np.int64), np.arange(V + 1)).astype(np.int32)
    return off, np.array([b for _, b in keys], np.int32)
