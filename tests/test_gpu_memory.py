"""The library's device block cache: memory released by graph handles and plans is
kept (bounded) and reused by the next handle, results do not depend on whether a
block came from the cache, and sp_cache_trim hands it all back."""
import ctypes

import numpy as np
import pytest

from oracle import oracle as O
from starplat_b200 import _lib
from starplat_b200 import generators as G
from starplat_b200.device import DeviceGraph

pytestmark = pytest.mark.gpu


def _cached():
    b = ctypes.c_int64(-1)
    assert _lib.lib().sp_cache_bytes(ctypes.byref(b)) == 0
    return b.value


def _trim():
    b = ctypes.c_int64(-1)
    assert _lib.lib().sp_cache_trim(ctypes.byref(b)) == 0
    return b.value


def test_released_blocks_are_reused_and_trimmed():
    import torch

    torch.cuda.set_device(0)
    g = G.rmat(14, 16, seed=5, directed=True)
    ref, rit, _ = O.pagerank(g.indexofNodes, g.rev_indexofNodes, g.srcList, 1e-6, 0.85, 100)
    _trim()
    assert _cached() == 0
    outs = []
    for _ in range(3):  # the 2nd and 3rd handles are built from cached blocks
        with DeviceGraph.from_csr(g) as dg:
            out, it, _ = dg.pagerank(1e-6, 0.85, 100)
            tc = dg.tc()
        outs.append((out, it, tc))
        assert _cached() > 4 * g.E  # at least the CSR arrays were kept
    for out, it, tc in outs:
        assert abs(it - rit) <= 2
        assert np.abs(out.astype(np.float64) - ref).sum() < 1e-6
        assert tc == outs[0][2]
        assert np.array_equal(out, outs[0][0])
    freed = _trim()
    assert freed > 0 and _cached() == 0
    with DeviceGraph.from_csr(g) as dg:  # fresh allocations after a trim
        assert dg.tc() == outs[0][2]
