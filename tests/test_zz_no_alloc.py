"""sp_pagerank_noalloc: the PageRank entry point for callers that cannot allocate
device memory (an engine owning all GPU memory through its own pool, a process
under a hard memory cap, a caller that cannot take an allocation's implicit
device synchronisation). It works only in the caller's buffers plus a fixed
scratch array compiled into the library, so its result must equal the
allocating entry point's (sp_pagerank) within the PageRank tolerance used
everywhere in these tests (L1 < 1e-6), call after call: the scratch keeps the
previous call's contents, and each call must clear what it relies on.

Collected last (file name) so a run that stops at the first failure has already
run every other test; it also passes alone in a fresh process."""
import ctypes

import numpy as np
import pytest

from oracle import oracle as O
from starplat_b200 import _lib
from starplat_b200 import generators as G
from starplat_b200.device import DeviceGraph

pytestmark = pytest.mark.gpu

MAX_V = 1 << 20


def _noalloc(off, roff, radj, V, E, beta, delta, max_iter, out):
    it = ctypes.c_int32(-1)
    rc = _lib.lib().sp_pagerank_noalloc(off.data_ptr(), roff.data_ptr(), radj.data_ptr(), V, E, beta, delta,
                                        max_iter, out.data_ptr(), ctypes.byref(it), None)
    return rc, it.value


def test_pagerank_noalloc_matches_allocating_entry_point():
    import torch

    torch.cuda.set_device(0)
    g = G.rmat(16, 16, seed=3, directed=True)
    assert g.V <= MAX_V
    with DeviceGraph.from_csr(g) as dg:
        ref, ref_it, _ = dg.pagerank(1e-6, 0.85, 100)
    # the FP64 oracle at the allocating path's iteration count
    exact, _, _ = O.pagerank(g.indexofNodes, g.rev_indexofNodes, g.srcList, 0.0, 0.85, ref_it)
    off = torch.from_numpy(g.indexofNodes).cuda()
    roff = torch.from_numpy(g.rev_indexofNodes).cuda()
    radj = torch.from_numpy(g.srcList).cuda()
    torch.cuda.synchronize()
    for call in range(2):  # the second call starts from the first call's scratch contents
        out = torch.full((g.V,), float("nan"), dtype=torch.float32, device="cuda")
        rc, it = _noalloc(off, roff, radj, g.V, g.E, 1e-6, 0.85, 100, out)
        assert rc == 0, _lib.lib().sp_last_error()
        got = out.cpu().numpy()
        assert it == ref_it, (call, it, ref_it)
        assert np.isfinite(got).all()
        assert np.abs(got.astype(np.float64) - ref.astype(np.float64)).sum() < 1e-6, call
        assert np.abs(got.astype(np.float64) - exact).sum() < 1e-6, call


def test_pagerank_noalloc_rejects_a_malformed_csr():
    # the device check runs before any gather, so a bad srcList entry or a decreasing
    # offset is reported instead of read through (the bad id here is V itself, and the
    # bad offsets only shrink rows)
    import torch

    g = G.rmat(8, 4, seed=2, directed=True)
    off = torch.from_numpy(g.indexofNodes).cuda()
    roff = torch.from_numpy(g.rev_indexofNodes).cuda()
    out = torch.zeros(g.V, dtype=torch.float32, device="cuda")
    bad_src = g.srcList.copy()
    bad_src[g.E // 2] = g.V
    rc, _ = _noalloc(off, roff, torch.from_numpy(bad_src).cuda(), g.V, g.E, 1e-6, 0.85, 10, out)
    assert rc == _lib.SP_ERR_INVALID_CODE
    assert b"srcList" in _lib.lib().sp_last_error()
    r = g.rev_indexofNodes.copy()
    k = int(np.flatnonzero((r[:-1] > 0) & (np.diff(r) > 0))[0])  # a row with in-edges, not the first
    r[k + 1] = r[k] - 1  # its end moves below its start
    rc, _ = _noalloc(off, torch.from_numpy(r).cuda(), torch.from_numpy(g.srcList).cuda(), g.V, g.E, 1e-6,
                     0.85, 10, out)
    assert rc == _lib.SP_ERR_INVALID_CODE
    assert b"rev_indexofNodes" in _lib.lib().sp_last_error()
    # a good call right after the failures still matches the oracle
    rc, it = _noalloc(off, roff, torch.from_numpy(g.srcList).cuda(), g.V, g.E, 1e-6, 0.85, 100, out)
    assert rc == 0
    exact, _, _ = O.pagerank(g.indexofNodes, g.rev_indexofNodes, g.srcList, 0.0, 0.85, it)
    assert np.abs(out.cpu().numpy().astype(np.float64) - exact).sum() < 1e-6


def test_pagerank_noalloc_rejects_graphs_above_its_scratch():
    import torch

    x = torch.zeros(4, dtype=torch.int32, device="cuda")
    out = torch.zeros(4, dtype=torch.float32, device="cuda")
    rc, _ = _noalloc(x, x, x, MAX_V + 1, 1, 1e-6, 0.85, 10, out)
    assert rc == _lib.SP_ERR_INVALID_CODE
    assert b"outside" in _lib.lib().sp_last_error()
