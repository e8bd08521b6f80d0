"""Parity against the reference's own runnable GPU code, through fixtures it produced
on a B200 (tests/golden/make_gpu_fixtures.py; the binaries are compiled from the
reference's sources by oracle/Makefile):

* BC: the manual CUDA Brandes (graphcode/manual_cuda/bcManualv5.cu) halves every
  dependency (BC += delta / 2, :101-105); the generated OpenMP code does not. So twice
  the reference's vector is the generated semantics. Its FP64 sigma and delta make it an
  FP64 reference: the oracle matches it to 1e-12 relative (CPU test), and the GPU path
  within the BC tolerance (GPU test). The fixture's own launch order is pinned to the
  reference's unchanged main: the values that main prints (BC[0..8]) match.
* Louvain: the modularity of the partition the reference's CUDA Louvain
  (communitydetection_sequential_allocation.cu) returns, computed in FP64 on the
  original graph, against this library's Louvain (GPU test).

Every graph is rebuilt by the seeded generators named in the fixture script, and its
CSR digest is checked first."""
import json
import os

import numpy as np
import pytest

from oracle import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
FIX = os.path.join(HERE, "golden", "reference_gpu")

pytestmark = pytest.mark.skipif(not os.path.exists(os.path.join(FIX, "bc_manual.json")),
                                reason="reference GPU fixtures not generated")


def _fixture_module():
    import importlib.util

    spec = importlib.util.spec_from_file_location("make_gpu_fixtures", os.path.join(HERE, "golden",
                                                                                    "make_gpu_fixtures.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def _bc_cases():
    M = _fixture_module()
    meta = json.load(open(os.path.join(FIX, "bc_manual.json")))
    vec = np.load(os.path.join(FIX, "bc_manual.npz"))
    builders = {k: v[0] for k, v in M.BC_GRAPHS.items()}
    builders[M.BC_TEXT_GRAPH[0]] = M.BC_TEXT_GRAPH[1]
    out = []
    for name, m in meta.items():
        g = builders[name]()
        assert M.digest(g) == m["digest"], name
        out.append((name, g, np.array(m["sources"], np.int32), vec[name], m))
    return out


def test_oracle_bc_matches_the_reference_manual_cuda_bc():
    for name, g, srcs, ref_half, m in _bc_cases():
        ref = 2.0 * ref_half
        got = O.bc(g.indexofNodes, g.edgeList, srcs)
        assert np.all(np.abs(got - ref) <= 1e-12 * np.abs(ref) + 1e-12), name
        if "main_printed_bc_0_8" in m:  # the reference's own main printed these (%lf)
            assert np.allclose(ref_half[:9], m["main_printed_bc_0_8"], rtol=0, atol=5e-7), name


@pytest.mark.gpu
def test_gpu_bc_matches_the_reference_manual_cuda_bc():
    from starplat_b200.device import DeviceGraph

    for name, g, srcs, ref_half, _ in _bc_cases():
        ref = 2.0 * ref_half
        with DeviceGraph.from_csr(g, with_weights=False) as dg:
            got = dg.bc(srcs).astype(np.float64)
        bar = 1e-5 * np.abs(ref) + 1e-9 * max(1.0, ref.max())
        assert np.all(np.abs(got - ref) <= bar), (name, float((np.abs(got - ref) / bar).max()))
