"""GPU: the autotuner times every knob candidate on the caller's graph, leaves the
fastest set, and results stay exact (TC counts, SSSP distances) or within tolerance
(BC) under the chosen setting."""
import numpy as np
import pytest

from oracle import oracle as O
from starplat_b200 import autotune
from starplat_b200 import generators as G
from starplat_b200.device import DeviceGraph

pytestmark = pytest.mark.gpu


def _check_table(dg, table, algo):
    space = autotune.KNOBS[algo]
    assert len(table) == int(np.prod([len(v) for v in space.values()]))
    times = [t for _, t in table]
    assert times == sorted(times) and times[0] > 0
    for k, v in table[0][0].items():
        assert dg.tune_get(k) == v


def test_tune_tc_sssp_bc():
    import torch

    stream = torch.cuda.current_stream()
    g = G.rmat(13, 16, seed=9)
    g.edgeLen = G.hash_weights(g, 9, 1, 100, True)
    with DeviceGraph.from_csr(g) as dg:
        dg.set_stream(stream)
        table = autotune.tune(dg, "tc", reps=2)
        _check_table(dg, table, "tc")
        assert dg.tc() == O.tc(g.indexofNodes, g.edgeList)

        table = autotune.tune(dg, "sssp", reps=2, src=3)
        _check_table(dg, table, "sssp")
        assert np.array_equal(dg.sssp(3)[0], O.sssp(g.indexofNodes, g.edgeList, g.edgeLen, 3))

        srcs = G.pick_sources(g, 40, seed=2)
        table = autotune.tune(dg, "bc", reps=2, sources=srcs)
        _check_table(dg, table, "bc")
        out = dg.bc(srcs).astype(np.float64)
        ref = O.bc(g.indexofNodes, g.edgeList, srcs)
        assert np.all(np.abs(out - ref) <= 1e-5 * np.abs(ref) + 1e-9 * max(1.0, ref.max()))


def test_tune_rejects_unknown_algorithm():
    with pytest.raises(ValueError):
        autotune.tune(None, "louvain")
