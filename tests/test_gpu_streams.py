"""GPU: stream order between the library and torch.

A graph's own stream is a blocking stream, so device inputs that torch writes on its
default (legacy) stream are seen by the library without a synchronisation; and
set_stream(torch.cuda.current_stream()) puts the library's kernels on that legacy
stream itself. Each case delays torch's write with a spin kernel (torch.cuda._sleep,
a fixed number of clock cycles) so that a library kernel not ordered after it would
read the stale buffer."""
import numpy as np
import pytest

from oracle import oracle as O
from starplat_b200 import generators as G
from starplat_b200.device import DeviceGraph

pytestmark = pytest.mark.gpu

SPIN = 20_000_000  # cycles, about 10 ms


def _weighted():
    g = G.rmat(12, 8, seed=4, directed=True)
    g.edgeLen = G.hash_weights(g, 9, 1, 100, False)
    return g


def _late_copy(src):
    import torch

    dst = torch.zeros_like(src)
    torch.cuda._sleep(SPIN)
    dst.copy_(src)
    return dst


@pytest.mark.parametrize("on_torch_stream", [False, True])
def test_device_weights_written_late_on_torch_default_stream(on_torch_stream):
    import torch

    g = _weighted()
    exact = O.sssp(g.indexofNodes, g.edgeList, g.edgeLen, 0)
    w_true = torch.from_numpy(np.ascontiguousarray(g.edgeLen, np.int32)).cuda()
    torch.cuda.synchronize()
    with DeviceGraph.from_csr(g) as dg:
        if on_torch_stream:
            dg.set_stream(torch.cuda.current_stream())
        for _ in range(3):
            w = _late_copy(w_true)
            d, _ = dg.sssp(0, weight=w)
            assert np.array_equal(d, exact)


def test_pagerank_parts_exchange_delayed_on_torch_stream():
    # the all-gather and diff sum of a one-part split run, each behind a spin kernel on
    # torch's default stream; the library's iterate / decide must wait for them
    import torch

    g = G.rmat(13, 16, seed=3, directed=True)
    with DeviceGraph.from_csr(g, with_weights=False) as dg:
        _, it1, _ = dg.pagerank(1e-6, 0.85, 100)
    with DeviceGraph.from_csr(g, with_weights=False) as dg:
        dg.set_stream(torch.cuda.current_stream())
        con = [torch.empty(g.V, dtype=torch.float32, device="cuda") for _ in range(2)]
        diff = torch.zeros(1, dtype=torch.float64, device="cuda")
        dg.pagerank_part_begin(0, 1, 1e-6, 0.85, 100, con[0], con[1], diff)
        k = 0
        while True:
            dg.pagerank_part_iterate(k)
            torch.cuda._sleep(SPIN // 10)
            diff.copy_(diff.clone())  # the one-rank "sum", behind the spin
            dg.pagerank_part_decide()
            k += 1
            it, done, _ = dg.pagerank_part_state()
            assert it == k
            if done:
                break
        assert abs(it - it1) <= 1, (it, it1)
