"""GPU: single-source SSSP split over ranks by vertices (sp_sssp_part_*).

One GPU is available here, so N ranks are emulated in one process: N device graphs,
each with its own part, step through the rounds in lockstep, and the exchange the
ranks' collectives would do (the all-to-all of the counts and of the (vertex, distance)
pairs, the sum of the frontier sizes, the minimum of the far distances, the minimum of
the dist vectors) is done by device copies and reductions between them. No kernel waits
on another part. Distances must equal the oracle's bit for bit."""
import numpy as np
import pytest

from oracle import oracle as O
from starplat_b200 import _lib
from starplat_b200 import generators as G
from starplat_b200.device import DeviceGraph

from graphs import directed_zoo, from_pairs, star, undirected_zoo

pytestmark = pytest.mark.gpu
INT_MAX = 2**31 - 1


def weighted(g, lo, hi, seed=3):
    g.edgeLen = G.hash_weights(g, seed, lo, hi, g.is_symmetric())
    return g


def run_parts(g, n, src, delta=0, weight=None):
    import torch

    dgs = [DeviceGraph.from_csr(g) for _ in range(n)]
    try:
        stream = torch.cuda.current_stream()
        caps = []
        for r, dg in enumerate(dgs):
            dg.set_stream(stream)
            caps.append(dg.sssp_part_begin(r, n, src, weight, delta))
        cap = caps[0]
        assert all(c == cap for c in caps) and cap == -(-g.V // n)
        send = [torch.empty((n * cap, 2), dtype=torch.int32, device="cuda") for _ in range(n)]
        recv = [torch.empty((n * cap, 2), dtype=torch.int32, device="cuda") for _ in range(n)]
        sc = [torch.zeros(n, dtype=torch.int32, device="cuda") for _ in range(n)]
        fr = [torch.zeros(1, dtype=torch.int32, device="cuda") for _ in range(n)]
        far = [torch.zeros(1, dtype=torch.int32, device="cuda") for _ in range(n)]
        rounds = buckets = 0
        while True:
            while True:
                for r in range(n):
                    dgs[r].sssp_part_relax(send[r], sc[r])
                counts = [c.tolist() for c in sc]  # counts[q][r]: pairs q sends to r
                assert all(counts[q][q] == 0 for q in range(n))
                for r in range(n):
                    at = 0
                    for q in range(n):
                        off = sum(counts[q][:r])
                        k = counts[q][r]
                        if k:
                            recv[r][at:at + k].copy_(send[q][off:off + k])
                        at += k
                    dgs[r].sssp_part_apply(recv[r], at, fr[r])
                rounds += 1
                if sum(int(f.item()) for f in fr) == 0:
                    break
                assert rounds < 4 * g.V + 100
            for r in range(n):
                dgs[r].sssp_part_far_min(far[r])
            m = min(int(f.item()) for f in far)
            if m == INT_MAX:
                break
            for r in range(n):
                far[r].fill_(m)
                dgs[r].sssp_part_advance(far[r], fr[r])
            buckets += 1
        dist = np.full(g.V, INT_MAX, np.int64)
        for r, dg in enumerate(dgs):
            part = np.empty(g.V, np.int32)
            dg.sssp_part_dist(part)
            own = np.arange(g.V) % n == r
            assert np.all(part[~own] == INT_MAX)
            dist = np.minimum(dist, part)
        return dist, rounds, buckets
    finally:
        for dg in dgs:
            dg.free()


def check(g, n, src, **kw):
    dist, rounds, buckets = run_parts(g, n, src, **kw)
    w = kw.get("weight")
    ref = O.sssp(g.indexofNodes, g.edgeList, g.edgeLen if w is None else w, src)
    assert np.array_equal(dist, ref), (g.name, n, src, int((dist != ref).sum()))
    return rounds, buckets


@pytest.mark.parametrize("n", [1, 2, 3, 8])
def test_sssp_parts_match_the_oracle(n):
    cases = [weighted(G.rmat(13, 16, seed=3, directed=True), 1, 100), weighted(G.grid(40, 50), 1, 1000),
             weighted(G.rmat(12, 8, seed=2), 1, 1000)] + [weighted(g, 1, 100) for g in directed_zoo()[:2]]
    for g in cases:
        for src in G.pick_sources(g, 2, seed=n):
            check(g, n, int(src))


@pytest.mark.parametrize("delta", [1, 7, 1000, 2**40])
def test_sssp_parts_any_bucket_width(delta):
    g = weighted(G.rmat(12, 16, seed=5, directed=True), 1, 100)
    r1, b1 = check(g, 3, int(G.pick_sources(g, 1, seed=1)[0]), delta=delta)
    if delta == 2**40:
        assert b1 == 0  # one bucket: rounds only


def test_sssp_parts_edge_cases():
    # unreachable vertices, zero weights, more parts than vertices, a hub, device weights
    import torch

    g = from_pairs(6, [[0, 1], [1, 2], [3, 4]], name="broken")
    g.edgeLen = np.array([0, 5, 2], np.int32)
    for n in (1, 2, 8):
        check(g, n, 0)
        check(g, n, 3)
    s = weighted(star(3000, directed_in=False), 1, 9)
    check(s, 4, 0)
    check(s, 4, 17)
    u = weighted(undirected_zoo()[3], 1, 1000)
    wdev = torch.from_numpy(np.ascontiguousarray(G.hash_weights(u, 11, 1, 50, True))).cuda()
    dist, _, _ = run_parts(u, 3, 0, weight=wdev)
    assert np.array_equal(dist, O.sssp(u.indexofNodes, u.edgeList, wdev.cpu().numpy(), 0))


def test_sssp_parts_negative_weights_and_cycle():
    rng = np.random.default_rng(5)
    n = 300
    pairs = np.array([(i, j) for i in range(n) for j in rng.choice(n, 4) if i < j], np.int32)
    g = from_pairs(n, pairs, name="dag_parts")
    g.edgeLen = rng.integers(-40, 100, g.E).astype(np.int32)
    for parts in (1, 3):
        check(g, parts, 0)
    c = from_pairs(3, [[0, 1], [1, 2], [2, 0]], name="negcycle_parts")
    c.edgeLen = np.array([1, -5, 1], np.int32)
    with pytest.raises(_lib.SPError) as ei:
        run_parts(c, 2, 0)
    assert ei.value.status == -6


def test_sssp_parts_reject_bad_calls_and_foreign_messages():
    import torch

    g = weighted(G.grid(8, 8), 1, 9)
    with DeviceGraph.from_csr(g) as dg:
        dg.set_stream(torch.cuda.current_stream())
        with pytest.raises(_lib.SPError):
            dg.sssp_part_relax(torch.empty((2, 2), dtype=torch.int32, device="cuda"),
                               torch.zeros(2, dtype=torch.int32, device="cuda"))  # not begun
        with pytest.raises(_lib.SPError):
            dg.sssp_part_begin(2, 2, 0)  # part out of range
        with pytest.raises(_lib.SPError):
            dg.sssp_part_begin(0, 2, g.V)  # source out of range
        cap = dg.sssp_part_begin(0, 2, 0)
        fr = torch.zeros(1, dtype=torch.int32, device="cuda")
        # a pair for vertex 1, which part 1 owns, handed to part 0: flagged, reported
        msg = torch.tensor([[1, 5]], dtype=torch.int32, device="cuda")
        dg.sssp_part_apply(msg, 1, fr)
        with pytest.raises(_lib.SPError) as ei:
            dg.sssp_part_dist(np.empty(g.V, np.int32))
        assert ei.value.status == -1
        with pytest.raises(_lib.SPError):
            dg.sssp_part_apply(msg, 2 * cap + 1, fr)  # more pairs than any part can receive


def test_sssp_on_gpus_single_rank_path():
    # the orchestration of distributed.sssp_on_gpus with one rank (no process group)
    import torch

    from starplat_b200.distributed import sssp_on_gpus
    from starplat_b200.replicas import Replicas

    g = weighted(G.rmat(13, 16, seed=5, directed=True), 1, 100)
    src = int(G.pick_sources(g, 1, seed=2)[0])
    with DeviceGraph.from_csr(g) as dg:
        out = torch.empty(g.V, dtype=torch.int32, device="cuda")
        d, rounds = sssp_on_gpus(dg, Replicas(), src, out=out)
        assert d is out and rounds > 0
    assert np.array_equal(out.cpu().numpy(), O.sssp(g.indexofNodes, g.edgeList, g.edgeLen, src))
