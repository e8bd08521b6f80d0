"""GPU: PageRank split over ranks by vertices (sp_pagerank_part_*).

One GPU is available here, so N ranks are emulated in one process: N device graphs,
each with its own part plan and buffers, step through the iterations in lockstep, and
the exchange the ranks' collectives would do (the all-gather of the contrib blocks and
the sum of the diffs) is done by device copies between them. No kernel waits on another
part. The result must match the FP64 oracle at the same iteration count (L1 < 1e-6), as
the single-GPU PageRank does, and every part must stop at the same iteration."""
import numpy as np
import pytest

from oracle import oracle as O
from starplat_b200 import generators as G
from starplat_b200.device import DeviceGraph

from graphs import directed_zoo, from_pairs

pytestmark = pytest.mark.gpu


def run_parts(g, n, beta=1e-6, delta=0.85, max_iter=100):
    import torch

    S = -(-g.V // n)
    dgs = [DeviceGraph.from_csr(g, with_weights=False) for _ in range(n)]
    try:
        con = [[torch.empty(n * S, dtype=torch.float32, device="cuda") for _ in range(2)] for _ in range(n)]
        diff = [torch.zeros(1, dtype=torch.float64, device="cuda") for _ in range(n)]
        for r, dg in enumerate(dgs):
            dg.set_stream(torch.cuda.current_stream())
            assert dg.pagerank_part_begin(r, n, beta, delta, max_iter, con[r][0], con[r][1], diff[r]) == S
        k = 0
        while True:
            for dg in dgs:
                dg.pagerank_part_iterate(k)
            nxt = (k + 1) & 1
            for q in range(n):  # all-gather: part q's block to every part
                for r in range(n):
                    if r != q:
                        con[r][nxt][q * S:(q + 1) * S].copy_(con[q][nxt][q * S:(q + 1) * S])
            total = sum(d.clone() for d in diff)  # all-reduce of the diffs
            for d in diff:
                d.copy_(total)
            for dg in dgs:
                dg.pagerank_part_decide()
            k += 1
            states = [dg.pagerank_part_state() for dg in dgs]
            assert len({(s[0], s[1]) for s in states}) == 1, states
            if states[0][1]:
                break
            assert k <= max_iter
        full = torch.empty(n * S, dtype=torch.float32, device="cuda")
        for r, dg in enumerate(dgs):
            dg.pagerank_part_ranks(full[r * S:(r + 1) * S])
        out = np.empty(g.V, np.float32)
        dgs[0].pagerank_part_finish(full, out)
        return out, states[0][0], states[0][2]
    finally:
        for dg in dgs:
            dg.free()


def check(g, n):
    pr, it, diff = run_parts(g, n)
    exact, _, _ = O.pagerank(g.indexofNodes, g.rev_indexofNodes, g.srcList, 0.0, 0.85, it)
    l1 = float(np.abs(pr.astype(np.float64) - exact).sum())
    assert l1 < 1e-6, (g.name, n, l1)
    with DeviceGraph.from_csr(g, with_weights=False) as dg:
        _, it1, _ = dg.pagerank(1e-6, 0.85, 100)
    assert abs(it - it1) <= 1, (g.name, n, it, it1)
    return it


@pytest.mark.parametrize("n", [1, 2, 3, 8])
def test_pagerank_parts_match_the_oracle(n):
    for g in [G.rmat(14, 16, seed=3, directed=True), G.rmat(12, 8, seed=2), G.grid(30, 41)] + directed_zoo()[:2]:
        check(g, n)


def test_pagerank_parts_more_parts_than_vertices_and_hubs():
    # parts without rows (V < nparts) and a hub row cut into chunks owned by one part
    g = from_pairs(5, [[0, 1], [1, 2], [2, 0], [3, 0], [4, 0]], name="tiny")
    check(g, 8)
    leaves = np.arange(1, 6001, dtype=np.int32)
    star = from_pairs(6001, np.stack([leaves, np.zeros_like(leaves)], 1), name="star_in")
    check(star, 3)


def test_pagerank_on_gpus_single_rank_path():
    # the orchestration of distributed.pagerank_on_gpus with one rank (no process group)
    import torch

    from starplat_b200.distributed import pagerank_on_gpus
    from starplat_b200.replicas import Replicas

    g = G.rmat(13, 16, seed=5, directed=True)
    rep = Replicas()
    with DeviceGraph.from_csr(g, with_weights=False) as dg:
        out = torch.empty(g.V, dtype=torch.float32, device="cuda")
        pr, it, diff = pagerank_on_gpus(dg, rep, out=out, check_every=5)
        assert pr is out and diff <= 1e-6
    exact, _, _ = O.pagerank(g.indexofNodes, g.rev_indexofNodes, g.srcList, 0.0, 0.85, it)
    assert np.abs(out.cpu().numpy().astype(np.float64) - exact).sum() < 1e-6
