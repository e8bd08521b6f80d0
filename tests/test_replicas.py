"""Multi-rank plumbing on the CPU: two gloo ranks run the replica collectives the
benchmark uses on N GPUs (barrier, max of the device time over ranks, sum of the
units processed), and the reference arm under torchrun prints one line, from rank 0."""
import json
import os
import socket
import subprocess
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "RANK": str(rank),
                       "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank)})
    sys.path.insert(0, ROOT)
    from starplat_b200.replicas import Replicas

    rep = Replicas(backend="gloo", timeout_s=60)
    rep.barrier()
    res = {
        "rank": rep.rank, "world": rep.world, "root": rep.is_root,
        "max": rep.max(1.5 * (rank + 1)),  # rank 1 is the slow one
        "sum": rep.sum(rank + 1),
        # rank r processed 10 (r + 1) units in r + 1 seconds: 30 units / 2 s
        "rate": rep.whole_job_rate(10 * (rank + 1), rank + 1.0),
    }
    rep.barrier()
    rep.close()
    with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
        json.dump(res, f)


def test_two_gloo_ranks_reduce_like_the_benchmark(tmp_path):
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    res = [json.load(open(tmp_path / f"rank{r}.json")) for r in range(world)]
    for r, d in enumerate(res):
        assert (d["rank"], d["world"], d["root"]) == (r, world, r == 0)
        assert d["max"] == 3.0 and d["sum"] == 3.0 and d["rate"] == 15.0


def test_single_process_needs_no_process_group(monkeypatch):
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    from starplat_b200.replicas import Replicas

    rep = Replicas()
    rep.barrier()
    assert (rep.world, rep.max(2.5), rep.sum(4), rep.whole_job_rate(8, 2.0)) == (1, 2.5, 4.0, 4.0)
    rep.close()


@pytest.mark.timeout(600)
def test_reference_arm_under_torchrun_prints_once_from_rank_zero():
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes", "1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()), "bench.py", "--impl", "reference",
           "--gpus", "2", "--scale", "12", "--steps", "1", "--warmup", "1"]
    out = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=550)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [json.loads(x) for x in out.stdout.splitlines() if x.startswith("{")]
    assert len(lines) == 1
    line = lines[0]
    assert line["impl"] == "reference" and line["n_gpus"] == 2 and line["value"] > 0
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["cpu_baseline"]["kind"] in ("port", "reference")


def _bc_rank_main(rank, world, port, out_dir):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "RANK": str(rank),
                       "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank)})
    sys.path.insert(0, ROOT)
    import numpy as np

    from oracle import oracle as O
    from starplat_b200 import generators as G
    from starplat_b200.distributed import bc_sharded, split_sources
    from starplat_b200.replicas import Replicas

    g = G.rmat(9, 8, seed=4)
    srcs = G.pick_sources(g, 37, seed=1)
    rep = Replicas(backend="gloo", timeout_s=60)
    mine = split_sources(srcs, world, rank)
    out = bc_sharded(g.V, srcs, rep, lambda s: O.bc(g.indexofNodes, g.edgeList, s).astype(np.float32))
    rep.close()
    np.save(os.path.join(out_dir, f"bc{rank}.npy"), out)
    np.save(os.path.join(out_dir, f"src{rank}.npy"), mine)


@pytest.mark.parametrize("world", [2, 3])
def test_bc_split_over_ranks_sums_to_the_whole(tmp_path, world):
    import numpy as np

    from oracle import oracle as O
    from starplat_b200 import generators as G

    mp.start_processes(_bc_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    g = G.rmat(9, 8, seed=4)
    srcs = G.pick_sources(g, 37, seed=1)
    ref = O.bc(g.indexofNodes, g.edgeList, srcs)
    slices = [np.load(tmp_path / f"src{r}.npy") for r in range(world)]
    assert np.array_equal(np.concatenate(slices), srcs)  # a partition, in order
    for r in range(world):
        out = np.load(tmp_path / f"bc{r}.npy").astype(np.float64)
        assert np.all(np.abs(out - ref) <= 1e-5 * np.abs(ref) + 1e-6)


def _cc_rank_main(rank, world, port, out_dir):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "RANK": str(rank),
                       "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank)})
    sys.path.insert(0, ROOT)
    import numpy as np

    from oracle import oracle as O
    from starplat_b200 import generators as G
    from starplat_b200.distributed import sum_over_sources
    from starplat_b200.replicas import Replicas

    g = G.rmat(9, 8, seed=6)
    g.edgeLen = G.hash_weights(g, 6, 1, 50, True)
    srcs = np.sort(G.pick_sources(g, 23, seed=2)).astype(np.int32)
    rep = Replicas(backend="gloo", timeout_s=60)
    w = sum_over_sources(g.V, srcs, rep, lambda s: O.closeness(g.indexofNodes, g.edgeList, g.edgeLen, s))
    u = sum_over_sources(g.V, srcs, rep, lambda s: O.closeness_unweighted(g.indexofNodes, g.edgeList, s))
    rep.close()
    np.save(os.path.join(out_dir, f"ccw{rank}.npy"), w)
    np.save(os.path.join(out_dir, f"ccu{rank}.npy"), u)


def test_closeness_split_over_ranks_is_exact(tmp_path):
    # each source's entry comes from one rank: the reduced vector equals the whole bit for bit
    import numpy as np

    from oracle import oracle as O
    from starplat_b200 import generators as G

    world = 3
    mp.start_processes(_cc_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    g = G.rmat(9, 8, seed=6)
    g.edgeLen = G.hash_weights(g, 6, 1, 50, True)
    srcs = np.sort(G.pick_sources(g, 23, seed=2)).astype(np.int32)
    rw = O.closeness(g.indexofNodes, g.edgeList, g.edgeLen, srcs)
    ru = O.closeness_unweighted(g.indexofNodes, g.edgeList, srcs)
    for r in range(world):
        assert np.array_equal(np.load(tmp_path / f"ccw{r}.npy"), rw)
        assert np.array_equal(np.load(tmp_path / f"ccu{r}.npy"), ru)


def _lcc_part(off, adj, part, nparts):
    """The Compute_TC loop over the outer vertices v = part, part + nparts, ..., each
    triangle (v, u, w) adding one to all three (a small-graph restatement)."""
    import numpy as np

    cf = np.zeros(len(off) - 1, np.int32)
    for v in range(part, len(off) - 1, nparts):
        nb = adj[off[v]:off[v + 1]]
        for u in nb[nb < v]:
            nu = set(adj[off[u]:off[u + 1]].tolist())
            for w in nb[nb > v]:
                if int(w) in nu:
                    cf[v] += 1
                    cf[u] += 1
                    cf[w] += 1
    return cf


def _tc_rank_main(rank, world, port, out_dir):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "RANK": str(rank),
                       "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank)})
    sys.path.insert(0, ROOT)
    import numpy as np

    from oracle import oracle as O
    from starplat_b200 import generators as G
    from starplat_b200.distributed import lcc_sharded, tc_sharded
    from starplat_b200.replicas import Replicas

    g = G.rmat(9, 8, seed=8)
    rep = Replicas(backend="gloo", timeout_s=60)
    tc = tc_sharded(rep, lambda r, n: O.tc_omp(g.indexofNodes, g.edgeList, 1, r, n))
    cf = lcc_sharded(g.V, rep, lambda r, n: _lcc_part(g.indexofNodes, g.edgeList, r, n))
    rep.close()
    np.save(os.path.join(out_dir, f"tc{rank}.npy"), np.array([tc], np.int64))
    np.save(os.path.join(out_dir, f"cf{rank}.npy"), cf)


@pytest.mark.parametrize("world", [2, 3])
def test_triangle_parts_over_ranks_sum_to_the_whole(tmp_path, world):
    # every rank counts one part of the outer vertices; one all-reduce of an int64 (and of
    # the int32 per-vertex counts) gives every rank the whole graph's figures, exactly
    import numpy as np

    from oracle import oracle as O
    from starplat_b200 import generators as G

    mp.start_processes(_tc_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    g = G.rmat(9, 8, seed=8)
    want_tc = O.tc(g.indexofNodes, g.edgeList)
    want_cf = O.lcc(g.indexofNodes, g.edgeList)
    assert want_tc > 0
    for r in range(world):
        assert int(np.load(tmp_path / f"tc{r}.npy")[0]) == want_tc
        assert np.array_equal(np.load(tmp_path / f"cf{r}.npy"), want_cf)


def _device_sum_rank_main(rank, world, port, out_dir):
    # the in-place path the GPUs take: each rank's slice is written into a tensor, which is
    # summed where it lives (a host tensor under gloo, a CUDA tensor under NCCL); plus the
    # all-gather of equal slices
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "RANK": str(rank),
                       "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank)})
    sys.path.insert(0, ROOT)
    import numpy as np
    import torch

    from oracle import oracle as O
    from starplat_b200 import generators as G
    from starplat_b200.distributed import bc_sharded, lcc_sharded
    from starplat_b200.replicas import Replicas

    g = G.rmat(9, 8, seed=4)
    srcs = G.pick_sources(g, 37, seed=1)
    rep = Replicas(backend="gloo", timeout_s=60)
    assert rep.device().type == "cpu"
    out = torch.full((g.V,), float("nan"), dtype=torch.float32)

    def compute(s, o):
        o.copy_(torch.from_numpy(O.bc(g.indexofNodes, g.edgeList, s).astype(np.float32)))

    got = bc_sharded(g.V, srcs, rep, compute, out=out)
    assert got is out
    cf = torch.zeros(g.V, dtype=torch.int32)
    lcc_sharded(g.V, rep, lambda r, n, o: o.copy_(torch.from_numpy(_lcc_part(g.indexofNodes, g.edgeList, r, n))),
                out=cf)
    part = torch.full((5,), float(rank), dtype=torch.float32)
    full = torch.empty(5 * world, dtype=torch.float32)
    rep.all_gather_into(full, part)
    rep.close()
    np.save(os.path.join(out_dir, f"bc{rank}.npy"), out.numpy())
    np.save(os.path.join(out_dir, f"cf{rank}.npy"), cf.numpy())
    np.save(os.path.join(out_dir, f"ag{rank}.npy"), full.numpy())


def test_device_tensor_sums_over_ranks(tmp_path):
    import numpy as np

    from oracle import oracle as O
    from starplat_b200 import generators as G

    world = 3
    mp.start_processes(_device_sum_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    g = G.rmat(9, 8, seed=4)
    srcs = G.pick_sources(g, 37, seed=1)
    ref = O.bc(g.indexofNodes, g.edgeList, srcs)
    want_cf = O.lcc(g.indexofNodes, g.edgeList)
    for r in range(world):
        out = np.load(tmp_path / f"bc{r}.npy").astype(np.float64)
        assert np.all(np.abs(out - ref) <= 1e-5 * np.abs(ref) + 1e-6)
        assert np.array_equal(np.load(tmp_path / f"cf{r}.npy"), want_cf)
        assert np.array_equal(np.load(tmp_path / f"ag{r}.npy"), np.repeat(np.arange(world, dtype=np.float32), 5))


class _HostPartGraph:
    """A host stand-in for DeviceGraph's split-PageRank calls (test infrastructure): the
    same contract (contiguous blocks of S ids per part, the caller's buffers, a stop test
    on the summed diff), computed with numpy in the identity vertex order, so that the
    collectives and the loop of distributed.pagerank_on_gpus run between real gloo ranks."""

    def __init__(self, g):
        self.g, self.V = g, g.V
        self.od = np.diff(g.indexofNodes).astype(np.float32)

    def pagerank_part_begin(self, part, nparts, beta, delta, max_iter, con0, con1, diff):
        self.r, self.n, self.S = part, nparts, -(-self.V // nparts)
        self.lo, self.hi = part * self.S, min(self.V, (part + 1) * self.S)
        self.beta, self.delta, self.max_iter = beta, delta, max(1, max_iter)
        self.con, self.diff = [con0, con1], diff
        V = self.V
        self.pr = [np.full(V, np.float32(1.0) / np.float32(V), np.float32), np.zeros(V, np.float32)]
        c = np.zeros(self.n * self.S, np.float32)
        c[:V] = np.where(self.od > 0, self.pr[0] / np.maximum(self.od, 1), 0)
        con0.copy_(torch_from(c))
        self.it, self.done, self.last = 0, False, 0.0
        return self.S

    def pagerank_part_iterate(self, k):
        if self.done:
            return
        g, c, nx = self.g, k & 1, (k + 1) & 1
        con = self.con[c].numpy()
        base = np.float32((1.0 - self.delta) / self.V)
        d = 0.0
        for v in range(self.lo, self.hi):
            s = float(con[g.srcList[g.rev_indexofNodes[v]:g.rev_indexofNodes[v + 1]]].astype(np.float64).sum())
            np_ = np.float32(base + np.float32(self.delta) * np.float32(s))
            d += abs(float(np_) - float(self.pr[c][v]))
            self.pr[nx][v] = np_
            self.con[nx][v] = float(np_ / self.od[v]) if self.od[v] > 0 else 0.0
        self.diff[0] = d
        self.it += 1

    def pagerank_part_decide(self):
        if not self.done:
            self.last = float(self.diff[0])
            self.done = not (self.last > self.beta and self.it < self.max_iter)

    def pagerank_part_state(self):
        return self.it, self.done, self.last

    def pagerank_part_ranks(self, out):
        block = np.zeros(self.S, np.float32)
        block[:self.hi - self.lo] = self.pr[self.it & 1][self.lo:self.hi]
        out.copy_(torch_from(block))

    def pagerank_part_finish(self, full, out):
        out[:] = full.numpy()[:self.V]


def torch_from(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a))


def _pr_rank_main(rank, world, port, out_dir):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "RANK": str(rank),
                       "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank)})
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from starplat_b200 import generators as G
    from starplat_b200.distributed import pagerank_on_gpus
    from starplat_b200.replicas import Replicas
    from test_replicas import _HostPartGraph

    g = G.rmat(9, 8, seed=11, directed=True)
    rep = Replicas(backend="gloo", timeout_s=60)
    pr, it, diff = pagerank_on_gpus(_HostPartGraph(g), rep, beta=1e-7, check_every=3)
    rep.close()
    np.save(os.path.join(out_dir, f"pr{rank}.npy"), pr)
    np.save(os.path.join(out_dir, f"it{rank}.npy"), np.array([it, diff]))


@pytest.mark.parametrize("world", [2, 3])
def test_pagerank_split_over_ranks_matches_the_oracle(tmp_path, world):
    # every rank owns one block of rows; the contrib blocks are all-gathered and the diff
    # summed by gloo each iteration; every rank ends with the whole vector at the same
    # iteration, equal to FP64 PageRank at that iteration count
    from oracle import oracle as O
    from starplat_b200 import generators as G

    mp.start_processes(_pr_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    g = G.rmat(9, 8, seed=11, directed=True)
    its = [np.load(tmp_path / f"it{r}.npy") for r in range(world)]
    assert len({int(x[0]) for x in its}) == 1
    it = int(its[0][0])
    exact, it64, _ = O.pagerank(g.indexofNodes, g.rev_indexofNodes, g.srcList, 1e-7, 0.85, 100)
    assert abs(it - it64) <= 1
    exact, _, _ = O.pagerank(g.indexofNodes, g.rev_indexofNodes, g.srcList, 0.0, 0.85, it)
    for r in range(world):
        pr = np.load(tmp_path / f"pr{r}.npy").astype(np.float64)
        assert np.abs(pr - exact).sum() < 1e-6


INT_MAX = 2**31 - 1


class _HostSsspPart:
    """A host stand-in for DeviceGraph's split-SSSP calls (test infrastructure): the same
    contract (vertices owned by v % nparts, one (vertex, distance) pair per foreign vertex
    per round packed in part order, frontier sizes and far minima for the caller to
    combine), computed with Python sets and numpy, so that the loop and the collectives
    of distributed.sssp_on_gpus run between real gloo ranks."""

    def __init__(self, g):
        self.g, self.V = g, g.V

    def sssp_part_begin(self, part, nparts, src, weight=None, delta=0):
        g = self.g
        self.r, self.n = part, nparts
        self.w = np.asarray(g.edgeLen if weight is None else weight, np.int64)
        if self.w.size and self.w.min() < 0:
            self.delta = 1 << 62
        else:
            self.delta = int(delta) if delta > 0 else max(1, int(self.w.max()) if self.w.size else 1)
        self.dist = np.full(self.V, INT_MAX, np.int64)
        self.Q, self.QN, self.F = set(), set(), set()
        if src % nparts == part:
            self.dist[src] = 0
            self.Q.add(src)
        self.thr, self.rounds = self.delta, 0
        self.cap = -(-self.V // nparts)
        return self.cap

    def _queue(self, u, d):
        (self.QN if d < self.thr else self.F).add(u)

    def sssp_part_relax(self, send, send_counts):
        g, out = self.g, [dict() for _ in range(self.n)]
        for v in sorted(self.Q):
            for k in range(g.indexofNodes[v], g.indexofNodes[v + 1]):
                u, nd = int(g.edgeList[k]), int(self.dist[v] + self.w[k])
                if nd >= INT_MAX:
                    continue
                q = u % self.n
                if q == self.r:
                    if nd < self.dist[u]:
                        self.dist[u] = nd
                        self._queue(u, nd)
                elif nd < out[q].get(u, INT_MAX):
                    out[q][u] = nd
        at = 0
        for q in range(self.n):
            pairs = sorted(out[q].items())
            for i, (u, d) in enumerate(pairs):
                send[at + i, 0], send[at + i, 1] = u, d
            send_counts[q] = len(pairs)
            at += len(pairs)

    def sssp_part_apply(self, msgs, n, frontier):
        for i in range(n):
            u, d = int(msgs[i, 0]), int(msgs[i, 1])
            assert u % self.n == self.r
            if d < self.dist[u]:
                self.dist[u] = d
                self._queue(u, d)
        self.Q, self.QN = self.QN, set()
        frontier[0] = len(self.Q)
        self.rounds += 1
        if self.rounds > 4 * self.V + 64:
            from starplat_b200 import _lib

            raise _lib.SPError(-6, "negative cycle")

    def sssp_part_far_min(self, far):
        far[0] = min([int(self.dist[u]) for u in self.F if self.dist[u] >= self.thr], default=INT_MAX)

    def sssp_part_advance(self, far, frontier):
        fm, old = int(far[0]), self.thr
        self.thr = (fm // self.delta + 1) * self.delta
        self.Q = {u for u in self.F if old <= self.dist[u] < self.thr}
        self.F = {u for u in self.F if self.dist[u] >= self.thr}
        frontier[0] = len(self.Q)

    def sssp_part_dist(self, out):
        own = np.arange(self.V) % self.n == self.r
        out.copy_(torch_from(np.where(own, self.dist, INT_MAX).astype(np.int32)))


def _sssp_graphs():
    from starplat_b200 import generators as G

    g = G.rmat(9, 8, seed=13, directed=True)
    g.edgeLen = G.hash_weights(g, 13, 1, 100, False)
    gg = G.grid(12, 17)
    gg.edgeLen = G.hash_weights(gg, 14, 1, 1000, True)
    return [(g, 3), (gg, 0), (gg, 100)]


def _sssp_rank_main(rank, world, port, out_dir):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "RANK": str(rank),
                       "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank)})
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from starplat_b200.distributed import sssp_on_gpus
    from starplat_b200.replicas import Replicas
    from test_replicas import _HostSsspPart, _sssp_graphs

    rep = Replicas(backend="gloo", timeout_s=60)
    for k, (g, src) in enumerate(_sssp_graphs()):
        d, rounds = sssp_on_gpus(_HostSsspPart(g), rep, src)
        np.save(os.path.join(out_dir, f"d{k}_{rank}.npy"), d)
    rep.close()


@pytest.mark.parametrize("world", [2, 3])
def test_sssp_split_over_ranks_matches_the_oracle(tmp_path, world):
    # every rank owns v % world; each round's pairs for other ranks' vertices go through
    # one gloo all-to-all, frontier sizes are summed, far minima and dist vectors reduced
    # by minimum; every rank ends with the whole dist vector, equal to the oracle's
    from oracle import oracle as O

    mp.start_processes(_sssp_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    for k, (g, src) in enumerate(_sssp_graphs()):
        ref = O.sssp(g.indexofNodes, g.edgeList, g.edgeLen, src)
        for r in range(world):
            assert np.array_equal(np.load(tmp_path / f"d{k}_{r}.npy"), ref), (k, r)
