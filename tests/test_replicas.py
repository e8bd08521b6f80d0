"""Multi-rank plumbing on the CPU: two gloo ranks run the replica collectives the
benchmark uses on N GPUs (barrier, max of the device time over ranks, sum of the
units processed), and the reference arm under torchrun prints one line, from rank 0."""
import json
import os
import socket
import subprocess
import sys

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
