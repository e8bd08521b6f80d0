"""Replica plumbing for runs on several GPUs of one node (one process per GPU,
launched by torchrun, which sets RANK / WORLD_SIZE / LOCAL_RANK / MASTER_*).

Every entry point of this library runs one graph on one GPU, so N GPUs run N
independent replicas with no data-path collective. The only collectives are the
barrier around a timed region and the reductions of its result: a whole-job rate is
the units all ranks processed over the SLOWEST rank's time. NCCL carries them on
GPUs; gloo does on the host (the CPU tests run two ranks that way).
"""
from __future__ import annotations

import datetime
import os


class Replicas:
    """This process's place among the replicas, plus the few collectives a timed run needs."""

    def __init__(self, backend: str | None = None, timeout_s: float = 600.0):
        self.rank = int(os.environ.get("RANK", "0"))
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.local_rank = int(os.environ.get("LOCAL_RANK", "0"))
        self.backend = None
        self._dist = None
        if self.world > 1:
            import torch
            import torch.distributed as dist

            backend = backend or ("nccl" if torch.cuda.is_available() else "gloo")
            kwargs = {"timeout": datetime.timedelta(seconds=timeout_s)}
            if backend == "nccl":
                kwargs["device_id"] = torch.device("cuda", self.local_rank)
            dist.init_process_group(backend, **kwargs)
            self._dist = dist
            self.backend = backend

    @property
    def is_root(self) -> bool:
        return self.rank == 0

    def barrier(self) -> None:
        if self._dist is not None:
            self._dist.barrier()

    def _reduce(self, x: float, op) -> float:
        import torch

        dev = "cuda" if self.backend == "nccl" else "cpu"
        t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
        self._dist.all_reduce(t, op=op)
        return float(t.item())

    def max(self, x: float) -> float:
        """The largest x over all ranks (the slowest rank's time)."""
        return float(x) if self._dist is None else self._reduce(x, self._dist.ReduceOp.MAX)

    def sum(self, x: float) -> float:
        """x summed over all ranks (the units the whole job processed)."""
        return float(x) if self._dist is None else self._reduce(x, self._dist.ReduceOp.SUM)

    def all_reduce_sum(self, a):
        """Element-wise sum of a float32 numpy array over all ranks (every rank gets it)."""
        if self._dist is None:
            return a
        import numpy as np
        import torch

        dev = "cuda" if self.backend == "nccl" else "cpu"
        t = torch.from_numpy(np.ascontiguousarray(a)).to(dev)
        self._dist.all_reduce(t, op=self._dist.ReduceOp.SUM)
        return t.cpu().numpy()

    def whole_job_rate(self, units: float, seconds: float) -> float:
        """Units all ranks processed per second of the slowest rank."""
        total, slowest = self.sum(units), self.max(seconds)
        return total / slowest if slowest > 0 else 0.0

    def close(self) -> None:
        if self._dist is not None:
            self._dist.destroy_process_group()
            self._dist = None
