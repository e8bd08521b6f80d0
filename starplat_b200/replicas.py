"""Process-group plumbing for runs on several GPUs of one node (one process per GPU,
launched by torchrun, which sets RANK / WORLD_SIZE / LOCAL_RANK / MASTER_*).

The single-graph entry points run one graph per GPU, so N GPUs run N replicas with
no data-path collective; the timed runs need only the barrier around the timed region
and the reductions of its result (a whole-job rate is the units all ranks processed
over the SLOWEST rank's time). The algorithms split over the ranks (distributed.py)
use the data-path collectives here: an in-place sum of a per-vertex vector and an
all-gather of per-rank slices, both on device tensors when NCCL carries them, so no
vector leaves the GPU. gloo carries them on the host (the CPU tests run 2 and 3 ranks
that way).
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
        """Element-wise sum over all ranks, every rank getting the result. A torch tensor
        is reduced in place where it lives (a CUDA tensor under NCCL, a host tensor under
        gloo) and returned; a numpy array goes through a tensor on the backend's device
        and comes back as numpy."""
        if self._dist is None:
            return a
        import torch

        if isinstance(a, torch.Tensor):
            self._dist.all_reduce(a, op=self._dist.ReduceOp.SUM)
            return a
        import numpy as np

        dev = "cuda" if self.backend == "nccl" else "cpu"
        t = torch.from_numpy(np.ascontiguousarray(a)).to(dev)
        self._dist.all_reduce(t, op=self._dist.ReduceOp.SUM)
        return t.cpu().numpy()

    def all_gather_into(self, full, part) -> None:
        """full[r * n : (r + 1) * n] = rank r's `part` (n elements each) on every rank:
        torch tensors on the backend's device, full holding world * n elements."""
        if self._dist is None:
            if full.data_ptr() != part.data_ptr():
                full[: part.numel()].copy_(part)
            return
        self._dist.all_gather_into_tensor(full, part)

    def all_reduce_min(self, t) -> None:
        """Element-wise minimum over all ranks, in place (a torch tensor on the backend's
        device)."""
        if self._dist is not None:
            self._dist.all_reduce(t, op=self._dist.ReduceOp.MIN)

    def all_to_all(self, out, inp, out_splits, in_splits) -> None:
        """Rank q's inp[sum(in_splits[:r]) : + in_splits[r]] lands in rank r's out at
        sum(out_splits[:q]); splits are element counts along dim 0 (host ints). One rank:
        a copy."""
        if self._dist is None:
            n = int(in_splits[0])
            if n:
                out[:n].copy_(inp[:n])
            return
        self._dist.all_to_all_single(out, inp, [int(x) for x in out_splits], [int(x) for x in in_splits])

    def device(self):
        """Where this rank's collective tensors live: the host under gloo, else this
        rank's GPU (NCCL, or a single process with a GPU), else the host."""
        import torch

        if self.backend != "gloo" and torch.cuda.is_available():
            return torch.device("cuda", torch.cuda.current_device())
        return torch.device("cpu")

    def whole_job_rate(self, units: float, seconds: float) -> float:
        """Units all ranks processed per second of the slowest rank."""
        total, slowest = self.sum(units), self.max(seconds)
        return total / slowest if slowest > 0 else 0.0

    def close(self) -> None:
        if self._dist is not None:
            self._dist.destroy_process_group()
            self._dist = None
