"""Host plumbing for running one workload as N independent replicas, one
process per GPU under torchrun (RANK / WORLD_SIZE / MASTER_* from the
environment).  The intersection paths shard without any data exchange (one
pair per rank, or disjoint tile pairs / pair lists), so the only collectives
are the ones that time the job: a barrier on each side of the timed region and
the maximum of the ranks' device times.  NCCL on GPUs; gloo carries the same
calls on CPU (the multi-process tests)."""
from __future__ import annotations

import datetime
import os

import torch


class Replicas:
    """rank / world from the environment; with world > 1 a process group with
    a short timeout, so that ranks waiting for a rank that died end with an
    error instead of waiting for good."""

    def __init__(self, backend: str = "nccl", device: torch.device | None = None, timeout_s: float = 300.0):
        self.rank = int(os.environ.get("RANK", 0))
        self.world = int(os.environ.get("WORLD_SIZE", 1))
        self.device = device if device is not None else torch.device("cpu")
        self._dist = None
        if self.world > 1:
            import torch.distributed as dist
            kw = {"device_id": self.device} if backend == "nccl" else {}
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s), **kw)
            self._dist = dist

    @property
    def active(self) -> bool:
        return self._dist is not None

    def barrier(self) -> None:
        if self._dist is not None:
            self._dist.barrier()

    def max(self, x: float) -> float:
        """The largest of the ranks' values (every rank gets it): a job's time
        is its slowest rank's."""
        if self._dist is None:
            return float(x)
        t = torch.tensor([float(x)], dtype=torch.float64, device=self.device)
        self._dist.all_reduce(t, op=self._dist.ReduceOp.MAX)
        return float(t.item())

    def rate(self, units_per_rank: float, ms: float) -> float:
        """Whole-job throughput: the units all ranks processed over the job's
        (slowest rank's) time in milliseconds."""
        return self.world * units_per_rank / (ms * 1e-3)

    def close(self) -> None:
        if self._dist is not None:
            self._dist.destroy_process_group()
            self._dist = None
