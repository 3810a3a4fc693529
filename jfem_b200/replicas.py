"""Multi-GPU plumbing of the benchmark: one process per GPU, each solving
its own replica of the system (the solve of one system has no data-path
collective), a barrier around every timed region and the step time taken as
the maximum over ranks.  NCCL on GPUs, gloo on CPU (tests)."""
from __future__ import annotations

import datetime
import os


def dist_env():
    """(rank, world_size, local_rank) from the torchrun environment."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


class Replicas:
    """Rank coordination: barrier() and max() are no-ops for one process."""

    def __init__(self, backend: str | None = None, timeout_s: int = 600):
        import torch
        self.rank, self.world, self.local = dist_env()
        self.backend = backend or ("nccl" if torch.cuda.is_available() else "gloo")
        self.device = f"cuda:{self.local}" if self.backend == "nccl" else "cpu"
        self._dist = None
        if self.world > 1:
            import torch.distributed as dist
            dist.init_process_group(self.backend, timeout=datetime.timedelta(seconds=timeout_s))
            self._dist = dist

    @property
    def leader(self) -> bool:
        return self.rank == 0

    def barrier(self):
        if self._dist:
            self._dist.barrier()

    def max(self, value: float) -> float:
        if not self._dist:
            return float(value)
        import torch
        t = torch.tensor([float(value)], dtype=torch.float64, device=self.device)
        self._dist.all_reduce(t, op=self._dist.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self._dist:
            self._dist.destroy_process_group()
            self._dist = None
