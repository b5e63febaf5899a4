"""Independent engine replicas, one process per GPU.

The BRKGA generation step has no exchange between instances: islands of one instance
migrate on their own device, and separate instances or requests never talk to each
other.  Scaling out therefore means running whole instances on every GPU (the reference's
multi-GPU island loop, core/solver.hpp:378-558, becomes a replica per device).  The only
collectives are the ones needed to time such a job: a barrier around the timed region and
the maximum of the elapsed time over ranks.

Ranks come from the torch.distributed.run environment (RANK, WORLD_SIZE, LOCAL_RANK,
MASTER_ADDR, MASTER_PORT).  With one process nothing is initialised.
"""
from __future__ import annotations

import datetime
import os


class Replicas:
    """torch.distributed plumbing for N independent replicas (NCCL on GPUs, gloo on CPU)."""

    def __init__(self, backend: str | None = None, timeout_s: float = 300.0):
        self.rank = int(os.environ.get("RANK", "0"))
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.local_rank = int(os.environ.get("LOCAL_RANK", "0"))
        self.dist = None
        self.device = "cpu"
        if self.world > 1:
            import torch
            import torch.distributed as dist

            if backend is None:
                backend = "nccl" if torch.cuda.is_available() else "gloo"
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
            self.dist = dist
            self.device = f"cuda:{self.local_rank}" if backend == "nccl" else "cpu"

    @property
    def leader(self) -> bool:
        """rank 0 reports for the whole job"""
        return self.rank == 0

    def seed(self, base: int) -> int:
        """a different GA seed per replica, so replicas explore different runs"""
        return base + self.rank

    def barrier(self) -> None:
        if self.dist is not None:
            self.dist.barrier()

    def _reduce(self, x: float, op) -> float:
        import torch

        t = torch.tensor([float(x)], dtype=torch.float64, device=self.device)
        self.dist.all_reduce(t, op=op)
        return float(t.item())

    def max(self, x: float) -> float:
        """maximum over ranks (every rank must call it, in the same order)"""
        if self.dist is None:
            return float(x)
        return self._reduce(x, self.dist.ReduceOp.MAX)

    def sum(self, x: float) -> float:
        """sum over ranks (every rank must call it, in the same order)"""
        if self.dist is None:
            return float(x)
        return self._reduce(x, self.dist.ReduceOp.SUM)

    def close(self) -> None:
        if self.dist is not None:
            self.dist.barrier()
            self.dist.destroy_process_group()
            self.dist = None


def whole_job_rate(world: int, units_per_rank: float, seconds_max_over_ranks: float) -> float:
    """units per second of the whole job: every rank processed units_per_rank, and the job
    took as long as its slowest rank"""
    if seconds_max_over_ranks <= 0:
        raise ValueError("elapsed time must be positive")
    return world * units_per_rank / seconds_max_over_ranks
