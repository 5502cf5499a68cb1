"""Independent replicas across GPUs: the rank plumbing of the multi-GPU bench.

The path does not exchange data between GPUs (each rank solves its own
problem), so the only collectives are the timing ones: a barrier around the
timed region and the maximum of the per-rank device times.  Ranks come from
the torchrun environment (RANK, LOCAL_RANK, WORLD_SIZE, MASTER_ADDR/PORT).
"""
from __future__ import annotations

import datetime
import os
from typing import Optional, Tuple


def env() -> Tuple[int, int, int]:
    """(world size, rank, local rank) from the launcher's environment."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


class Replicas:
    """Process group of the replicas (none for a single process).

    backend "nccl" for GPU ranks, "gloo" for CPU ranks; the timeout bounds
    every collective, so a rank that never arrives ends the others with an
    error instead of a hang."""

    def __init__(self, backend: str = "nccl", timeout_s: float = 600.0, device: Optional[int] = None):
        self.world, self.rank, self.local = env()
        self.backend = backend
        self.device = device
        self.dist = None
        if self.world > 1:
            import torch.distributed as dist
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
            self.dist = dist

    def _tensor(self, x: float):
        import torch
        dev = f"cuda:{self.device}" if self.backend == "nccl" else "cpu"
        return torch.tensor([float(x)], dtype=torch.float64, device=dev)

    def barrier(self):
        if self.dist is not None:
            if self.backend == "nccl":
                self.dist.barrier(device_ids=[self.device])
            else:
                self.dist.barrier()
        if self.backend == "nccl":
            import torch
            torch.cuda.synchronize(self.device)

    def max(self, x: float) -> float:
        """Maximum of x over the ranks (every rank gets it)."""
        if self.dist is None:
            return float(x)
        t = self._tensor(x)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.dist is not None:
            self.dist.barrier()
            self.dist.destroy_process_group()
            self.dist = None
