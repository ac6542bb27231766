"""Host logic of multi-GPU runs.  The timestep runs on one GPU with GIP's topology
collapsed to one rank, so N GPUs run N independent replicas (weak scaling): the only
cross-rank traffic is a barrier around the timed region and the max of the ranks'
device times.  Works with any torch.distributed backend (NCCL on GPUs, gloo on CPU)."""
from __future__ import annotations

import torch


class Replicas:
    def __init__(self, dist=None, device: str = "cpu"):
        self.dist = dist
        self.device = device
        self.world = dist.get_world_size() if dist is not None else 1
        self.rank = dist.get_rank() if dist is not None else 0

    def barrier(self) -> None:
        if self.dist is not None:
            self.dist.barrier()

    def max(self, x: float) -> float:
        """Max over ranks (the job's time is its slowest replica's)."""
        if self.dist is None:
            return float(x)
        t = torch.tensor([float(x)], dtype=torch.float64, device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def sum(self, x: float) -> float:
        if self.dist is None:
            return float(x)
        t = torch.tensor([float(x)], dtype=torch.float64, device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM)
        return float(t.item())

    def job_ms_per_step(self, local_ms_total: float, steps: int) -> float:
        """Whole-job time per timestep: all replicas' steps over the slowest rank's time."""
        return self.max(local_ms_total) / (steps * self.world)
