"""Replica plumbing for multi-GPU runs of the sort benchmarks.

The sort path does not shard: one sort has one global order, and exchanging
keys between GPUs is outside the path. N processes (one per GPU, launched by
torchrun) therefore run N independent replicas of a workload. The only
collectives are a barrier around timed regions and the maximum of each
rank's timing, so that a whole-job figure is limited by the slowest rank.
The backend is NCCL on GPUs; the tests drive the same code with gloo on CPU.
"""
from __future__ import annotations

import datetime
import os
from dataclasses import dataclass


@dataclass
class Replicas:
    world: int
    rank: int
    local: int
    device: object = None     # torch.device the collectives run on

    @property
    def leader(self) -> bool:
        """Rank 0 prints the result line."""
        return self.rank == 0

    def barrier(self) -> None:
        if self.world > 1:
            import torch.distributed as dist
            dist.barrier()

    def max_over_ranks(self, x: float) -> float:
        """The largest x over all ranks (every rank gets it)."""
        if self.world == 1:
            return float(x)
        import torch
        import torch.distributed as dist
        t = torch.tensor([float(x)], dtype=torch.float64, device=self.device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def close(self) -> None:
        """Every rank takes this last collective step in the same order."""
        if self.world > 1:
            import torch.distributed as dist
            dist.barrier()
            dist.destroy_process_group()


def from_env(backend: str = "nccl", timeout_s: int = 120) -> Replicas:
    """Rank layout from RANK / WORLD_SIZE / LOCAL_RANK (torchrun's
    variables); joins the process group when there is more than one rank.
    With NCCL each rank binds its local GPU; with gloo collectives run on
    the CPU."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    import torch
    if backend == "nccl":
        torch.cuda.set_device(local)
        device = torch.device("cuda", local)
    else:
        device = torch.device("cpu")
    r = Replicas(world, rank, local, device)
    if world > 1:
        import torch.distributed as dist
        kwargs = {"timeout": datetime.timedelta(seconds=timeout_s)}
        if backend == "nccl":
            kwargs["device_id"] = device
        dist.init_process_group(backend, **kwargs)
    return r


def whole_job_rate(units_per_rank: int, world: int, max_ms: float, steps: int) -> float:
    """Units per second for the whole job: every rank processed
    units_per_rank per step, and the job took the slowest rank's time."""
    return units_per_rank * world / (max_ms / steps * 1e-3)
