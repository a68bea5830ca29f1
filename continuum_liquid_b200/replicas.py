"""Replica runs: one process per GPU, each advancing its own independent scene.

The FLIP step does not shard (the solver is single-GPU and scenes exchange no data), so several GPUs
run independent replicas. Ranks only meet at barriers around a timed region and in one MAX
reduction of the measured time, so a job's time is its slowest rank's. NCCL carries these on GPUs;
gloo carries them in the CPU tests.
"""

from __future__ import annotations

import datetime
import os

import torch
import torch.distributed as dist


class ReplicaGroup:
    """Rank bookkeeping from the torchrun environment (RANK, WORLD_SIZE, LOCAL_RANK, MASTER_*)."""

    def __init__(self, backend: str = "nccl", timeout_s: float = 300.0):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local_rank = int(os.environ.get("LOCAL_RANK", "0"))
        self.backend = backend
        self.device = torch.device("cuda", self.local_rank) if backend == "nccl" else torch.device("cpu")
        if self.world > 1:
            os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
            kwargs = {"timeout": datetime.timedelta(seconds=timeout_s)}
            if backend == "nccl":
                torch.cuda.set_device(self.local_rank)
                kwargs["device_id"] = self.device
            dist.init_process_group(backend, **kwargs)

    def barrier(self) -> None:
        if self.world > 1:
            dist.barrier()

    def max(self, value: float) -> float:
        """The maximum of ``value`` over ranks (every rank gets it)."""
        if self.world == 1:
            return float(value)
        t = torch.tensor([float(value)], dtype=torch.float64, device=self.device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def close(self) -> None:
        if self.world > 1 and dist.is_initialized():
            dist.destroy_process_group()


def throughput(group: ReplicaGroup, steps_per_rank: int, elapsed_ms: float) -> tuple[float, float]:
    """Whole-job steps/s from each rank's own elapsed time: (steps of all ranks) / (slowest rank's
    time), plus that time in ms."""
    slowest = group.max(elapsed_ms)
    return group.world * steps_per_rank / (slowest / 1e3), slowest
