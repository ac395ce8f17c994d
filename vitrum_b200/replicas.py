"""One process per GPU, each rendering its own replica of the workload.

Pixels, samples and frames are independent, so N GPUs run N replicas with no
data-path collective (weak scaling); the only collectives are the barrier
around the timed region and the max-over-ranks of the device time, as the
timing rules ask.  Rank, world size and local rank come from the torchrun
environment (RANK, WORLD_SIZE, LOCAL_RANK); rendezvous uses MASTER_ADDR /
MASTER_PORT.
"""
from __future__ import annotations

import datetime
import os


def env_rank():
    """(rank, world_size, local_rank) from the launcher's environment (1 process: 0, 1, 0)."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


class Group:
    """Process group for N > 1 (NCCL on GPUs, gloo for CPU tests); inert for N = 1."""

    def __init__(self, world: int, backend: str = "nccl", device=None, timeout_s: float = 120.0):
        self.world = world
        self.device = device
        self._dist = None
        if world > 1:
            import torch.distributed as dist
            kw = {"timeout": datetime.timedelta(seconds=timeout_s)}
            if backend == "nccl" and device is not None:
                kw["device_id"] = device
            dist.init_process_group(backend, **kw)
            self._dist = dist

    def barrier(self) -> None:
        if self._dist:
            self._dist.barrier()

    def max(self, x: float) -> float:
        """The maximum of x over all ranks (every rank gets it)."""
        if not self._dist:
            return float(x)
        import torch
        t = torch.tensor([float(x)], dtype=torch.float64, device=self.device)
        self._dist.all_reduce(t, op=self._dist.ReduceOp.MAX)
        return float(t.item())

    def close(self) -> None:
        if self._dist:
            self._dist.barrier()
            self._dist.destroy_process_group()
            self._dist = None


def replica_seed(rank: int, step: int) -> int:
    """Frame seed of a replica's step: distinct per rank so replicas do distinct work."""
    return rank * 100000 + step


def whole_job_rate(units_per_rank: float, world: int, max_seconds: float) -> float:
    """Aggregate throughput: all ranks' units over the slowest rank's time."""
    return world * units_per_rank / max_seconds
