"""Replica plumbing for multi-GPU runs: one independent simulation per rank.

The step has no exchange between simulations, so N GPUs run N replicas (weak scaling)
and the process group carries only the barrier around the timed region and the
max-over-ranks of the measured time. Launched by torchrun (RANK, WORLD_SIZE,
LOCAL_RANK, MASTER_ADDR/PORT from the environment); NCCL on GPUs, gloo on CPU.
"""
from __future__ import annotations

import datetime
import os


class Replicas:
    def __init__(self, backend: str | None = None, timeout_s: float = 120.0):
        import torch
        import torch.distributed as dist

        self._torch, self._dist = torch, dist
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.backend = backend or ("nccl" if torch.cuda.is_available() else "gloo")
        if self.backend == "nccl":
            torch.cuda.set_device(self.local if self.world > 1 else 0)
        if self.world > 1:
            dist.init_process_group(self.backend, timeout=datetime.timedelta(seconds=timeout_s))

    def _device(self):
        return "cuda" if self.backend == "nccl" else "cpu"

    def barrier(self) -> None:
        if self.world > 1:
            self._dist.barrier()

    def max(self, v: float) -> float:
        """Largest value over ranks (every rank calls it, in the same order)."""
        if self.world == 1:
            return float(v)
        t = self._torch.tensor([float(v)], device=self._device(), dtype=self._torch.float64)
        self._dist.all_reduce(t, op=self._dist.ReduceOp.MAX)
        return float(t.item())

    def throughput(self, cells_per_rank: int, steps: int, seconds_local: float) -> float:
        """Whole-job Gcell-steps/s: every rank's cells over the slowest rank's time."""
        return cells_per_rank * steps * self.world / self.max(seconds_local) / 1e9

    def close(self) -> None:
        if self.world > 1 and self._dist.is_initialized():
            self._dist.destroy_process_group()
