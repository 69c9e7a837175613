"""Replica plumbing for running the codec on N GPUs of one node: one process
per GPU, launched by torchrun (RANK / LOCAL_RANK / WORLD_SIZE in the
environment).

Frames are independent, so every rank runs its own batch on its own GPU
with no data-path collective; the process group carries only the barrier
around a timed region and the max over ranks of its device time, and the
whole-job rate is the units all ranks processed over that time.  The
reference has no multi-GPU code (its batch API is a per-frame loop,
fastvid/__init__.py:44-53); this mirrors it by running whole replicas.

The backend is "nccl" on GPUs; the same object runs on "gloo" with CPU
tensors, which is how the multi-rank logic is tested without GPUs.
"""

from __future__ import annotations

import datetime
import os


class Replicas:
    def __init__(self, backend: str = "nccl", device=None, timeout_s: float = 300.0, env=None):
        env = os.environ if env is None else env
        self.world = int(env.get("WORLD_SIZE", "1"))
        self.rank = int(env.get("RANK", "0"))
        self.local_rank = int(env.get("LOCAL_RANK", "0"))
        self.backend = backend
        self.device = device
        self.dist = None
        if self.world > 1:
            import torch.distributed as dist

            kw = {"device_id": device} if backend == "nccl" and device is not None else {}
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s), **kw)
            self.dist = dist

    def barrier(self) -> None:
        if self.dist is not None:
            self.dist.barrier()

    def max(self, x: float) -> float:
        """The largest x over all ranks (every rank gets it)."""
        if self.dist is None:
            return float(x)
        import torch

        dev = self.device if self.backend == "nccl" else "cpu"
        t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def rate(self, units_per_rank: float, ms: float) -> float:
        """Whole-job units per second: all ranks' units over the slowest
        rank's time (`ms`, already the max over ranks)."""
        return self.world * units_per_rank / (ms / 1e3)

    @property
    def leader(self) -> bool:
        """Rank 0 alone prints and runs the single-GPU legs."""
        return self.rank == 0

    def close(self) -> None:
        if self.dist is not None:
            self.dist.destroy_process_group()
            self.dist = None
