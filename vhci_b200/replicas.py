"""Replica plumbing for running independent solves on several GPUs, one process per GPU.

Solves share no data, so ranks never exchange anything on the data path: they meet only at the
barriers around a timed region and in a max-reduction of each rank's time (the job's time is the
slowest rank's).  The backend is NCCL with device tensors when CUDA is available, gloo with host
tensors otherwise (the CPU tests run two gloo ranks).  Rank and world size come from the launcher's
environment (RANK, LOCAL_RANK, WORLD_SIZE, MASTER_ADDR, MASTER_PORT).
"""
from __future__ import annotations

import datetime
import os


def rank_info() -> tuple[int, int, int]:
    """(world size, rank, local rank) from the launcher's environment."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


class Replicas:
    """Process group of the replica ranks (none for a single process)."""

    def __init__(self, backend: str | None = None, timeout_s: float = 600.0):
        import torch
        self.world, self.rank, self.local = rank_info()
        self.dist = None
        use_cuda = torch.cuda.is_available() and backend != "gloo"
        self.device = torch.device("cuda", self.local) if use_cuda else torch.device("cpu")
        if self.world > 1:
            import torch.distributed as dist
            kw = {"timeout": datetime.timedelta(seconds=timeout_s)}
            if use_cuda:
                kw["device_id"] = self.device
            dist.init_process_group(backend or ("nccl" if use_cuda else "gloo"), **kw)
            self.dist = dist

    def barrier(self) -> None:
        import torch
        if self.dist is not None:
            self.dist.barrier()
        if self.device.type == "cuda":
            torch.cuda.synchronize(self.device)

    def _reduce(self, x: float, op) -> float:
        import torch
        if self.dist is None:
            return float(x)
        t = torch.tensor([float(x)], dtype=torch.float64, device=self.device)
        self.dist.all_reduce(t, op=op)
        return float(t.item())

    def allmax(self, x: float) -> float:
        return self._reduce(x, self.dist.ReduceOp.MAX if self.dist else None)

    def allsum(self, x: float) -> float:
        return self._reduce(x, self.dist.ReduceOp.SUM if self.dist else None)

    def close(self) -> None:
        if self.dist is not None:
            self.dist.destroy_process_group()
            self.dist = None


def job_seconds_per_solve(t_max_s: float, steps: int, world: int) -> float:
    """Whole-job seconds per solve: every rank completed `steps` solves, the job took the slowest
    rank's time."""
    return t_max_s / float(steps * world)
