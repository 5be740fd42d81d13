"""Independent replicas on several GPUs of one node.

The finite-volume path does not shard: one problem is one grid on one GPU.
Several GPUs run independent replicas (one process per GPU, launched by
torchrun), and torch.distributed is used only around the timed region: a
barrier on both sides and the maximum of the per-rank times, so a whole-job
rate is (ranks x units per rank) / slowest rank.  There is no collective on
the data path.

The backend is NCCL on GPUs; the same code runs on gloo with CPU tensors,
which is how the multi-process logic is tested without a GPU.  A short
process-group timeout makes ranks that wait for a missing peer fail instead
of hanging.
"""
from __future__ import annotations

import datetime
import os
from typing import Callable, Optional


def _env_int(key: str, default: int) -> int:
    try:
        return int(os.environ.get(key, default))
    except ValueError:
        return default


class Replicas:
    def __init__(self, backend: str = "nccl", timeout_s: float = 300.0,
                 device_sync: Optional[Callable[[], None]] = None):
        self.rank = _env_int("RANK", 0)
        self.world = _env_int("WORLD_SIZE", 1)
        self.local_rank = _env_int("LOCAL_RANK", 0)
        self.backend = backend
        self._sync = device_sync
        self._dist = None
        if self.world > 1:
            import torch.distributed as dist
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
            self._dist = dist

    def barrier(self) -> None:
        """All ranks meet; then this rank's device work is drained."""
        if self._dist is not None:
            self._dist.barrier()
        if self._sync is not None:
            self._sync()

    def _reduce(self, x: float, op: str) -> float:
        if self._dist is None:
            return float(x)
        import torch
        dev = "cuda" if self.backend == "nccl" else "cpu"
        t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
        self._dist.all_reduce(t, op=getattr(self._dist.ReduceOp, op))
        return float(t.item())

    def max(self, x: float) -> float:
        """The maximum of x over the ranks (x itself with one rank)."""
        return self._reduce(x, "MAX")

    def sum(self, x: float) -> float:
        """The sum of x over the ranks (x itself with one rank), e.g. the
        units the ranks processed when they differ per rank."""
        return self._reduce(x, "SUM")

    def rate(self, units_per_rank: float, seconds_this_rank: float) -> float:
        """Whole-job rate: every rank's units over the slowest rank's time
        (a collective: every rank must call it)."""
        return self.world * float(units_per_rank) / self.max(seconds_this_rank)

    @property
    def is_root(self) -> bool:
        return self.rank == 0

    def close(self) -> None:
        if self._dist is not None:
            self._dist.destroy_process_group()
            self._dist = None
