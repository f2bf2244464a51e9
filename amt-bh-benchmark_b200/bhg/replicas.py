"""Multi-GPU plumbing of the benchmark: independent replicas, one process
per GPU.

A Barnes-Hut system never spans GPUs here, so ranks exchange nothing on the
data path: each rank runs its own replica of the workload (seeded by its
rank) and the ranks only meet to line up the timed region (barrier) and to
combine their results (max of the device times, sum of the work done).  The
process group is NCCL on GPUs; the same code runs on the gloo backend on CPU
for tests.  Rendezvous comes from torchrun's environment (RANK, WORLD_SIZE,
LOCAL_RANK, MASTER_ADDR, MASTER_PORT).
"""
from __future__ import annotations

import datetime
import os


class Replicas:
    def __init__(self, backend="nccl", device=None, timeout_s=300):
        import torch

        self.torch = torch
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.device = device if device is not None else f"cuda:{self.local}"
        if self.world > 1 and not torch.distributed.is_initialized():
            torch.distributed.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))

    def barrier(self):
        if self.world > 1:
            self.torch.distributed.barrier()

    def _reduce(self, v, op):
        if self.world == 1:
            return v
        t = self.torch.tensor([float(v)], dtype=self.torch.float64, device=self.device)
        self.torch.distributed.all_reduce(t, op=op)
        return float(t.item())

    def max(self, v):
        """The maximum of v over the ranks (device times: the job takes as long
        as its slowest rank)."""
        return self._reduce(v, self.torch.distributed.ReduceOp.MAX)

    def sum(self, v):
        """The sum of v over the ranks (work done: particle-steps)."""
        return self._reduce(v, self.torch.distributed.ReduceOp.SUM)

    def close(self):
        if self.world > 1 and self.torch.distributed.is_initialized():
            self.torch.distributed.barrier()
            self.torch.distributed.destroy_process_group()


def replica_seed(seed: int, rank: int) -> int:
    """The seed of rank `rank`'s replica: every rank simulates different
    particles of the same workload."""
    return seed + rank
