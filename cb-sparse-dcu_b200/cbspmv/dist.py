"""Process-group plumbing for multi-GPU runs (one process per GPU).

The replica runs of bench.py (one copy of the workload per GPU) use the group
only to line the ranks up (barrier) and to time a step as the maximum over
ranks; one matrix sharded by block rows (cbspmv.shard.RowShard) also
exchanges x (an all-gather) and, for the adjoint, partial A^T g (a
reduce-scatter) through it.  Backend "nccl" on GPUs, "gloo" in CPU tests.
"""
from __future__ import annotations

import datetime
import os


def world_info():
    """(world size, rank, local rank) from the torchrun environment."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


class Group:
    def __init__(self, backend: str, device=None, timeout_s: float = 120.0):
        import torch.distributed as dist
        self.dist = dist
        self.world, self.rank, self.local = world_info()
        self.active = self.world > 1
        self.device = device
        if self.active:
            kw = {"timeout": datetime.timedelta(seconds=timeout_s)}
            if backend == "nccl" and device is not None:
                kw["device_id"] = device
            dist.init_process_group(backend, **kw)

    def barrier(self):
        if self.active:
            self.dist.barrier()

    def max(self, value: float) -> float:
        """The largest value over all ranks (every rank gets it)."""
        if not self.active:
            return float(value)
        import torch
        t = torch.tensor([float(value)], dtype=torch.float64,
                         device=self.device if self.device is not None else "cpu")
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.active:
            self.dist.barrier()
            self.dist.destroy_process_group()
            self.active = False
