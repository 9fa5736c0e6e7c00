"""Replica runs: one process per GPU, each solving its own copy of the workload.

The inverter path runs on one GPU and needs no collective in its data path, so
N GPUs run N independent replicas (launched by torchrun, one rank per GPU).
What the ranks share is the host plumbing of a timed run: a barrier on both
sides of the timed region, the maximum of the per-rank device times, and the
whole-job rate (units of work of all ranks over that maximum).  It runs over a
torch.distributed process group: NCCL between GPUs, gloo on CPU (the tests).
"""
from __future__ import annotations

import datetime
import os


class Replicas:
    """The rank's view of a replica run (WORLD_SIZE / RANK / LOCAL_RANK from the
    environment; a single process when WORLD_SIZE is unset or 1)."""

    def __init__(self, backend: str = "nccl", timeout_s: float = 600.0, device=None):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.backend = backend
        self.pg = None
        if self.world > 1:
            import torch.distributed as dist
            kw = {"timeout": datetime.timedelta(seconds=timeout_s)}
            if backend == "nccl" and device is not None:
                kw["device_id"] = device
            dist.init_process_group(backend, **kw)
            self.pg = dist

    def barrier(self):
        if self.pg is not None:
            self.pg.barrier()

    def max_over_ranks(self, seconds: float) -> float:
        """The slowest rank's time (every rank gets it)."""
        if self.pg is None:
            return seconds
        import torch
        dev = f"cuda:{self.local}" if self.backend == "nccl" else "cpu"
        t = torch.tensor([float(seconds)], dtype=torch.float64, device=dev)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def rate(self, units_per_rank: float, seconds: float) -> float:
        """Whole-job throughput: the units of all ranks over the slowest rank's time."""
        return self.world * units_per_rank / self.max_over_ranks(seconds)

    def close(self):
        if self.pg is not None:
            self.pg.destroy_process_group()
            self.pg = None
