"""Replica plumbing for more than one GPU.

A single solve does not shard without a halo exchange per hop and an allreduce per
dot product (HILA's MPI layout, field_comm.h / lattice.cpp), which this library
does not do. The units that do shard are independent: solves, right-hand sides and
gauge fields (HILA runs such ensembles as separate `-partitions`,
initialize.cpp:415-470). So several GPUs run replicas: one process per GPU (launched
by torchrun), each with its own context, gauge fields and server, and requests
routed to the rank that owns their gauge field. torch.distributed is used only for
the barrier and for combining timings (max over ranks) and counts (sum); nothing in
the data path crosses GPUs.
"""
from __future__ import annotations

import datetime
import os
from typing import Sequence, TypeVar

T = TypeVar("T")


class ReplicaGroup:
    """Rank, world size and the few collectives a replica run needs.

    Reads RANK / LOCAL_RANK / WORLD_SIZE (torchrun); with one process nothing is
    initialised and every reduction is the identity."""

    def __init__(self, backend: str = "nccl", timeout_s: float = 300.0):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local_rank = int(os.environ.get("LOCAL_RANK", "0"))
        self.backend = backend
        self.pg = False
        if self.world > 1:
            import torch.distributed as dist
            os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
            self.pg = True

    def _reduce(self, v: float, op) -> float:
        import torch
        import torch.distributed as dist
        dev = f"cuda:{self.local_rank}" if self.backend == "nccl" else "cpu"
        t = torch.tensor([float(v)], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=op)
        return float(t.item())

    def barrier(self) -> None:
        if self.pg:
            import torch.distributed as dist
            dist.barrier()

    def max(self, v: float) -> float:
        """Largest value over ranks (device times: the job ends with the slowest rank)."""
        if not self.pg:
            return float(v)
        import torch.distributed as dist
        return self._reduce(v, dist.ReduceOp.MAX)

    def sum(self, v: float) -> float:
        """Sum over ranks (units processed)."""
        if not self.pg:
            return float(v)
        import torch.distributed as dist
        return self._reduce(v, dist.ReduceOp.SUM)

    def close(self) -> None:
        if self.pg:
            import torch.distributed as dist
            dist.destroy_process_group()
            self.pg = False


def owner(gauge_id: int, world: int) -> int:
    """Rank that holds gauge field `gauge_id` (round-robin over ranks)."""
    if world < 1:
        raise ValueError("world must be >= 1")
    return gauge_id % world


def shard(items: Sequence[T], rank: int, world: int) -> list:
    """This rank's share of independent work units (every unit on exactly one rank)."""
    return [it for k, it in enumerate(items) if owner(k, world) == rank]
