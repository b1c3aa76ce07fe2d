"""Replica groups: one process per GPU, each rank solving its own studies.

A static solve does not shard: every operator product would need a halo exchange and every dot
product an all-reduce, for a system that fits one GPU's HBM many times over. So N GPUs run N
independent replicas (the plate workload: one plate per rank; the serving stream: one server per
rank over a round-robin share of the requests), and no collective touches the data path. The group
carries only the measurement plumbing around the replicas: a barrier before and after a timed
region, the maximum over ranks of a device-timed duration, sums and gathers of per-rank counts and
latencies, and the request split.

The rank layout is torchrun's (`RANK`, `WORLD_SIZE`, `LOCAL_RANK`, `MASTER_ADDR`, `MASTER_PORT`).
On GPUs the group runs over NCCL with the reduction tensors on this rank's device; the host-side
logic is the same over gloo on CPU tensors.
"""
from __future__ import annotations

import datetime
import os
from dataclasses import dataclass
from typing import Any, Sequence


@dataclass
class ReplicaGroup:
    rank: int = 0
    world: int = 1
    local_rank: int = 0
    dist: Any = None
    device: Any = None

    @classmethod
    def from_env(cls, backend: str = "nccl", timeout_seconds: float = 600.0) -> "ReplicaGroup":
        """The group of the processes torchrun started; a single process needs no process group.
        `backend` "nccl" binds this rank to GPU `LOCAL_RANK`; "gloo" keeps everything on the host."""
        rank = int(os.environ.get("RANK", 0))
        world = int(os.environ.get("WORLD_SIZE", 1))
        local = int(os.environ.get("LOCAL_RANK", rank))
        if world == 1:
            return cls(rank, world, local)
        import torch
        import torch.distributed as dist

        timeout = datetime.timedelta(seconds=timeout_seconds)
        if backend == "nccl":
            device = torch.device("cuda", local)
            torch.cuda.set_device(device)
            dist.init_process_group("nccl", timeout=timeout, device_id=device)
        else:
            device = torch.device("cpu")
            dist.init_process_group(backend, timeout=timeout)
        if dist.get_world_size() != world or dist.get_rank() != rank:
            raise RuntimeError(f"process group is rank {dist.get_rank()} of {dist.get_world_size()}, "
                               f"environment says {rank} of {world}")
        return cls(rank, world, local, dist, device)

    @property
    def leader(self) -> bool:
        return self.rank == 0

    def barrier(self) -> None:
        if self.dist:
            self.dist.barrier()

    def _reduce(self, x: float, op_name: str) -> float:
        if not self.dist:
            return float(x)
        import torch

        t = torch.tensor([float(x)], dtype=torch.float64, device=self.device)
        self.dist.all_reduce(t, op=getattr(self.dist.ReduceOp, op_name))
        return float(t.item())

    def max(self, x: float) -> float:
        """The slowest rank's value: a timed region ends when every replica has finished."""
        return self._reduce(x, "MAX")

    def sum(self, x: float) -> float:
        return self._reduce(x, "SUM")

    def gather(self, values: Sequence[Any]) -> list:
        """Every rank's `values`, concatenated in rank order (on every rank)."""
        if not self.dist:
            return list(values)
        parts = [None] * self.world
        self.dist.all_gather_object(parts, list(values))
        return [v for p in parts for v in p]

    def shard(self, items: Sequence[Any]) -> list:
        """This rank's round-robin share of a request stream: item i goes to rank i mod world, so
        every item is served exactly once and arrival order is kept within each share."""
        return list(items[self.rank::self.world])

    def rate(self, units_per_rank: float, seconds: float) -> float:
        """Whole-job throughput: the units all ranks processed over the slowest rank's time."""
        return self.sum(units_per_rank) / self.max(seconds)

    def close(self) -> None:
        if self.dist:
            self.dist.destroy_process_group()
            self.dist = None
