"""Replicas across GPUs: one process per GPU, no data-path collective.

The path shards naturally by column batch or by request (every LDE, NTT batch
or served request is independent), so N GPUs run N independent replicas.
The process group is used only for the measurement plumbing: a barrier
around timed regions and the maximum of per-rank times.  `partition` splits a
list of independent work items (uneven-batch polynomials, served requests)
across ranks by estimated work, deterministically, so every rank computes
the same assignment without communicating.

Backends: "nccl" on GPUs (torchrun), "gloo" for CPU tests.  The rendezvous
uses MASTER_ADDR / MASTER_PORT / RANK / WORLD_SIZE from the environment.
"""
from __future__ import annotations

import os
from datetime import timedelta
from typing import Callable, Sequence


class Replicas:
    """Rank, world size, barrier and max-over-ranks for N independent replicas."""

    def __init__(self, backend: str = "nccl", timeout_s: float = 120.0, device=None):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local_rank = int(os.environ.get("LOCAL_RANK", "0"))
        self.backend = backend
        self._dist = None
        self._device = device
        if self.world > 1:
            import torch.distributed as dist
            kw = {"timeout": timedelta(seconds=timeout_s)}
            if backend == "nccl" and device is not None:
                kw["device_id"] = device
            dist.init_process_group(backend, **kw)
            self._dist = dist

    @property
    def active(self) -> bool:
        return self._dist is not None

    def barrier(self) -> None:
        if self._dist is not None:
            self._dist.barrier()

    def max(self, value: float) -> float:
        """Maximum of `value` over ranks (every rank gets it)."""
        if self._dist is None:
            return float(value)
        import torch
        dev = self._device if (self.backend == "nccl" and self._device is not None) else "cpu"
        t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
        self._dist.all_reduce(t, op=self._dist.ReduceOp.MAX)
        return float(t.item())

    def close(self) -> None:
        if self._dist is not None:
            self._dist.destroy_process_group()
            self._dist = None


def job_time_per_unit(max_step_time: float, world: int) -> float:
    """Weak scaling: each rank runs one unit (e.g. one 256-column LDE) per
    step, so the job delivers `world` units per slowest-rank step time."""
    return max_step_time / max(1, world)


def partition(items: Sequence, world: int, rank: int, weight: Callable = lambda it: 1.0) -> list[int]:
    """Indices of `items` that rank `rank` runs: largest estimated work first,
    each to the least-loaded rank (ties to the lower rank).  Deterministic, so
    every rank derives the same assignment; the parts are disjoint and cover
    all items."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} of world {world}")
    order = sorted(range(len(items)), key=lambda i: (-float(weight(items[i])), i))
    load = [0.0] * world
    mine = []
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        load[r] += float(weight(items[i]))
        if r == rank:
            mine.append(i)
    return sorted(mine)


def lde_work(item: dict) -> float:
    """Estimated work of an LDE / blow-up item: output words x layers."""
    ext = item["log_n"] + item["added_bits"]
    return float(item["batch"] << ext) * max(1, ext)
