"""Rank coordination for runs on several GPUs of one node.

One process per GPU (torchrun sets RANK / LOCAL_RANK / WORLD_SIZE).  Beams
are sharded across ranks with no collective on the data path: every rank
searches its own beams.  The only collectives are the timing barrier and the
maximum over ranks of a measured step time, so the job's time is its slowest
rank's.  The same class runs over NCCL on GPUs and over gloo on CPU (the
multi-rank tests).
"""
from __future__ import annotations

import datetime
import os

import torch
import torch.distributed as dist


class Ranks:
    def __init__(self, backend: str = "nccl", device: torch.device | None = None, timeout_s: float = 120.0):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.backend = backend
        self.device = device
        self._owns_group = False
        if self.world > 1 and not dist.is_initialized():
            kw = {"device_id": device} if backend == "nccl" and device is not None else {}
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s), **kw)
            self._owns_group = True

    def barrier(self) -> None:
        if self.world == 1:
            return
        if self.backend == "nccl":
            dist.barrier(device_ids=[self.local])
        else:
            dist.barrier()

    def max(self, v: float) -> float:
        """The largest v over all ranks (every rank gets it)."""
        if self.world == 1:
            return v
        dev = self.device if self.backend == "nccl" else torch.device("cpu")
        t = torch.tensor([v], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def close(self) -> None:
        if self._owns_group and dist.is_initialized():
            dist.destroy_process_group()
            self._owns_group = False
