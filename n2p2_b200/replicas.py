"""Replica coordination for runs of one process per GPU (weak scaling).

Prediction shards over independent frames or structures with no exchange
between them, so a run on N GPUs is N independent replicas: each rank
evaluates its own frames, and the only collectives are a barrier around the
timed region and the maximum of the ranks' times (the time of the whole
job).  Ranks come from the launcher's environment (RANK, WORLD_SIZE,
LOCAL_RANK, MASTER_ADDR, MASTER_PORT); with one process no process group is
created.  The backend is NCCL on GPUs; gloo runs the same protocol on CPU.
"""
from __future__ import annotations

import datetime
import os


class Replicas:
    def __init__(self, backend: str = "nccl", timeout_s: float = 600.0):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self._dist = None
        self._device = None
        if backend == "nccl":
            import torch
            torch.cuda.set_device(self.local)
            self._device = torch.device("cuda", self.local)
        if self.world > 1:
            import torch.distributed as dist
            kw = {}
            if self._device is not None:
                kw["device_id"] = self._device
            dist.init_process_group(
                backend, timeout=datetime.timedelta(seconds=timeout_s), **kw)
            self._dist = dist

    def barrier(self):
        """All of this rank's device work done, then all ranks here."""
        if self._device is not None:
            import torch
            torch.cuda.synchronize()
        if self._dist is not None:
            self._dist.barrier()

    def max(self, x: float) -> float:
        """Maximum of x over the ranks (every rank gets it)."""
        if self._dist is None:
            return x
        import torch
        dev = self._device if self._device is not None else "cpu"
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        self._dist.all_reduce(t, op=self._dist.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self._dist is not None:
            self._dist.destroy_process_group()
            self._dist = None
