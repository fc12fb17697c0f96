"""One process per GPU: the multi-GPU plumbing of the rigid path.

Sessions share nothing, so N GPUs run N independent session sets (weak
scaling) with no collective on the data path.  The only cross-rank steps
are host-side: the barrier around a timed region, the max over ranks of the
device time, sums of frame counts, and the placement of arriving sessions
on the GPU with the most free budget (decided on rank 0, broadcast).  A
single session does not shard (one 6x6 reduction per ICP iteration, one
hash table), so for one scene the ranks are replicas.

Launch with torchrun (RANK / LOCAL_RANK / WORLD_SIZE / MASTER_ADDR set);
NCCL on GPUs, gloo on CPU.
"""
from __future__ import annotations

import datetime
import os


class Ranks:
    """Rank identity plus the few host collectives the benchmark needs."""

    def __init__(self, backend: str | None = None, timeout_s: float = 300.0,
                 device_id=None):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.dist = None
        self._device = "cpu"
        if self.world > 1:
            import torch
            import torch.distributed as dist
            if backend is None:
                backend = "nccl" if torch.cuda.is_available() else "gloo"
            kw = {}
            if backend == "nccl":
                self._device = f"cuda:{self.local}"
                kw["device_id"] = device_id if device_id is not None else torch.device(
                    "cuda", self.local)
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s),
                                    **kw)
            self.dist = dist

    def barrier(self) -> None:
        if self.dist is not None:
            self.dist.barrier()

    def _reduce(self, x: float, op) -> float:
        if self.dist is None:
            return float(x)
        import torch
        v = torch.tensor([float(x)], dtype=torch.float64, device=self._device)
        self.dist.all_reduce(v, op=op)
        return float(v.item())

    def max(self, x: float) -> float:
        """Max over ranks (device times: the slowest rank bounds the job)."""
        return self._reduce(x, None if self.dist is None else self.dist.ReduceOp.MAX)

    def sum(self, x: float) -> float:
        return self._reduce(x, None if self.dist is None else self.dist.ReduceOp.SUM)

    def broadcast(self, obj):
        """Rank 0's object on every rank."""
        if self.dist is None:
            return obj
        box = [obj if self.rank == 0 else None]
        self.dist.broadcast_object_list(box, src=0)
        return box[0]

    def close(self) -> None:
        if self.dist is not None:
            self.dist.destroy_process_group()
            self.dist = None


def least_loaded(need_bytes, free_bytes):
    """Place sessions, in arrival order, on the GPU with the most free bytes
    that holds them (ties: the lower index).  Returns the GPU index of each
    session (-1: no GPU has room) and the free bytes left per GPU."""
    free = list(free_bytes)
    out = []
    for need in need_bytes:
        best = -1
        for g, f in enumerate(free):
            if f >= need and (best < 0 or f > free[best]):
                best = g
        if best >= 0:
            free[best] -= need
        out.append(best)
    return out, free
