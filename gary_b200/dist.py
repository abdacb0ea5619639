"""Multi-GPU plumbing for sharded counts: one process per GPU.

Every rank holds the whole graph (it is replicated: about 4.5 GB at RMAT-24
ef32) and counts its shard of the tile plan with gary_count_shard_async
(shard = rank, nshards = world).  The shard totals are the only data that
crosses ranks: one 8-byte sum.  Timing takes the maximum over ranks.

    d = Dist.from_env()                 # RANK / WORLD_SIZE / LOCAL_RANK / MASTER_*
    d.init()                            # nccl with CUDA, gloo without
    total = d.allreduce(local_count, "sum")
    ms = d.allreduce(local_ms, "max")
    d.close()

The reference has no multi-GPU path (src/DeviceGraph.cu:91-96 pins one
device).  Every rank takes the same collective steps in the same order; the
process group has a short timeout so that ranks waiting for a rank that
failed end with an error instead of hanging.
"""
from __future__ import annotations

import datetime
import os
from dataclasses import dataclass


@dataclass
class Dist:
    rank: int = 0
    world: int = 1
    local: int = 0
    backend: str | None = None
    timeout_s: float = 600.0
    _pg: object = None

    @classmethod
    def from_env(cls, timeout_s: float = 600.0) -> "Dist":
        return cls(rank=int(os.environ.get("RANK", "0")), world=int(os.environ.get("WORLD_SIZE", "1")),
                   local=int(os.environ.get("LOCAL_RANK", "0")), timeout_s=timeout_s)

    def init(self, backend: str | None = None) -> "Dist":
        """Select this rank's GPU (when there is one) and join the process group
        (only when world > 1)."""
        import torch

        cuda = torch.cuda.is_available()
        if cuda:
            torch.cuda.set_device(self.local)
        if self.world > 1:
            import torch.distributed as td

            self.backend = backend or ("nccl" if cuda else "gloo")
            kw = {}
            if self.backend == "nccl":
                kw["device_id"] = torch.device("cuda", self.local)
            td.init_process_group(self.backend, rank=self.rank, world_size=self.world,
                                  timeout=datetime.timedelta(seconds=self.timeout_s), **kw)
            self._pg = td
        return self

    @property
    def active(self) -> bool:
        return self._pg is not None

    def _device(self):
        import torch

        return torch.device("cuda", self.local) if self.backend == "nccl" else torch.device("cpu")

    def barrier(self) -> None:
        if self._pg:
            self._pg.barrier()

    def allreduce(self, x: float | int, op: str):
        """Sum or max of a Python scalar over all ranks; ints stay exact (int64)."""
        if not self._pg:
            return x
        import torch

        dt = torch.float64 if isinstance(x, float) else torch.int64
        t = torch.tensor([x], dtype=dt, device=self._device())
        red = {"sum": self._pg.ReduceOp.SUM, "max": self._pg.ReduceOp.MAX, "min": self._pg.ReduceOp.MIN}[op]
        self._pg.all_reduce(t, op=red)
        return t.item()

    def gather(self, x: float | int) -> list:
        """Every rank's value, in rank order, on every rank."""
        if not self._pg:
            return [x]
        import torch

        dt = torch.float64 if isinstance(x, float) else torch.int64
        out = [torch.zeros(1, dtype=dt, device=self._device()) for _ in range(self.world)]
        self._pg.all_gather(out, torch.tensor([x], dtype=dt, device=self._device()))
        return [t.item() for t in out]

    def close(self) -> None:
        if self._pg:
            self._pg.destroy_process_group()
            self._pg = None


def sharded_total(dist: Dist, count_shard) -> tuple[int, int]:
    """(local shard count, total over ranks): count_shard(shard, nshards) -> int
    runs this rank's shard; the totals are summed with one all-reduce."""
    local = int(count_shard(dist.rank, dist.world))
    if local < 0 or local >= 1 << 63:
        raise ValueError(f"shard count {local} does not fit the int64 all-reduce")
    return local, int(dist.allreduce(local, "sum"))


__all__ = ["Dist", "sharded_total"]
