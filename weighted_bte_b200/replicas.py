"""Multi-GPU plumbing of the decryption service: replicas only.

Batches and requests are independent and the key material is read-only, so
N GPUs run N replicas, one process per GPU, each with its own copy of the
keys and its own requests; no collective touches the data path.  The process
group (NCCL on GPUs, gloo on CPU) only aligns the ranks around a timed region
and takes the maximum of the ranks' times.  Requests are dealt to replicas
round-robin.
"""
from __future__ import annotations

import datetime
import os
from dataclasses import dataclass
from typing import List, Sequence, TypeVar

T = TypeVar("T")


@dataclass
class Ranks:
    rank: int
    world: int
    local_rank: int

    @property
    def leader(self) -> bool:
        return self.rank == 0

    def barrier(self):
        if self.world > 1:
            import torch.distributed as dist

            dist.barrier()

    def max(self, x: float) -> float:
        """The maximum of x over the ranks (every rank gets it)."""
        if self.world == 1:
            return float(x)
        import torch
        import torch.distributed as dist

        device = "cuda" if dist.get_backend() == "nccl" else "cpu"
        t = torch.tensor([float(x)], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def seed(self, base: int) -> int:
        """A per-replica seed: distinct inputs on every rank."""
        return base + 7919 * self.rank

    def share(self, items: Sequence[T]) -> List[T]:
        """This replica's requests: items rank, rank + world, ..."""
        return list(items[self.rank :: self.world])

    def close(self):
        if self.world > 1:
            import torch.distributed as dist

            dist.barrier()
            dist.destroy_process_group()


def init(backend: str = "nccl", timeout_s: int = 600) -> Ranks:
    """Ranks from the launcher's environment (RANK, WORLD_SIZE, LOCAL_RANK,
    MASTER_ADDR / MASTER_PORT); joins the process group when world > 1."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch.distributed as dist

        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return Ranks(rank, world, local)
