"""Replica runs over several GPUs (one process per GPU): a single dam break
is not partitioned, each rank steps its own scene (or, for a batch of
independent scenes, its size-balanced share of them), and the ranks only
agree on the timing.

  * every rank gets the same scene with its own lattice seed;
  * the timed region is bracketed by a barrier and the device
    synchronisation on every rank;
  * the reported time is the maximum over ranks, the throughput the total
    particle-steps of all ranks over that time.

The rendezvous reads RANK / WORLD_SIZE / LOCAL_RANK / MASTER_* from the
environment, as torch.distributed.run sets them.
"""
from __future__ import annotations

import datetime
import os
from dataclasses import dataclass
from typing import Optional

SEED_STRIDE = 1000


@dataclass
class Replicas:
    rank: int = 0
    world: int = 1
    local: int = 0
    dist: Optional[object] = None     # torch.distributed when world > 1
    device: Optional[object] = None   # where the reduction tensor lives

    def barrier(self) -> None:
        if self.dist is not None:
            self.dist.barrier()

    def max_over_ranks(self, value: float) -> float:
        """The largest `value` over all ranks (every rank gets it)."""
        if self.dist is None:
            return float(value)
        import torch
        t = torch.tensor([float(value)], dtype=torch.float64, device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def seed(self, base_seed: int) -> int:
        """The lattice seed of this rank's replica."""
        return int(base_seed) + SEED_STRIDE * self.rank

    def close(self) -> None:
        if self.dist is not None:
            self.dist.barrier()
            self.dist.destroy_process_group()
            self.dist = None


def assign_scenes(sizes, world: int):
    """Size-balanced assignment of independent scenes to `world` ranks
    (longest processing time first: each scene, largest first, goes to the
    rank with the fewest particles so far; ties to the lower rank). Every
    rank computes the same assignment from the same sizes, so the ranks need
    no exchange. Returns, per rank, its scene indices in increasing order."""
    order = sorted(range(len(sizes)), key=lambda i: (-int(sizes[i]), i))
    load = [0] * world
    out = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        out[r].append(i)
        load[r] += int(sizes[i])
    return [sorted(v) for v in out]


def env_ranks():
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend: str = "nccl", timeout_s: float = 120.0) -> Replicas:
    """Joins the process group when WORLD_SIZE > 1 (nccl: one GPU per local
    rank; gloo: CPU tensors), with a bounded timeout so that ranks waiting on
    a missing peer fail instead of hanging."""
    rank, world, local = env_ranks()
    r = Replicas(rank=rank, world=world, local=local)
    if world <= 1:
        return r
    import torch
    import torch.distributed as dist
    os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
    kw = {"timeout": datetime.timedelta(seconds=timeout_s)}
    if backend == "nccl":
        torch.cuda.set_device(local)
        kw["device_id"] = torch.device("cuda", local)
        r.device = torch.device("cuda", local)
    else:
        r.device = torch.device("cpu")
    dist.init_process_group(backend, **kw)
    r.dist = dist
    return r
