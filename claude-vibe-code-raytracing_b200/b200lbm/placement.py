"""Placing independent scenes on several GPUs.

Scenes (batched or served) are independent: nothing crosses between them, so
several GPUs share a workload by taking whole scenes, one process per GPU,
with no collective on the data path.  shard() balances the scenes by weight
(cells x steps, or device footprint) with the longest-processing-time rule:
heaviest first, each to the currently lightest rank; ties go to the lower
rank, so every rank computes the same assignment without communicating.
The only collectives are for reporting: the slowest rank's time
(max_over_ranks) and the work summed over ranks (sum_over_ranks), on
whatever process group is initialised (NCCL on GPUs, gloo in the CPU tests).

A served request stream is not split up front: ClaimQueue hands the requests
out in arrival order through one atomic counter in the process group's
key-value store, and each serving process claims the next request when its
GPU has room for it, so a GPU whose scenes finish early takes more of the
stream (balance by live footprint, not by a static guess).
"""
from __future__ import annotations


def shard(items, world_size, weight):
    """Split `items` over `world_size` ranks; returns a list of per-rank lists
    (each in the items' original order)."""
    if world_size < 1:
        raise ValueError("world_size must be >= 1")
    order = sorted(range(len(items)), key=lambda i: (-weight(items[i]), i))
    load = [0.0] * world_size
    owner = [0] * len(items)
    for i in order:
        r = min(range(world_size), key=lambda k: (load[k], k))
        owner[i] = r
        load[r] += weight(items[i])
    return [[it for i, it in enumerate(items) if owner[i] == r] for r in range(world_size)]


def _reduce(v, op):
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(v)
    dev = "cpu"
    if dist.get_backend() == "nccl":
        dev = f"cuda:{torch.cuda.current_device()}"
    t = torch.tensor([float(v)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=op)
    return float(t.item())


def max_over_ranks(v):
    import torch.distributed as dist
    return _reduce(v, dist.ReduceOp.MAX)


def sum_over_ranks(v):
    import torch.distributed as dist
    return _reduce(v, dist.ReduceOp.SUM)


class ClaimQueue:
    """Requests shared by the serving processes of one job.  Every process
    builds the same list (the same seeded trace); `claim` takes the next
    unclaimed one in arrival order, atomically across processes (the store's
    add), and `peek` shows it without taking it.  With store=None the queue
    is local to one process."""

    def __init__(self, requests, store=None, key="lbm-serve-next"):
        self.requests = sorted(requests, key=lambda r: (r["arrival"], r["rid"]))
        self.store = store
        self.key = key
        self._next = 0

    def _counter(self, add):
        if self.store is None:
            self._next += add
            return self._next
        return int(self.store.add(self.key, add))

    def peek(self):
        i = self._counter(0)
        return self.requests[i] if i < len(self.requests) else None

    def claim(self):
        i = self._counter(1) - 1
        return self.requests[i] if i < len(self.requests) else None

    def exhausted(self):
        return self._counter(0) >= len(self.requests)


def default_store():
    """The key-value store of the initialised default process group (the
    rendezvous store every rank already shares)."""
    from torch.distributed import distributed_c10d
    return distributed_c10d._get_default_store()
