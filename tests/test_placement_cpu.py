"""Multi-GPU placement logic on CPU: world_size-2 gloo ranks shard a seeded
scene list (whole scenes per rank, no data-path collective), agree on the
assignment without communicating, and reduce their timings (max) and work
(sum) -- the same steps bench.py and the server take on N GPUs."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from b200lbm import placement, workloads


def _weight(spec):
    return workloads.cells(spec)


def test_shard_balances_and_covers():
    specs = workloads.scene_specs(64, seed=0)
    parts = placement.shard(specs, 4, _weight)
    assert sorted(id(s) for p in parts for s in p) == sorted(id(s) for s in specs)
    loads = [sum(_weight(s) for s in p) for p in parts]
    assert max(loads) - min(loads) <= max(_weight(s) for s in specs)
    assert placement.shard(specs, 4, _weight) == parts  # deterministic
    assert placement.shard(specs, 1, _weight) == [specs]
    with pytest.raises(ValueError):
        placement.shard(specs, 0, _weight)


def _rank(rank, ws, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=ws)
    try:
        specs = workloads.scene_specs(16, seed=2)
        mine = placement.shard(specs, ws, _weight)[rank]
        idx = [specs.index(s) for s in mine]
        got = [None] * ws
        dist.all_gather_object(got, idx)
        t = placement.max_over_ranks(1.0 + rank)
        w = placement.sum_over_ranks(sum(_weight(s) for s in mine))
        q.put((rank, got, t, w, sum(_weight(s) for s in specs)))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_agree():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, got, t, w, total in res:
        assert sorted(got[0] + got[1]) == list(range(16)) and not set(got[0]) & set(got[1])
        assert t == 2.0
        assert w == total
