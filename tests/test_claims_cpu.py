"""The served stream shared by several serving processes through
placement.ClaimQueue (one process per GPU): two gloo ranks on CPU claim from
one store counter while they have room -- every request is claimed exactly
once, in arrival order per rank, and a rank that finishes its work sooner
claims more of the stream."""
import json
import os
import socket
import time

import pytest
import torch.multiprocessing as mp

from b200lbm import placement


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _reqs(n):
    return [dict(rid=i, arrival=0.0, steps=40 + 20 * (i % 3)) for i in range(n)]


def _worker(rank, ws, port, out, speed):
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=ws)
    q = placement.ClaimQueue(_reqs(40), store=placement.default_store(), key="test-claims")
    dist.barrier()
    got = []
    while True:
        r = q.claim()
        if r is None:
            break
        got.append(r["rid"])
        time.sleep(0.002 * r["steps"] / 40 * speed[rank])  # the time the GPU would spend on it
    dist.barrier()
    with open(os.path.join(out, f"r{rank}.json"), "w") as f:
        json.dump(got, f)
    dist.destroy_process_group()


@pytest.mark.parametrize("speed", [(1.0, 1.0), (1.0, 4.0)])
def test_two_ranks_claim_every_request_once(tmp_path, speed):
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, str(tmp_path), speed)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = [json.load(open(tmp_path / f"r{r}.json")) for r in range(2)]
    assert sorted(got[0] + got[1]) == list(range(40))
    assert not set(got[0]) & set(got[1])
    for g in got:
        assert g == sorted(g) and len(g) > 0
    if speed[1] > speed[0]:
        assert len(got[0]) > len(got[1])  # the faster rank took more of the stream


def test_local_queue_claims_in_order():
    q = placement.ClaimQueue(list(reversed(_reqs(5))))
    assert q.peek()["rid"] == 0
    assert [q.claim()["rid"] for _ in range(5)] == [0, 1, 2, 3, 4]
    assert q.claim() is None and q.exhausted() and q.peek() is None
