"""Replica plumbing across ranks on CPU (gloo, world size 2): the unit shards
cover every unit once, the timing is the max over ranks, and the whole-job rate
is all units over the slowest rank's time."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from moao_b200.replicas import max_over_ranks, shard, sum_over_ranks, whole_job_rate


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    units = list(range(11))
    mine = shard(units, rank, world)
    secs = 1.0 + rank          # rank 1 is the slower one
    out = {"rank": rank, "mine": mine, "max": max_over_ranks(secs, dist),
           "sum": sum_over_ranks(len(mine), dist),
           "rate": whole_job_rate(len(mine), secs, dist)}
    dist.barrier()
    dist.destroy_process_group()
    q.put(out)


def test_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted([q.get(timeout=120) for _ in procs], key=lambda d: d["rank"])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert sorted(res[0]["mine"] + res[1]["mine"]) == list(range(11))
    for r in res:
        assert r["max"] == 2.0
        assert r["sum"] == 11
        assert r["rate"] == pytest.approx(11 / 2.0)


def test_single_process_fallbacks():
    assert shard([1, 2, 3], 0, 1) == [1, 2, 3]
    assert max_over_ranks(3.5) == 3.5
    assert whole_job_rate(4, 2.0) == 2.0
    with pytest.raises(ValueError):
        shard([1], 2, 2)
