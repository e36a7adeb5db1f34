"""Member sharding across ranks, on CPU with the gloo backend (world size 2).

The assignment is computed independently by every rank and must agree, cover every member once
and balance the footprint; the job's time is the max over ranks; results gather in rank order."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from gschism_b200.shard import gather_results, max_over_ranks, shard_members


def test_shard_members_balanced_and_complete():
    w = [5, 3, 8, 1, 1, 9, 4, 4, 2, 7]
    s = shard_members(w, 3)
    flat = sorted(i for part in s for i in part)
    assert flat == list(range(len(w)))
    loads = [sum(w[i] for i in part) for part in s]
    assert max(loads) - min(loads) <= max(w)
    assert shard_members(w, 1) == [list(range(len(w)))]
    with pytest.raises(ValueError):
        shard_members(w, 0)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, weights, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        mine = shard_members(weights, world)[rank]
        # stand-in for the rank's device time: proportional to its share of the work
        t = float(sum(weights[i] for i in mine))
        tmax = max_over_ranks(t, dist)
        everyone = gather_results({"rank": rank, "members": mine}, dist)
        q.put((rank, mine, tmax, everyone))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_agree_on_shards_and_time():
    weights = [40, 10, 25, 25, 5, 30, 15]
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, weights, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    out.sort()
    expect = shard_members(weights, world)
    for rank, mine, tmax, everyone in out:
        assert mine == expect[rank]
        assert tmax == max(sum(weights[i] for i in s) for s in expect)
        assert [e["members"] for e in everyone] == expect
    assert sorted(i for s in expect for i in s) == list(range(len(weights)))
