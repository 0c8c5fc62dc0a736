"""Multi-rank (replicas) host logic on CPU with gloo, world_size 2: member
partition and whole-job throughput aggregation (sum of work / max time)."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from torchannel_b200.ensemble import make_members, partition


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import torch.distributed as dist
    from torchannel_b200.ensemble import aggregate
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mine = partition(16, world, rank)
        members = make_members(16, seed=3)
        pts = sum(members[m]["nx"] * members[m]["ny"] * members[m]["nz"] for m in mine) * 10
        ms = 100.0 + 50.0 * rank            # rank 1 is the slowest
        value, tot_pts, max_ms = aggregate(pts, ms)
        q.put((rank, mine, value, tot_pts, max_ms))
    finally:
        dist.destroy_process_group()


def test_partition_covers_members_once():
    for world in (1, 2, 3, 4, 8):
        seen = sorted(m for r in range(world) for m in partition(16, world, r))
        assert seen == list(range(16))


def test_members_are_seeded_and_in_range():
    a, b = make_members(16, seed=1), make_members(16, seed=1)
    assert a == b
    for m in a:
        assert m["nx"] in (64, 96, 128) and m["ny"] in (64, 96, 128) and m["nz"] in (48, 64, 96)
        assert 2000 <= m["Re"] <= 5600 and 2.2 <= m["gamma"] <= 2.8


@pytest.mark.timeout(120)
def test_gloo_two_rank_aggregate():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=90) for _ in range(world))
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    members = make_members(16, seed=3)
    total = sum(m["nx"] * m["ny"] * m["nz"] for m in members) * 10
    for rank, mine, value, tot_pts, max_ms in res:
        assert tot_pts == total
        assert max_ms == 150.0
        assert abs(value - total / 0.150) < 1e-6 * value
    assert sorted(res[0][1] + res[1][1]) == list(range(16))
