"""Sharding of independent systems across ranks (host logic; gloo, world size 2, CPU):
every rank derives the same assignment, the subsets cover every system exactly once,
the load is balanced to within the largest single cost, and the job time is the
maximum over ranks."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from fenzi_b200.shard import lpt_assign, max_over_ranks, route_online

COSTS = [3 * n * s for n, s in zip([648, 6000, 1200, 3300, 900, 5100, 2400, 777, 4100, 1500, 2950],
                                   [100, 100, 100, 100, 100, 100, 100, 100, 100, 100, 100])]


def test_lpt_single_rank_and_balance():
    assert lpt_assign([5, 1, 3], 1) == [[0, 1, 2]]
    parts = lpt_assign(COSTS, 3)
    flat = sorted(i for p in parts for i in p)
    assert flat == list(range(len(COSTS)))
    loads = [sum(COSTS[i] for i in p) for p in parts]
    assert max(loads) - min(loads) <= max(COSTS)
    with pytest.raises(ValueError):
        lpt_assign(COSTS, 0)


def test_online_routing_covers_and_balances():
    parts = route_online(COSTS, 3)
    assert sorted(i for p in parts for i in p) == list(range(len(COSTS)))
    assert all(p == sorted(p) for p in parts)  # arrival order kept per rank
    loads = [sum(COSTS[i] for i in p) for p in parts]
    assert max(loads) - min(loads) <= max(COSTS)
    assert route_online(COSTS, 1) == [list(range(len(COSTS)))]
    # online: a job's rank does not depend on later arrivals
    assert [route_online(COSTS[:k + 1], 3) for k in range(len(COSTS))][-1] == parts
    for k in range(1, len(COSTS)):
        head = route_online(COSTS[:k], 3)
        assert all(set(h) <= set(p) for h, p in zip(head, parts))


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
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    mine = lpt_assign(COSTS, world)[rank]
    gathered = [None] * world
    dist.all_gather_object(gathered, mine)
    routed = [None] * world
    dist.all_gather_object(routed, route_online(COSTS, world)[rank])
    t = max_over_ranks(1.0 + rank, dist)
    dist.destroy_process_group()
    q.put((rank, gathered, t, routed))


def test_sharding_over_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, gathered, t, routed in out:
        assert gathered == lpt_assign(COSTS, 2)  # every rank sees the same split
        assert routed == route_online(COSTS, 2)  # and the same routing of the stream
        assert t == 2.0                          # the slowest rank's time
    parts = out[0][1]
    assert sorted(parts[0] + parts[1]) == list(range(len(COSTS)))
    assert not set(parts[0]) & set(parts[1])
