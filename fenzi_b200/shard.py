"""Sharding of independent systems (the batched ensemble and served jobs) across GPUs.

A single system does not shard (one system per GPU, replicas only); a set of
independent systems does, with no per-step exchange: each rank takes a subset and runs
it as its own batch or serving loop.  A known set (the ensemble) is split by
longest-processing-time-first greedy assignment on a per-system cost (atoms x steps);
a stream of served jobs is routed online, each arrival to the least-loaded rank.  Both
are identical on every rank because they depend only on the costs.
"""
from __future__ import annotations


def lpt_assign(costs, nranks: int):
    """Assigns item i (cost costs[i]) to ranks: items in decreasing cost, each to the
    rank with the smallest load so far (lowest rank on ties).  Returns one sorted list
    of item indices per rank."""
    if nranks < 1:
        raise ValueError("nranks must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    load = [0.0] * nranks
    out = [[] for _ in range(nranks)]
    for i in order:
        r = min(range(nranks), key=lambda k: (load[k], k))
        out[r].append(i)
        load[r] += float(costs[i])
    return [sorted(x) for x in out]


def route_online(costs, nranks: int):
    """Routes a stream of jobs (in arrival order, cost costs[i] = atoms x steps) to
    ranks as they arrive: each job to the rank with the least work routed to it so far
    (lowest rank on ties).  The rule needs no knowledge of later jobs, and every rank
    derives the same routing from the same stream.  Returns the job indices per rank."""
    if nranks < 1:
        raise ValueError("nranks must be >= 1")
    load = [0.0] * nranks
    out = [[] for _ in range(nranks)]
    for i, c in enumerate(costs):
        r = min(range(nranks), key=lambda k: (load[k], k))
        out[r].append(i)
        load[r] += float(c)
    return out


def max_over_ranks(value: float, dist=None, device=None) -> float:
    """The largest value over the ranks of the default process group (the job's time
    is that of its slowest rank); the value itself without a process group."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
