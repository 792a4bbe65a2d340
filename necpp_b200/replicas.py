"""Independent replicas, one process per GPU.

A single solve of the thin-wire hot path fits one GPU, so runs on N GPUs are N
independent replicas: no collective touches the data path.  The only
exchange is after the timed region, where the ranks agree on the slowest
rank's time and on the total work done, so that a whole-job rate is the units
of all ranks divided by the time of the slowest.
"""
import os


def rank_env(env=None):
    """(rank, world_size, local_rank) from the launcher's environment."""
    env = os.environ if env is None else env
    return int(env.get("RANK", "0")), int(env.get("WORLD_SIZE", "1")), int(env.get("LOCAL_RANK", "0"))


def _reduce(values, op, device):
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return [float(v) for v in values]
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=op)
    return [float(v) for v in t.cpu().tolist()]


def max_over_ranks(x, device="cpu"):
    """The largest x over all ranks (x itself without a process group)."""
    import torch.distributed as dist
    return _reduce([x], dist.ReduceOp.MAX, device)[0]


def whole_job_rate(units, seconds, device="cpu"):
    """Units processed by all ranks / the slowest rank's seconds.

    Every rank must call this at the same point (it is one collective for the
    sum and one for the max, in that order on every rank)."""
    import torch.distributed as dist
    total = _reduce([units], dist.ReduceOp.SUM, device)[0]
    slowest = _reduce([seconds], dist.ReduceOp.MAX, device)[0]
    if not slowest > 0:
        raise ValueError("whole_job_rate: non-positive time")
    return total / slowest, total, slowest


def partition_by_cost(costs, world, rank):
    """Indices of the units this rank solves when independent units of
    uneven cost (e.g. N^3 of each problem of a batched sweep) are shared
    out: largest first, each to the rank whose total is smallest so far
    (ties to the lowest rank).  The most loaded rank then exceeds the
    average by less than the cost of one unit.  Every rank computes the
    same assignment, so no exchange is needed."""
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    loads = [0.0] * world
    mine = []
    for i in order:
        r = min(range(world), key=lambda q: (loads[q], q))
        loads[r] += float(costs[i])
        if r == rank:
            mine.append(i)
    return sorted(mine)
