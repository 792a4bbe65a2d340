"""Replica bookkeeping on two gloo ranks (CPU): the whole-job rate is the
units of all ranks over the slowest rank's time, the same on every rank."""
import os
import socket

import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    import datetime

    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        from necpp_b200.replicas import max_over_ranks, rank_env, whole_job_rate
        r, w, lr = rank_env()
        # rank r did (r + 1) * 3 solves in (r + 1) * 0.5 s
        rate, total, slowest = whole_job_rate((r + 1) * 3, (r + 1) * 0.5)
        m = max_over_ranks(10.0 + r)
        out.put((r, w, lr, rate, total, slowest, m))
    finally:
        dist.destroy_process_group()


def test_whole_job_rate_two_gloo_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    for r, (rank, world, local, rate, total, slowest, m) in enumerate(res):
        assert (rank, world, local) == (r, 2, r)
        assert total == 9.0 and slowest == 1.0 and rate == 9.0
        assert m == 11.0


def test_single_process_needs_no_group():
    from necpp_b200.replicas import max_over_ranks, whole_job_rate
    assert max_over_ranks(3.0) == 3.0
    assert whole_job_rate(4, 2.0) == (2.0, 4.0, 2.0)
    with pytest.raises(ValueError):
        whole_job_rate(4, 0.0)


def test_partition_by_cost_covers_all_units_evenly():
    import numpy as np
    from necpp_b200.replicas import partition_by_cost
    rng = np.random.default_rng(0)
    n = rng.integers(33, 616, size=1000)
    cost = (n.astype(float)) ** 3
    parts = [partition_by_cost(cost, 4, r) for r in range(4)]
    allidx = sorted(i for p in parts for i in p)
    assert allidx == list(range(1000))
    shares = [cost[p].sum() / cost.sum() for p in parts]
    assert max(shares) - min(shares) < 0.02
    # the largest total exceeds the average by less than one unit's cost
    loads = [cost[p].sum() for p in parts]
    assert max(loads) - cost.sum() / 4 < cost.max()
