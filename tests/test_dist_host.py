"""Host side of multi-GPU runs (replicas only), as two gloo ranks on CPU.

Each GPU runs its own replica of the batch or its own share of the served
jobs; only host-side numbers cross ranks.  These tests run the same functions
the bench uses between two CPU processes: the slowest rank's time, the sum of
the node updates, the whole-job MLUPS built from them, and the job dispatch
every rank computes without communicating.
"""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from symmetry_b200.dist import ReplicaEnv, aggregate_mlups, dispatch_jobs, max_over_ranks, sum_over_ranks


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        env = ReplicaEnv.from_environ()
        # rank r timed (r + 1) * 10 ms over its replica of 1,000 node updates
        t = max_over_ranks(torch, dist, (env.rank + 1) * 10.0)
        n = sum_over_ranks(torch, dist, 1000.0)
        jobs = dispatch_jobs([5, 3, 8, 1, 1, 7], env.world)
        dist.barrier()
        q.put((env.rank, env.world, env.local, t, n, aggregate_mlups(n, t), jobs))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_agree_on_the_aggregates():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    out.sort()
    for rank, (r, w, local, t, n, v, jobs) in enumerate(out):
        assert (r, w, local) == (rank, 2, rank)
        assert t == 20.0                      # the slowest rank's time, on every rank
        assert n == 2000.0                    # both replicas' node updates
        assert v == pytest.approx(2000.0 / 0.020 / 1e6)
        assert jobs == out[0][6]              # the same dispatch on every rank


def test_single_process_needs_no_process_group():
    assert max_over_ranks(torch, None, 3.5) == 3.5
    assert sum_over_ranks(torch, None, 7.0) == 7.0
    assert ReplicaEnv.from_environ({}) == ReplicaEnv(0, 1, 0)


def test_dispatch_balances_footprint_in_arrival_order():
    # least assigned footprint first, lower rank on a tie
    assert dispatch_jobs([5, 3, 8, 1, 1, 7], 2) == [0, 1, 1, 0, 0, 0]
    assert dispatch_jobs([4, 4, 4, 4], 4) == [0, 1, 2, 3]
    assert dispatch_jobs([], 3) == []
    with pytest.raises(ValueError):
        dispatch_jobs([1], 0)
    with pytest.raises(ValueError):
        aggregate_mlups(10.0, 0.0)
