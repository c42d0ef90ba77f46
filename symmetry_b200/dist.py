"""Host side of running the library on several GPUs of one node.

The per-timestep update does not shard: domains and served jobs are
independent, so N GPUs run N replicas, one process per GPU, and no kernel
exchanges data with another GPU.  What crosses ranks is host-side
bookkeeping only, through torch.distributed (NCCL between GPUs; the same
functions run on gloo between CPU processes, which is how they are tested):

  ReplicaEnv       rank, world size and local device from the launcher's
                   environment (RANK / WORLD_SIZE / LOCAL_RANK)
  max_over_ranks   the slowest rank's device time (every timed number is the
                   max over ranks, never a wall clock)
  sum_over_ranks   totals such as node updates or retired jobs
  aggregate_mlups  whole-job MLUPS = all ranks' node updates / max time
  dispatch_jobs    which rank serves which job: each job goes to the rank
                   with the least HBM footprint assigned so far (ties to the
                   lower rank), in arrival order -- deterministic, so every
                   rank computes the same assignment without communicating

Every rank calls the collective functions in the same order with the same
arguments' shapes; a rank that skips one leaves the others waiting until the
process group's timeout.
"""
from __future__ import annotations

import os
from dataclasses import dataclass
from typing import List, Sequence


@dataclass(frozen=True)
class ReplicaEnv:
    rank: int = 0
    world: int = 1
    local: int = 0

    @staticmethod
    def from_environ(env=None) -> "ReplicaEnv":
        e = os.environ if env is None else env
        return ReplicaEnv(int(e.get("RANK", "0")), int(e.get("WORLD_SIZE", "1")), int(e.get("LOCAL_RANK", "0")))


def _reduce(torch, dist, value: float, op, device):
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=op)
    return float(t.item())


def max_over_ranks(torch, dist, value: float, device="cpu") -> float:
    """The largest `value` over all ranks (e.g. the device time of the slowest)."""
    return _reduce(torch, dist, value, dist.ReduceOp.MAX if dist is not None else None, device)


def sum_over_ranks(torch, dist, value: float, device="cpu") -> float:
    """The sum of `value` over all ranks."""
    return _reduce(torch, dist, value, dist.ReduceOp.SUM if dist is not None else None, device)


def aggregate_mlups(node_updates: float, max_ms: float) -> float:
    """Whole-job throughput: node updates of all ranks over the slowest rank's
    time (ms), in millions of updates per second."""
    if not max_ms > 0.0:
        raise ValueError("max_ms must be positive")
    return node_updates / (max_ms / 1e3) / 1e6


def dispatch_jobs(footprints: Sequence[int], world: int) -> List[int]:
    """Rank of each job, in arrival order: the rank with the least footprint
    assigned so far (the lower rank on a tie)."""
    if world < 1:
        raise ValueError("world must be >= 1")
    load = [0] * world
    out = []
    for f in footprints:
        r = min(range(world), key=lambda k: (load[k], k))
        out.append(r)
        load[r] += int(f)
    return out
