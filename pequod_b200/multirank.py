"""One process per GPU: the host-side plumbing of multi-GPU runs.

Ensembles shard: the members of one batched-Helmholtz workload and the
requests of one serving stream are independent, so they are partitioned
across the ranks as whole members, balanced by their work (ii * jj * L, and
times the step count for a serving request), with no exchange while they
run; only the measurement's collectives follow (the slowest rank's time,
the serving statistics over all ranks).  A single domain does not shard
without an exchange step, so single runs are independent replicas (one per
rank, each with its own seed).  The process group is NCCL on GPUs; the same
functions run on gloo (CPU) in the tests.
"""
from __future__ import annotations

import datetime
import os

import numpy as np


def env_ranks():
    """(rank, world, local_rank) from the launcher's environment."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(world: int, backend: str = "nccl", timeout_s: float = 300.0):
    """The default process group when world > 1 (None otherwise)."""
    if world <= 1:
        return None
    import torch.distributed as dist

    if not dist.is_initialized():
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return dist


def rank_seed(base: int, rank: int) -> int:
    """Each replica draws its own workload."""
    return base + rank


def partition(weights, world: int):
    """Split items of the given work weights over `world` ranks: the longest
    processing time first rule (heaviest item to the least-loaded rank, ties
    to the lower index), deterministic.  Returns, per rank, the sorted item
    indices; the heaviest rank carries at most the mean load plus the
    heaviest item."""
    load = [0.0] * world
    parts = [[] for _ in range(world)]
    order = sorted(range(len(weights)), key=lambda k: (-float(weights[k]), k))
    for k in order:
        r = min(range(world), key=lambda q: (load[q], q))
        parts[r].append(k)
        load[r] += float(weights[k])
    return [sorted(p) for p in parts]


def shard(items, weights, rank: int, world: int):
    """This rank's share of `items` (in their original order)."""
    return [items[k] for k in partition(weights, world)[rank]]


def max_over_ranks(dist, values, device=None):
    """Element-wise maximum of a list of floats over the ranks (the slowest
    rank's times); the values unchanged without a process group."""
    if dist is None:
        return [float(v) for v in values]
    import torch

    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.cpu().tolist()]


def gather_lists(dist, items):
    """The concatenation, in rank order, of every rank's list."""
    if dist is None:
        return list(items)
    out = [None] * dist.get_world_size()
    dist.all_gather_object(out, list(items))
    return [x for part in out for x in part]


def serving_summary(done):
    """Latency percentiles and throughput of finished requests, each
    (latency_s, cell_layer_steps, finish_s) with finish times on one clock
    origin per rank: p50 and p99 over all requests, and the total work over
    the longest span."""
    lat = np.array([d[0] for d in done], dtype=np.float64)
    work = float(sum(d[1] for d in done))
    span = max(d[2] for d in done)
    return {"p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "runs": len(done), "throughput": work / span}


def close(dist):
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
