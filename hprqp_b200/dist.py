"""Multi-GPU plumbing: one process per GPU, torch.distributed for the
host-side collectives only.

A single HPR solve does not shard (every iteration would need all-gathers
of w_bar, tempv and y_bar between ranks), so N GPUs run N independent
solves: replicas of one instance (bench.py) or disjoint slices of a batched
family (`solve_batch_sharded`).  Nothing on the data path crosses GPUs; the
only collectives are the max-over-ranks of a timing and the gather of the
per-instance results to rank 0.  The same code runs on `gloo` (CPU) and
`nccl` (GPU) process groups.
"""
from __future__ import annotations

import numpy as np


def shard(costs, rank: int, world: int):
    """Indices of the instances rank `rank` of `world` solves: a greedy
    longest-processing-time split of `costs` (one per instance, e.g. its
    nonzeros), so every rank gets about the same work.  Deterministic: every
    rank computes the same assignment without communicating."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad rank / world size")
    order = sorted(range(len(costs)), key=lambda k: (-float(costs[k]), k))
    load = [0.0] * world
    owner = [0] * len(costs)
    for k in order:
        r = min(range(world), key=lambda q: (load[q], q))
        owner[k] = r
        load[r] += float(costs[k])
    return [k for k in range(len(costs)) if owner[k] == rank]


def max_over_ranks(value: float, device=None) -> float:
    """max of `value` over all ranks (the job's time is the slowest rank's);
    the value itself when no process group is initialised."""
    import torch
    import torch.distributed as td
    if not (td.is_available() and td.is_initialized()):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    td.all_reduce(t, op=td.ReduceOp.MAX)
    return float(t.item())


def gather_to_root(obj):
    """List of every rank's `obj` on rank 0 (rank order), None elsewhere."""
    import torch.distributed as td
    if not (td.is_available() and td.is_initialized()):
        return [obj]
    out = [None] * td.get_world_size() if td.get_rank() == 0 else None
    td.gather_object(obj, out, dst=0)
    return out


def instance_cost(model) -> float:
    """Work estimate of one instance: its nonzeros (data matrix, constraint
    matrix and an n_k^3 term for a dense QAP operator)."""
    q = getattr(model, "Q", None)
    cost = float(getattr(model.A, "nnz", 0) or 0)
    a = getattr(q, "A", None)
    if a is not None and hasattr(a, "nnz"):
        cost += float(a.nnz)
    elif a is not None:
        n = np.asarray(a).shape[0]
        cost += float(n) ** 3
    return max(cost, 1.0)


def solve_batch_sharded(models, params=None, initial_x=None, sigma0=None, device=0):
    """Batched solve of a family split across the ranks of the initialised
    process group: each rank solves its shard with one `solve_batch` on its
    own GPU; rank 0 returns the results in the original order, the other
    ranks None."""
    import torch.distributed as td

    from .batch import solve_batch
    world = td.get_world_size() if td.is_initialized() else 1
    rank = td.get_rank() if td.is_initialized() else 0
    mine = shard([instance_cost(m) for m in models], rank, world)
    res = []
    if mine:
        x0 = None if initial_x is None else [initial_x[k] for k in mine]
        s0 = None if sigma0 is None else [sigma0[k] for k in mine]
        res = solve_batch([models[k] for k in mine], params, initial_x=x0, sigma0=s0, device=device)
    parts = gather_to_root([(k, r) for k, r in zip(mine, res)])
    if parts is None:
        return None
    out = [None] * len(models)
    for part in parts:
        for k, r in part:
            out[k] = r
    return out
