"""CPU tests of the multi-process plumbing (hprqp_b200.dist) on a gloo
process group of world size 2, spawned here on 127.0.0.1: the instance
split covers every instance once and balances the work, the max over ranks
is the slowest rank's value, and the gather returns every rank's part in
rank order.  No GPU is involved (the solves themselves are single-GPU and
tested in the gpu suite)."""
import os
import socket

import numpy as np
import pytest

from hprqp_b200 import dist
from hprqp_b200 import workloads as W


def test_shard_covers_each_instance_once_and_balances():
    rng = np.random.default_rng(0)
    costs = rng.integers(1, 1000, size=257).astype(float)
    for world in (1, 2, 3, 8):
        parts = [dist.shard(costs, r, world) for r in range(world)]
        flat = sorted(k for p in parts for k in p)
        assert flat == list(range(len(costs)))
        loads = [costs[p].sum() for p in parts]
        assert max(loads) - min(loads) <= costs.max()  # greedy LPT bound
    with pytest.raises(ValueError):
        dist.shard(costs, 2, 2)


def test_instance_cost_orders_families():
    small, big = W.qap_instance(8, 1), W.qap_instance(16, 1)
    assert dist.instance_cost(big) > dist.instance_cost(small) > 0
    assert dist.instance_cost(W.small_lasso()) > 0


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import torch.distributed as td
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    td.init_process_group("gloo", rank=rank, world_size=world)
    try:
        costs = [5.0, 1.0, 3.0, 3.0, 2.0, 8.0]
        mine = dist.shard(costs, rank, world)
        m = dist.max_over_ranks(10.0 + rank)
        parts = dist.gather_to_root((rank, mine))
        td.barrier()
        if rank == 0:
            out.put((m, parts))
        else:
            out.put((m, None))
    finally:
        td.destroy_process_group()


def test_gloo_world_size_2():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert all(m == 11.0 for m, _ in got)
    parts = next(p for _, p in got if p is not None)
    assert [r for r, _ in parts] == [0, 1]
    flat = sorted(k for _, ks in parts for k in ks)
    assert flat == list(range(6))
