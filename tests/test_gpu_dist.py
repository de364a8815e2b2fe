"""GPU test of the instance-sharded batched solve (hprqp_b200.dist.
solve_batch_sharded), end to end: two ranks on a gloo process group split a
family by the greedy cost rule, each solves its shard with one batched
solve, and rank 0 gathers the results in the original order.  They must be
the results of one unsharded batched solve of the whole family.

The two ranks share this run's single GPU.  Their kernels never wait on one
another (the only exchange is the host-side gather over gloo), so sharing a
device is safe; with N GPUs each rank would use its own.
"""
import os
import socket

import numpy as np
import pytest

from hprqp_b200 import HPRQP_parameters
from hprqp_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _families():
    return {
        "qap": ([W.qap_instance(n, 40 + n) for n in (6, 9, 12, 17, 23, 8)], "QAP"),
        "lasso": (W.lasso_family(6, m=200, n=1000, start=77), "LASSO"),
    }


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, name, out):
    import torch.distributed as td

    from hprqp_b200 import dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    td.init_process_group("gloo", rank=rank, world_size=world)
    try:
        models, ptype = _families()[name]
        res = dist.solve_batch_sharded(models, HPRQP_parameters(verbose=False, problem_type=ptype), device=0)
        td.barrier()
        if rank == 0:
            out.put([(r.status, r.iter, r.primal_obj, r.x) for r in res])
        else:
            out.put(None if res is None else "rank 1 got results")
    finally:
        td.destroy_process_group()


@pytest.mark.parametrize("name", ["qap", "lasso"])
def test_sharded_batch_equals_one_batch(name):
    import torch.multiprocessing as mp

    from hprqp_b200.batch import solve_batch
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, name, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = [q.get(timeout=600) for _ in range(2)]
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert None in got  # rank 1 returns nothing
    sharded = next(g for g in got if g is not None)
    models, ptype = _families()[name]
    whole = solve_batch(models, HPRQP_parameters(verbose=False, problem_type=ptype))
    assert len(sharded) == len(models)
    for (st, it, obj, x), r in zip(sharded, whole):
        assert st == r.status == "OPTIMAL"
        # every reduction of the batched engines is per instance (segmented, in a
        # fixed order), so an instance's solve does not depend on the batch it
        # is in: the same iterations, objective and solution
        assert it == r.iter, (it, r.iter)
        assert abs(obj - r.primal_obj) <= 1e-12 * (1 + abs(r.primal_obj)), (obj, r.primal_obj)
        assert np.max(np.abs(x - r.x)) <= 1e-12 * max(1.0, np.max(np.abs(r.x)))
