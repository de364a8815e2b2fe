"""GPU test of the schedule cache (the autotuner's timed choices kept per
process by sparsity signature): a second handle that loads a problem of the
same pattern takes the first one's schedules without timing, builds only the
chosen format copies, and, the kernels being deterministic, reproduces the
first solve bit for bit.  With HPRQP_SCHED_CACHE=0 every handle times again.
"""
import os

import numpy as np
import pytest

from hprqp_b200 import HPRQP_parameters, Solver
from hprqp_b200 import workloads as W

pytestmark = pytest.mark.gpu


def solve_once(model, ptype):
    s = Solver().load(model)
    p = HPRQP_parameters(verbose=False, problem_type=ptype, max_iter=300)
    r = s.solve(p)
    st = s.profile_iterations(HPRQP_parameters(verbose=False, problem_type=ptype), iters=2)
    s.close()
    return r, [q["threads_per_row"] for q in st["passes"]]


@pytest.mark.parametrize("name", ["lasso", "grid"])
def test_second_handle_reuses_the_schedules(name):
    model, ptype = ((W.lasso(m=400, n=60000, seed=33, mu=5.0), "LASSO") if name == "lasso"
                    else (W.grid_qp(N=120), "QP"))
    r1, s1 = solve_once(model, ptype)
    r2, s2 = solve_once(model, ptype)
    assert s1 == s2
    assert r1.iter == r2.iter and np.array_equal(r1.x, r2.x)
    # the cache only skips timing: without it the solve is the same method
    os.environ["HPRQP_SCHED_CACHE"] = "0"
    try:
        r3, _ = solve_once(model, ptype)
    finally:
        os.environ.pop("HPRQP_SCHED_CACHE", None)
    assert r3.status == r1.status
    assert abs(r3.primal_obj - r1.primal_obj) <= 1e-9 * (1 + abs(r1.primal_obj))
