"""GPU test of the GPU-side scaling (scale.cu): for a sparse problem above
the size threshold, hprqp_prepare scales on the device; the scaled problem
must be bitwise the host restatement's, so the first iterates of the two
paths are identical (exact equality, not a tolerance)."""
import os

import numpy as np
import pytest
import scipy.sparse as sp

from hprqp_b200 import HPRQP_parameters, Solver
from hprqp_b200 import workloads as W

pytestmark = pytest.mark.gpu


def trace(model, host):
    if host:
        os.environ["HPRQP_HOST_SCALING"] = "1"
    try:
        s = Solver().load(model)
        xt, yt, wt = s.set_trace(30)
        # a pinned row schedule: the autotuner may pick different ones in
        # two runs, and schedules sum rows in different orders
        r = s.solve(HPRQP_parameters(verbose=False, max_iter=30, spmv_mode_Q=1, spmv_mode_A=1))
        s.close()
    finally:
        os.environ.pop("HPRQP_HOST_SCALING", None)
    return r, xt.copy(), yt.copy(), wt.copy()


@pytest.mark.parametrize("N", [120, 200])
def test_gpu_scaling_is_bitwise_the_host_scaling(N):
    m = W.grid_qp(N=N)
    assert m.A.nnz + m.Q.Q.nnz >= 100000  # the GPU path
    r_gpu, xg, yg, wg = trace(m, host=False)
    r_host, xh, yh, wh = trace(m, host=True)
    assert np.array_equal(xg, xh) and np.array_equal(yg, yh) and np.array_equal(wg, wh)
    assert r_gpu.lambda_max_A == r_host.lambda_max_A and r_gpu.lambda_max_Q == r_host.lambda_max_Q
    assert r_gpu.primal_obj == r_host.primal_obj


def test_gpu_scaling_asymmetric_Q_pattern():
    """Q given as its upper triangle: the pattern of Q + Q' is merged on the
    host with index maps (the symmetric-pattern shortcut does not apply)."""
    m = W.grid_qp(N=150)
    m.Q.Q = sp.triu(m.Q.Q).tocsc()  # past the builder's own symmetrisation: the library merges
    assert m.A.nnz + m.Q.Q.nnz >= 100000 and (m.Q.Q != m.Q.Q.T).nnz > 0
    r_gpu, xg, yg, wg = trace(m, host=False)
    r_host, xh, yh, wh = trace(m, host=True)
    assert np.array_equal(xg, xh) and np.array_equal(yg, yh) and np.array_equal(wg, wh)
    assert r_gpu.primal_obj == r_host.primal_obj
